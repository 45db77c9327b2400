// Incident-triangle counts for a vertex subset without a whole-graph pass.
//
// For u in the subset, t(u) = 1/2 * sum_{v in N(u)} |N(u) & N(v)| on the
// symmetric store (no self-loops, no duplicates).  Each subset vertex u is
// a group: N(u) goes into an open-addressing hash set (shared memory when it
// has at most TL_SMEM_LIVE live entries, else a table in global memory that
// stays in L2), and every neighbour list N(v), v in N(u), is streamed block
// by block with 16-byte loads and probed against it.  The work is cut into
// pieces (32 blocks of one N(v)) and units (64 consecutive pieces of one
// group, one CTA pass), so a hub neighbour is spread over many warps and
// CTAs.  Cost: sum over the subset of sum_{v in N(u)} deg(v) entry reads,
// against the whole-graph oriented count the reference's tc_kernel_VC
// (src/algorithm/tc/tc_kernel.cu:3-74) would run; the caller takes the
// whole-graph path when that sum exceeds TL_WHOLE_RATIO passes over the store.
#include <algorithm>
#include <vector>
#include "store.cuh"
#include "prims.cuh"
#include "launch.hpp"

namespace gv {
namespace {

constexpr int TL_THREADS = 256;
constexpr uint32_t TL_PIECE_BLOCKS = 32;                     // blocks of N(v) per piece (one per lane)
constexpr uint32_t TL_UNIT_PIECES = 64;                      // pieces per unit
constexpr uint32_t TL_SMEM_LOG = 14;                         // shared hash: 16384 slots, 64 KB
constexpr uint32_t TL_SMEM_LIVE = (1u << TL_SMEM_LOG) / 2;   // load factor <= 1/2
constexpr int TL_COUNT_CTAS_PER_SM = 3;                      // 64 KB of shared memory each
constexpr double TL_WHOLE_RATIO = 128.0;                     // streamed / stored entries where the paths cross

struct TlGroups {
    const uint32_t *hv;                   // hashed vertex per group
    const unsigned long long *pair_off;   // G + 1: scanned vertices of group g are pair_v[pair_off[g], pair_off[g+1])
    const uint32_t *pair_v;
    const unsigned long long *piece_off;  // P + 1
    const uint32_t *unit_off;             // G + 1
    const unsigned long long *gh_off;     // slot offset of the group's global table (~0: shared memory)
    const uint32_t *tab_log;              // log2 of the table's slots
    uint32_t *gh;                         // global tables
    uint32_t G;
};

__device__ __forceinline__ uint32_t tl_hash(uint32_t w, uint32_t logc) { return (w * 0x9E3779B1u) >> (32 - logc); }

__device__ __forceinline__ void tl_insert(uint32_t *tab, uint32_t logc, uint32_t w, uint32_t *err) {
    const uint32_t mask = (1u << logc) - 1u;
    uint32_t h = tl_hash(w, logc);
    for (uint32_t i = 0; i <= mask; ++i) {
        const uint32_t old = atomicCAS(tab + h, GV_NIL, w);
        if (old == GV_NIL || old == w) return;
        h = (h + 1u) & mask;
    }
    atomicOr(err, 2u);  // table full: live counts and entries disagree
}

__device__ __forceinline__ uint32_t tl_probe(const uint32_t *tab, uint32_t logc, uint32_t w) {
    const uint32_t mask = (1u << logc) - 1u;
    uint32_t h = tl_hash(w, logc);
    for (uint32_t i = 0; i <= mask; ++i) {
        const uint32_t x = tab[h];
        if (x == w) return 1u;
        if (x == GV_NIL) return 0u;
        h = (h + 1u) & mask;
    }
    return 0u;
}

// Pool index of block kb0 + lane of a vertex, GV_NIL past its last block.
__device__ __forceinline__ uint32_t tl_lane_block(const DevGraph &g, uint32_t root, uint32_t kb0, uint32_t nb) {
    const uint32_t k = kb0 + (threadIdx.x & 31u);
    if (k >= nb) return GV_NIL;
    return k == 0 ? root : cbt_block(g.left, g.right, root, k);
}

// Calls f(w) for every live entry of blocks [kb0, kb0 + nblk) of a vertex
// with `fill` used slots.  Block kb0 + r is held in `blk` by lane
// lane_off + r (tl_lane_block of the run starting lane_off blocks earlier).
// The warp reads each block with 16-byte loads (B/4 lanes per block).  Every
// lane of the warp must call it with the same kb0 / lane_off / nblk.
template <typename F>
__device__ __forceinline__ void tl_scan_blocks(const DevGraph &g, uint32_t blk, uint32_t kb0, uint32_t lane_off,
                                               uint32_t nblk, uint32_t fill, F &&f) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lpb = min(32u, g.B >> 2), bpw = 32u / lpb, sub = lane / lpb, sl = lane % lpb;
    for (uint32_t s0 = 0; s0 < nblk; s0 += bpw) {
        const uint32_t kr = s0 + sub;
        const uint32_t b = __shfl_sync(GV_FULL_MASK, blk, (lane_off + kr) & 31u);
        if (kr < nblk) {
            const uint32_t e = ((kb0 + kr) << g.logB) + sl * 4u;
            if (e < fill) {
                const uint4 q = *reinterpret_cast<const uint4 *>(g.pool + ((size_t)b << g.logB) + sl * 4u);
                const uint32_t ev[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (e + j < fill && ev[j] != GV_TOMB) f(ev[j]);
            }
        }
    }
}

__global__ void k_tl_deg(DevGraph g, const uint32_t *__restrict__ hv, uint32_t G, uint2 *__restrict__ du) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < G; i += gridDim.x * blockDim.x) {
        const uint32_t u = hv[i];
        if (u >= g.n) {
            du[i] = make_uint2(GV_NIL, 0u);  // rejected on the host
            continue;
        }
        const uint4 rec = g.vtx[u];
        du[i] = make_uint2(rec.z, rec.y);  // live, fill
    }
}

// Scan lists of the subset groups: pair_v = the live entries of N(u), and per
// entry the pieces its own list takes.  One CTA per group, warps over blocks.
__global__ void __launch_bounds__(TL_THREADS) k_tl_pairs(DevGraph g, TlGroups t, uint32_t *__restrict__ cursor,
                                                         uint32_t *__restrict__ pair_v, uint32_t *__restrict__ pieces,
                                                         unsigned long long *__restrict__ words) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nwarps = TL_THREADS / 32;
    uint32_t *err = reinterpret_cast<uint32_t *>(words + 1);
    unsigned long long blocks = 0;
    for (uint32_t gi = blockIdx.x; gi < t.G; gi += gridDim.x) {
        const uint32_t u = t.hv[gi];
        const uint4 rec = g.vtx[u];
        const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB);
        const unsigned long long p0 = t.pair_off[gi], cap = t.pair_off[gi + 1] - p0;
        for (uint32_t kb = warp * TL_PIECE_BLOCKS; kb < nb; kb += nwarps * TL_PIECE_BLOCKS) {
            const uint32_t blk = tl_lane_block(g, rec.x, kb, nb);
            const uint32_t nblk = min(TL_PIECE_BLOCKS, nb - kb);
            const uint32_t lpb = min(32u, g.B >> 2), bpw = 32u / lpb;
            // one step = bpw blocks; every lane holds up to 4 entries
            for (uint32_t s0 = 0; s0 < nblk; s0 += bpw) {
                uint32_t mine[4];
                uint32_t c = 0;
                tl_scan_blocks(g, blk, kb + s0, s0, min(bpw, nblk - s0), fill, [&](uint32_t w) { mine[c++] = w; });
                uint32_t incl = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t y = __shfl_up_sync(GV_FULL_MASK, incl, o);
                    if (lane >= (uint32_t)o) incl += y;
                }
                const uint32_t tot = __shfl_sync(GV_FULL_MASK, incl, 31);
                uint32_t base = 0;
                if (lane == 0 && tot) base = atomicAdd(cursor + gi, tot);
                base = __shfl_sync(GV_FULL_MASK, base, 0);
                const uint32_t at = base + incl - c;
                for (uint32_t j = 0; j < c; ++j) {
                    if ((unsigned long long)(at + j) >= cap) {
                        atomicOr(err, 1u);
                        break;
                    }
                    const uint32_t w = mine[j];
                    const uint32_t nbw = blocks_for(g.vtx[w].y, g.logB);
                    pair_v[p0 + at + j] = w;
                    pieces[p0 + at + j] = (nbw + TL_PIECE_BLOCKS - 1) / TL_PIECE_BLOCKS;
                    blocks += nbw;
                }
            }
        }
    }
    blocks = warp_sum(blocks);
    if (lane == 0 && blocks) atomicAdd(words, blocks);
}

__global__ void k_tl_units(TlGroups t, uint32_t *__restrict__ units) {
    for (uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x; gi < t.G; gi += gridDim.x * blockDim.x) {
        const unsigned long long np = t.piece_off[t.pair_off[gi + 1]] - t.piece_off[t.pair_off[gi]];
        units[gi] = (uint32_t)((np + TL_UNIT_PIECES - 1) / TL_UNIT_PIECES);
    }
}

// Inserts the live entries of N(hv) into a table: warps over 32-block runs.
__device__ void tl_build(const DevGraph &g, uint32_t u, uint32_t *tab, uint32_t logc, uint32_t *err) {
    const uint32_t warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint4 rec = g.vtx[u];
    const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB);
    for (uint32_t kb = warp * TL_PIECE_BLOCKS; kb < nb; kb += nwarps * TL_PIECE_BLOCKS) {
        const uint32_t blk = tl_lane_block(g, rec.x, kb, nb);
        tl_scan_blocks(g, blk, kb, 0, min(TL_PIECE_BLOCKS, nb - kb), fill, [&](uint32_t w) { tl_insert(tab, logc, w, err); });
    }
}

__global__ void __launch_bounds__(TL_THREADS) k_tl_gbuild(DevGraph g, TlGroups t, const uint32_t *__restrict__ big,
                                                          uint32_t nbig, uint32_t *err) {
    for (uint32_t b = blockIdx.x; b < nbig; b += gridDim.x) {
        const uint32_t gi = big[b];
        tl_build(g, t.hv[gi], t.gh + t.gh_off[gi], t.tab_log[gi], err);
    }
}

template <bool SHARED>
__device__ __forceinline__ uint32_t tl_count_pieces(const DevGraph &g, const TlGroups &t, const uint32_t *tab,
                                                    uint32_t logc, unsigned long long lo, unsigned long long hi,
                                                    unsigned long long pstart, const uint32_t *qpair) {
    const uint32_t warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    uint32_t c = 0;
    for (unsigned long long q = lo + warp; q < hi; q += nwarps) {
        const unsigned long long p = pstart + qpair[q - lo];
        const uint32_t v = t.pair_v[p];
        const uint4 rec = g.vtx[v];
        const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB);
        const uint32_t kb0 = (uint32_t)(q - t.piece_off[p]) * TL_PIECE_BLOCKS;
        if (kb0 >= nb) continue;  // warp-uniform
        const uint32_t blk = tl_lane_block(g, rec.x, kb0, nb);
        tl_scan_blocks(g, blk, kb0, 0, min(TL_PIECE_BLOCKS, nb - kb0), fill, [&](uint32_t w) { c += tl_probe(tab, logc, w); });
    }
    return c;
}

__global__ void __launch_bounds__(TL_THREADS) k_tl_count(DevGraph g, TlGroups t, uint32_t U,
                                                         unsigned long long *__restrict__ cnt, uint32_t *err) {
    extern __shared__ uint32_t stab[];
    __shared__ uint32_t s_gi;
    __shared__ unsigned long long s_pstart;
    __shared__ uint32_t qpair[TL_UNIT_PIECES];
    __shared__ uint32_t red[TL_THREADS / 32];
    for (uint32_t unit = blockIdx.x; unit < U; unit += gridDim.x) {
        if (threadIdx.x == 0) {
            uint32_t lo = 0, hi = t.G;  // last group with unit_off <= unit
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (t.unit_off[mid] <= unit) lo = mid;
                else hi = mid;
            }
            s_gi = lo;
        }
        __syncthreads();
        const uint32_t gi = s_gi;
        const unsigned long long p0 = t.pair_off[gi], p1 = t.pair_off[gi + 1];
        const unsigned long long lo = t.piece_off[p0] + (unsigned long long)(unit - t.unit_off[gi]) * TL_UNIT_PIECES;
        const unsigned long long hi = min(lo + TL_UNIT_PIECES, t.piece_off[p1]);
        if (threadIdx.x == 0) {
            unsigned long long a = p0, b = p1;  // last pair with piece_off <= lo
            while (b - a > 1) {
                const unsigned long long mid = (a + b) >> 1;
                if (t.piece_off[mid] <= lo) a = mid;
                else b = mid;
            }
            s_pstart = a;
        }
        const uint32_t logc = t.tab_log[gi];
        const bool shared = t.gh_off[gi] == ~0ull;
        if (shared) {
            for (uint32_t k = threadIdx.x; k < (1u << logc); k += blockDim.x) stab[k] = GV_NIL;
        }
        __syncthreads();
        const unsigned long long pstart = s_pstart;
        for (unsigned long long p = pstart + threadIdx.x; p < p1 && t.piece_off[p] < hi; p += blockDim.x) {
            const unsigned long long a = max(t.piece_off[p], lo), b = min(t.piece_off[p + 1], hi);
            for (unsigned long long q = a; q < b; ++q) qpair[q - lo] = (uint32_t)(p - pstart);
        }
        if (shared) tl_build(g, t.hv[gi], stab, logc, err);
        __syncthreads();
        uint32_t c = shared ? tl_count_pieces<true>(g, t, stab, logc, lo, hi, pstart, qpair)
                            : tl_count_pieces<false>(g, t, t.gh + t.gh_off[gi], logc, lo, hi, pstart, qpair);
        c = warp_sum(c);
        if ((threadIdx.x & 31u) == 0) red[threadIdx.x >> 5] = c;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long tot = 0;
            for (int w = 0; w < TL_THREADS / 32; ++w) tot += red[w];
            if (tot) atomicAdd(cnt + gi, tot);
        }
        __syncthreads();
    }
}

__global__ void k_tl_out(const unsigned long long *__restrict__ cnt, uint32_t G, unsigned long long *__restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < G; i += gridDim.x * blockDim.x) out[i] = cnt[i] >> 1;
}

inline size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

uint32_t ceil_log2(uint64_t x) {
    uint32_t l = 0;
    while ((1ull << l) < x) ++l;
    return l;
}

}  // namespace

gv_status tc_local_subset(gv_graph *g, const uint32_t *d_sub, uint64_t ns, unsigned long long *d_out,
                          cudaStream_t s, bool *done, bool force) {
    *done = false;
    const DevGraph &d = g->d;
    if (ns == 0 || ns > 0xFFFFFFF0ull) return GV_OK;
    const uint32_t G = (uint32_t)ns;
    uint64_t live = 0;
    {
        Ctl c;
        gv_status st = read_ctl(g, &c, s);
        if (st != GV_OK) return st;
        live = c.live_edges;
    }
    // group-sized arrays (aux slot 4)
    const size_t o_du = 0, o_poff = o_du + al256(8ull * G), o_ghoff = o_poff + al256(8ull * (G + 1));
    const size_t o_tlog = o_ghoff + al256(8ull * G), o_cur = o_tlog + al256(4ull * G);
    const size_t o_uoff = o_cur + al256(4ull * G), o_cnt = o_uoff + al256(4ull * (G + 1));
    const size_t o_words = o_cnt + al256(8ull * G), bytes4 = o_words + 256;
    char *b4 = (char *)aux_scratch(g, 4, bytes4);
    if (!b4) return GV_ERR_NOMEM;
    uint2 *du = (uint2 *)(b4 + o_du);
    GV_LAUNCH(k_tl_deg, grid_for(G, 256), 256, 0, s, d, d_sub, G, du);
    std::vector<uint2> hdu(G);
    cudaError_t e = cudaMemcpyAsync(hdu.data(), du, 8ull * G, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "tc subset degrees");
    std::vector<unsigned long long> poff(G + 1), ghoff(G);
    std::vector<uint32_t> tlog(G), big;
    unsigned long long gslots = 0;
    poff[0] = 0;
    for (uint32_t i = 0; i < G; ++i)
        if (hdu[i].x == GV_NIL) {
            set_error("subset vertex out of range");
            return GV_ERR_INVALID;
        }
    for (uint32_t i = 0; i < G; ++i) {
        const uint32_t lv = hdu[i].x;
        poff[i + 1] = poff[i] + lv;
        tlog[i] = std::max<uint32_t>(5, ceil_log2(2ull * lv));
        if (lv > TL_SMEM_LIVE) {
            ghoff[i] = gslots;
            gslots += 1ull << tlog[i];
            big.push_back(i);
        } else {
            ghoff[i] = ~0ull;
        }
    }
    const uint64_t P = poff[G];
    // the scan lists alone reach half of the store: the whole-graph count is cheaper
    if (!force && P > live / 2) return GV_OK;
    // list-sized arrays (aux slot 5)
    const uint64_t scan_n = std::max<uint64_t>(P + 1, (uint64_t)G + 1);
    const size_t o_pv = 0, o_pc = o_pv + al256(4ull * (P + 1)), o_qoff = o_pc + al256(4ull * (P + 1));
    const size_t o_tmp = o_qoff + al256(8ull * (P + 1)), o_gh = o_tmp + al256(scan_scratch_bytes(scan_n));
    const size_t o_big = o_gh + al256(4ull * gslots), bytes5 = o_big + al256(4ull * big.size() + 4);
    char *b5 = (char *)aux_scratch(g, 5, bytes5);
    if (!b5) return GV_ERR_NOMEM;
    TlGroups t;
    t.hv = d_sub;
    t.pair_off = (const unsigned long long *)(b4 + o_poff);
    t.pair_v = (const uint32_t *)(b5 + o_pv);
    t.piece_off = (const unsigned long long *)(b5 + o_qoff);
    t.unit_off = (const uint32_t *)(b4 + o_uoff);
    t.gh_off = (const unsigned long long *)(b4 + o_ghoff);
    t.tab_log = (const uint32_t *)(b4 + o_tlog);
    t.gh = (uint32_t *)(b5 + o_gh);
    t.G = G;
    unsigned long long *words = (unsigned long long *)(b4 + o_words);
    uint32_t *err = (uint32_t *)(words + 1);
    uint32_t *units = (uint32_t *)(b4 + o_uoff);
    unsigned long long *cnt = (unsigned long long *)(b4 + o_cnt);
    e = cudaMemcpyAsync(b4 + o_poff, poff.data(), 8ull * (G + 1), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b4 + o_ghoff, ghoff.data(), 8ull * G, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b4 + o_tlog, tlog.data(), 4ull * G, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && !big.empty())
        e = cudaMemcpyAsync(b5 + o_big, big.data(), 4ull * big.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b4 + o_cur, 0, 4ull * G, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(cnt, 0, 8ull * G, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(words, 0, 16, s);
    if (e != cudaSuccess) return cuda_status(e, "tc subset setup");
    uint32_t *pv = (uint32_t *)(b5 + o_pv), *pc = (uint32_t *)(b5 + o_pc);
    GV_LAUNCH(k_tl_pairs, std::min<uint32_t>(G, 148 * 8), TL_THREADS, 0, s, d, t, (uint32_t *)(b4 + o_cur), pv, pc, words);
    scan_exclusive_u32_to_u64(pc, (unsigned long long *)(b5 + o_qoff), P, (unsigned long long *)(b5 + o_qoff) + P,
                              b5 + o_tmp, s);
    GV_LAUNCH(k_tl_units, grid_for(G, 256), 256, 0, s, t, units);
    scan_exclusive_u32(units, units, G, units + G, b5 + o_tmp, s);
    struct {
        unsigned long long blocks, err;
    } hw{};
    uint32_t U = 0;
    e = cudaMemcpyAsync(&hw, words, 16, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&U, units + G, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "tc subset plan");
    if ((uint32_t)hw.err) {
        set_error("tc subset: live counts and stored entries disagree");
        return GV_ERR_STATE;
    }
    // Hub lists are read again and again from L2, so a streamed entry costs
    // far less than one stored entry does in the whole-graph count (R-MAT
    // scale 22, B200: 1.2e10 streamed entries in 99 ms against 208 ms for the
    // whole-graph count of 1.3e8 entries).  Past TL_WHOLE_RATIO streamed
    // entries per stored entry the whole-graph count wins.
    if (!force && (double)hw.blocks * d.B > TL_WHOLE_RATIO * (double)live + (double)d.B * 1024.0) return GV_OK;
    if (gslots) {
        e = cudaMemsetAsync(t.gh, 0xFF, 4ull * gslots, s);
        if (e != cudaSuccess) return cuda_status(e, "tc subset tables");
        GV_LAUNCH(k_tl_gbuild, std::min<uint32_t>((uint32_t)big.size(), 148 * 4), TL_THREADS, 0, s, d, t,
                  (const uint32_t *)(b5 + o_big), (uint32_t)big.size(), err);
    }
    if (U) {
        const size_t smem = (1u << TL_SMEM_LOG) * 4u;
        cudaFuncSetAttribute(k_tl_count, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        GV_LAUNCH(k_tl_count, std::min<uint32_t>(U, 148 * TL_COUNT_CTAS_PER_SM), TL_THREADS, smem, s, d, t, U, cnt, err);
    }
    GV_LAUNCH(k_tl_out, grid_for(G, 256), 256, 0, s, (const unsigned long long *)cnt, G, d_out);
    uint32_t herr = 0;
    e = cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "tc subset count");
    if (herr) {
        set_error("tc subset: a neighbour table overflowed (live counts and stored entries disagree)");
        return GV_ERR_STATE;
    }
    *done = true;
    return GV_OK;
}

}  // namespace gv

// ------------------------------------------------------- batch deltas
// Exact change of the triangle counts across one batch (inserts, then
// deletes, as gv_insert_edges / gv_delete_edges apply them).  With A the
// inserted pairs that were not in the graph and R the deleted pairs that were
// in it after the inserts, both counted on the graph between the two steps
// (G_mid):
//   created   = triangles of G_mid with at least one edge in A,
//   destroyed = triangles of G_mid with at least one edge in R,
//   T_after = T_before + created - destroyed.
// A triangle is counted once, at its smallest changed edge (pairs ordered by
// their canonical key min << bitsn | max): for a changed pair (a, b) and a
// common neighbour w, (a, w) or (b, w) being a smaller changed pair skips it.
// Work: sum over changed pairs of the shorter list (plus one table of each
// heavy endpoint), against a whole-graph count.
namespace gv {
namespace {

constexpr int TD_THREADS = 256;
constexpr int TD_WARPS = TD_THREADS / 32;
constexpr unsigned long long TD_NONE = ~0ull;

__device__ __forceinline__ unsigned long long td_key(uint32_t a, uint32_t b, uint32_t bitsn) {
    return a < b ? ((unsigned long long)a << bitsn) | b : ((unsigned long long)b << bitsn) | a;
}

__global__ void k_td_keys(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst, uint64_t k, uint32_t n,
                          uint32_t bitsn, unsigned long long *__restrict__ keys, uint32_t *bad) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < k; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t a = src[i], b = dst[i];
        if (a >= n || b >= n) {
            atomicOr(bad, 1u);
            keys[i] = TD_NONE;
        } else {
            keys[i] = a == b ? TD_NONE : td_key(a, b, bitsn);  // self-loops are never stored
        }
    }
}

// flag[i] = 1 for the first copy of each real key (keys sorted).
__global__ void k_td_first(const unsigned long long *__restrict__ keys, uint64_t k, uint32_t *__restrict__ flag) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < k; i += (uint64_t)gridDim.x * blockDim.x)
        flag[i] = keys[i] != TD_NONE && (i == 0 || keys[i - 1] != keys[i]);
}

__global__ void k_td_compact(const unsigned long long *__restrict__ keys, const uint32_t *__restrict__ flag,
                             const uint32_t *__restrict__ pos, uint64_t k, unsigned long long *__restrict__ out) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < k; i += (uint64_t)gridDim.x * blockDim.x)
        if (flag[i]) out[pos[i]] = keys[i];
}

// present[i] = pair i is in the graph: the warp scans the shorter list.
__global__ void __launch_bounds__(TD_THREADS) k_td_member(DevGraph g, const unsigned long long *__restrict__ keys,
                                                          uint32_t cnt, uint32_t bitsn, uint32_t *__restrict__ present) {
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned long long mask = (1ull << bitsn) - 1;
    for (uint32_t i = blockIdx.x * TD_WARPS + (threadIdx.x >> 5); i < cnt; i += gridDim.x * TD_WARPS) {
        const uint32_t a = (uint32_t)(keys[i] >> bitsn), b = (uint32_t)(keys[i] & mask);
        const uint4 ra = g.vtx[a], rb = g.vtx[b];
        const bool a_short = ra.y <= rb.y;
        const uint4 rs = a_short ? ra : rb;
        const uint32_t want = a_short ? b : a;
        const uint32_t fill = rs.y, nb = blocks_for(fill, g.logB);
        uint32_t hit = 0;
        for (uint32_t kb = 0; kb < nb && !hit; kb += TL_PIECE_BLOCKS) {  // warp-uniform
            const uint32_t blk = tl_lane_block(g, rs.x, kb, nb);
            uint32_t mine = 0;
            tl_scan_blocks(g, blk, kb, 0, min(TL_PIECE_BLOCKS, nb - kb), fill, [&](uint32_t w) { mine |= (w == want); });
            hit = __any_sync(GV_FULL_MASK, mine);
        }
        if (lane == 0) present[i] = hit;
    }
}

// keep[i] = present[i] == want (A: pairs not yet in the graph; R: pairs in it).
__global__ void k_td_select(const uint32_t *__restrict__ present, uint32_t cnt, uint32_t want, uint32_t *__restrict__ keep) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x)
        keep[i] = present[i] == want;
}

__device__ __forceinline__ uint32_t td_slot(unsigned long long key, uint32_t log) {
    return (uint32_t)((key * 0x9E3779B97F4A7C15ull) >> (64 - log));
}

__global__ void k_td_set_build(const unsigned long long *__restrict__ keys, uint32_t cnt, unsigned long long *set,
                               uint32_t log, uint32_t *err) {
    const uint32_t mask = (1u << log) - 1u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        uint32_t h = td_slot(keys[i], log);
        uint32_t p = 0;
        for (; p <= mask; ++p) {
            const unsigned long long old = atomicCAS(set + h, TD_NONE, keys[i]);
            if (old == TD_NONE || old == keys[i]) break;
            h = (h + 1u) & mask;
        }
        if (p > mask) atomicOr(err, 4u);
    }
}

__device__ __forceinline__ bool td_set_has(const unsigned long long *set, uint32_t log, unsigned long long key) {
    const uint32_t mask = (1u << log) - 1u;
    uint32_t h = td_slot(key, log);
    for (uint32_t p = 0; p <= mask; ++p) {
        const unsigned long long x = set[h];
        if (x == key) return true;
        if (x == TD_NONE) return false;
        h = (h + 1u) & mask;
    }
    return false;
}

// Heavy endpoints (more than TD_LIGHT live entries) of the changed pairs get a
// hash table of their whole list in global memory, built once per call, so
// a pair costs its shorter list: the warp streams it against the longer
// endpoint's table (its own shared table when that list is light too).
constexpr uint32_t TD_LIGHT = 256;
constexpr uint32_t TD_WLOG = 9;  // per-warp shared table: 512 slots

__global__ void k_td_mark(DevGraph g, const unsigned long long *__restrict__ keys, uint32_t cnt, uint32_t bitsn,
                          uint32_t *__restrict__ flag, uint32_t *__restrict__ hlist, uint32_t *nh) {
    const unsigned long long mask = (1ull << bitsn) - 1;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        const uint32_t ends[2] = {(uint32_t)(keys[i] >> bitsn), (uint32_t)(keys[i] & mask)};
        for (int e = 0; e < 2; ++e) {
            const uint32_t v = ends[e];
            if (g.vtx[v].z > TD_LIGHT && atomicCAS(flag + v, 0u, 1u) == 0u) hlist[atomicAdd(nh, 1u)] = v;
        }
    }
}

__global__ void k_td_caps(DevGraph g, const uint32_t *__restrict__ hlist, const uint32_t *nh,
                          unsigned long long *__restrict__ cap, uint32_t *__restrict__ hlog, uint32_t *__restrict__ hidx) {
    const uint32_t nhv = *nh;
    for (uint32_t h = blockIdx.x * blockDim.x + threadIdx.x; h < nhv; h += gridDim.x * blockDim.x) {
        const uint32_t v = hlist[h];
        const uint32_t live = g.vtx[v].z;
        uint32_t l = 10;
        while ((1ull << l) < 2ull * live) ++l;
        cap[h] = 1ull << l;
        hlog[h] = l;
        hidx[v] = h;
    }
}

__global__ void __launch_bounds__(TD_THREADS) k_td_build(DevGraph g, const uint32_t *__restrict__ hlist, const uint32_t *nh,
                                                         const unsigned long long *__restrict__ hoff,
                                                         const uint32_t *__restrict__ hlog, uint32_t *gtab, uint32_t *err) {
    const uint32_t nhv = *nh;
    for (uint32_t h = blockIdx.x; h < nhv; h += gridDim.x) {
        const uint32_t v = hlist[h];
        const uint4 rec = g.vtx[v];
        const uint32_t nb = blocks_for(rec.y, g.logB);
        uint32_t *tab = gtab + hoff[h];
        for (uint32_t kb = (threadIdx.x >> 5) * TL_PIECE_BLOCKS; kb < nb; kb += TD_WARPS * TL_PIECE_BLOCKS) {
            const uint32_t blk = tl_lane_block(g, rec.x, kb, nb);
            tl_scan_blocks(g, blk, kb, 0, min(TL_PIECE_BLOCKS, nb - kb), rec.y,
                           [&](uint32_t w) { tl_insert(tab, hlog[h], w, err); });
        }
    }
}

// Triangles through each changed pair (a, b), counted at their smallest
// changed edge.
__global__ void __launch_bounds__(TD_THREADS) k_td_count(DevGraph g, const unsigned long long *__restrict__ keys,
                                                         uint32_t cnt, uint32_t bitsn, const unsigned long long *set,
                                                         uint32_t set_log, const uint32_t *__restrict__ hidx,
                                                         const unsigned long long *__restrict__ hoff,
                                                         const uint32_t *__restrict__ hlog, const uint32_t *gtab,
                                                         unsigned long long *total, long long *__restrict__ owner,
                                                         long long sign, uint32_t *err) {
    __shared__ uint32_t wtab[TD_WARPS][1u << TD_WLOG];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const unsigned long long mask = (1ull << bitsn) - 1;
    unsigned long long mine = 0;
    for (uint32_t i = blockIdx.x * TD_WARPS + warp; i < cnt; i += gridDim.x * TD_WARPS) {
        const unsigned long long ke = keys[i];
        const uint32_t a = (uint32_t)(ke >> bitsn), b = (uint32_t)(ke & mask);
        const uint4 ra = g.vtx[a], rb = g.vtx[b];
        const bool a_long = ra.z >= rb.z;
        const uint4 rl = a_long ? ra : rb, rs = a_long ? rb : ra;
        const uint32_t l = a_long ? a : b;
        const uint32_t *tab;
        uint32_t tlog;
        if (rl.z > TD_LIGHT) {  // warp-uniform
            const uint32_t h = hidx[l];
            tab = gtab + hoff[h];
            tlog = hlog[h];
        } else {
            uint32_t *wt = wtab[warp];
            for (uint32_t t = lane; t < (1u << TD_WLOG); t += 32) wt[t] = GV_NIL;
            __syncwarp();
            const uint32_t nbl = blocks_for(rl.y, g.logB);
            for (uint32_t kb = 0; kb < nbl; kb += TL_PIECE_BLOCKS) {
                const uint32_t blk = tl_lane_block(g, rl.x, kb, nbl);
                tl_scan_blocks(g, blk, kb, 0, min(TL_PIECE_BLOCKS, nbl - kb), rl.y,
                               [&](uint32_t w) { tl_insert(wt, TD_WLOG, w, err); });
            }
            __syncwarp();
            tab = wt;
            tlog = TD_WLOG;
        }
        const uint32_t nbs = blocks_for(rs.y, g.logB);
        for (uint32_t kb = 0; kb < nbs; kb += TL_PIECE_BLOCKS) {
            const uint32_t blk = tl_lane_block(g, rs.x, kb, nbs);
            tl_scan_blocks(g, blk, kb, 0, min(TL_PIECE_BLOCKS, nbs - kb), rs.y, [&](uint32_t w) {
                if (!tl_probe(tab, tlog, w)) return;
                const unsigned long long k1 = td_key(a, w, bitsn), k2 = td_key(b, w, bitsn);
                if (k1 < ke && td_set_has(set, set_log, k1)) return;
                if (k2 < ke && td_set_has(set, set_log, k2)) return;
                ++mine;
                if (owner)  // two's complement: adding (u64)-1 subtracts one
                    atomicAdd(reinterpret_cast<unsigned long long *>(owner) + min(w, min(a, b)),
                              (unsigned long long)sign);
            });
        }
        __syncwarp();
    }
    mine = warp_sum(mine);
    if (lane == 0 && mine) atomicAdd(total, mine);
}

}  // namespace

// Changed pairs of one side of the batch: canonical, deduplicated, and kept
// when their presence in the graph now equals `want_present`.  Returns the
// count; the keys sit in *out (scratch slot 4).
static gv_status td_pairs(gv_graph *g, const uint32_t *dsrc, const uint32_t *ddst, uint64_t k, uint32_t want_present,
                          unsigned long long **out, uint32_t *count, cudaStream_t s, bool ids_only = false) {
    const uint32_t n = g->d.n, bitsn = g->bitsn;
    *count = 0;
    if (k == 0) return GV_OK;
    const uint64_t rc = radix_counts_elems(k);
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t o_k1 = 0, o_k2 = o_k1 + al(k * 8), o_out = o_k2 + al(k * 8), o_f = o_out + al(k * 8);
    const size_t o_p = o_f + al(k * 4), o_c = o_p + al((k + 1) * 4), o_t = o_c + al(rc * 4);
    const size_t bytes = o_t + al(scan_scratch_bytes(std::max<uint64_t>(rc, k + 1))) + 256;
    char *b = (char *)aux_scratch(g, 4, bytes);
    if (!b) return GV_ERR_NOMEM;
    unsigned long long *k1 = (unsigned long long *)(b + o_k1), *k2 = (unsigned long long *)(b + o_k2);
    unsigned long long *outk = (unsigned long long *)(b + o_out);
    uint32_t *flag = (uint32_t *)(b + o_f), *pos = (uint32_t *)(b + o_p), *cnts = (uint32_t *)(b + o_c);
    void *tmp = b + o_t;
    uint32_t *bad = flag;  // checked before the flags are written
    cudaMemsetAsync(bad, 0, 4, s);
    GV_LAUNCH(k_td_keys, grid_for(k, 256, 148 * 16), 256, 0, s, dsrc, ddst, k, n, bitsn, k1, bad);
    uint32_t hbad = 0;
    cudaError_t e = cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "tc delta keys");
    if (hbad) {
        set_error("vertex id out of range");
        return GV_ERR_INVALID;
    }
    if (ids_only) return GV_OK;
    const int which = radix_sort_u64(k1, k2, nullptr, nullptr, k, 2 * (int)bitsn, cnts, tmp, s);
    const unsigned long long *sk = which ? k2 : k1;
    GV_LAUNCH(k_td_first, grid_for(k, 256, 148 * 16), 256, 0, s, sk, k, flag);
    scan_exclusive_u32(flag, pos, k, pos + k, tmp, s);
    GV_LAUNCH(k_td_compact, grid_for(k, 256, 148 * 16), 256, 0, s, sk, (const uint32_t *)flag, (const uint32_t *)pos, k,
              outk);
    uint32_t nu = 0;
    e = cudaMemcpyAsync(&nu, pos + k, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "tc delta unique");
    if (nu == 0) return GV_OK;
    // presence in the graph as it is now, then keep the wanted side
    uint32_t *present = flag;  // reuse (nu <= k)
    GV_LAUNCH(k_td_member, grid_for(nu, TD_WARPS, 148 * 8), TD_THREADS, 0, s, g->d, (const unsigned long long *)outk, nu,
              bitsn, present);
    GV_LAUNCH(k_td_select, grid_for(nu, 256), 256, 0, s, (const uint32_t *)present, nu, want_present, present);
    scan_exclusive_u32(present, pos, nu, pos + nu, tmp, s);
    GV_LAUNCH(k_td_compact, grid_for(nu, 256), 256, 0, s, (const unsigned long long *)outk, (const uint32_t *)present,
              (const uint32_t *)pos, nu, k1);  // k1 is free again
    e = cudaMemcpyAsync(count, pos + nu, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "tc delta select");
    *out = k1;
    return GV_OK;
}

// Neighbour tables of the heavy endpoints of the changed pairs (slots 8 and
// 9), built once for both halves of a batch: the created pairs are counted
// after the inserts and the destroyed ones before the deletes, on the same
// graph.
struct TdTables {
    const uint32_t *hidx = nullptr, *hlog = nullptr, *gtab = nullptr;
    const unsigned long long *hoff = nullptr;
};

static gv_status td_tables(gv_graph *g, const unsigned long long *const *lists, const uint32_t *counts, int nlists,
                           uint32_t *err, TdTables *out, cudaStream_t s) {
    const uint32_t n = g->d.n;
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t o_flag = 0, o_list = al((size_t)n * 4), o_hidx = o_list + al((size_t)n * 4);
    const size_t o_log = o_hidx + al((size_t)n * 4), o_cap = o_log + al((size_t)n * 4);
    const size_t o_off = o_cap + al(((size_t)n + 1) * 8), o_tmp = o_off + al(((size_t)n + 1) * 8);
    const size_t bytes = o_tmp + al(scan_scratch_bytes((uint64_t)n + 1)) + 256;
    char *b8 = (char *)aux_scratch(g, 8, bytes);
    if (!b8) return GV_ERR_NOMEM;
    uint32_t *flag = (uint32_t *)(b8 + o_flag), *hlist = (uint32_t *)(b8 + o_list);
    uint32_t *hidx = (uint32_t *)(b8 + o_hidx), *hlog = (uint32_t *)(b8 + o_log);
    unsigned long long *cap = (unsigned long long *)(b8 + o_cap), *hoff = (unsigned long long *)(b8 + o_off);
    uint32_t *nh = reinterpret_cast<uint32_t *>(hoff + n);  // scratch word until the scan writes the offsets
    cudaMemsetAsync(flag, 0, (size_t)n * 4, s);
    cudaMemsetAsync(nh, 0, 4, s);
    for (int l = 0; l < nlists; ++l)
        if (counts[l])
            GV_LAUNCH(k_td_mark, grid_for(counts[l], 256), 256, 0, s, g->d, lists[l], counts[l], g->bitsn, flag, hlist, nh);
    uint32_t hn = 0;
    cudaError_t e = cudaMemcpyAsync(&hn, nh, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "tc delta heavy");
    uint32_t *dn = flag;  // the count, in a word the scan does not touch
    cudaMemcpyAsync(dn, nh, 4, cudaMemcpyDeviceToDevice, s);
    uint32_t *gtab = nullptr;
    if (hn) {
        GV_LAUNCH(k_td_caps, grid_for(hn, 256), 256, 0, s, g->d, (const uint32_t *)hlist, (const uint32_t *)dn, cap,
                  hlog, hidx);
        scan_exclusive_u64(cap, hoff, hn, hoff + hn, b8 + o_tmp, s);
        unsigned long long slots = 0;
        e = cudaMemcpyAsync(&slots, hoff + hn, 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e, "tc delta tables");
        gtab = (uint32_t *)aux_scratch(g, 9, slots * 4 + 256);
        if (!gtab) return GV_ERR_NOMEM;
        cudaMemsetAsync(gtab, 0xFF, slots * 4, s);
        GV_LAUNCH(k_td_build, std::min<uint32_t>(hn, 148 * 8), TD_THREADS, 0, s, g->d, (const uint32_t *)hlist,
                  (const uint32_t *)dn, (const unsigned long long *)hoff, (const uint32_t *)hlog, gtab, err);
    }
    out->hidx = hidx;
    out->hlog = hlog;
    out->hoff = hoff;
    out->gtab = gtab;
    return cuda_status(cudaGetLastError(), "tc delta tables");
}

// Counts the triangles of the current graph through the `cnt` changed pairs
// (the set of those pairs decides at which changed edge a triangle counts).
static gv_status td_count(gv_graph *g, const unsigned long long *pairs, uint32_t cnt, const TdTables &t,
                          unsigned long long *total, long long *owner, long long sign, uint32_t *err, cudaStream_t s) {
    if (cnt == 0) return GV_OK;
    uint32_t log = 10;
    while ((1ull << log) < 2ull * cnt) ++log;
    unsigned long long *set = (unsigned long long *)aux_scratch(g, 5, (8ull << log) + 256);
    if (!set) return GV_ERR_NOMEM;
    cudaMemsetAsync(set, 0xFF, 8ull << log, s);
    GV_LAUNCH(k_td_set_build, grid_for(cnt, 256), 256, 0, s, pairs, cnt, set, log, err);
    GV_LAUNCH(k_td_count, grid_for(cnt, TD_WARPS, 148 * 8), TD_THREADS, 0, s, g->d, pairs, cnt, g->bitsn,
              (const unsigned long long *)set, log, t.hidx, t.hoff, t.hlog, t.gtab, total, owner, sign, err);
    return cuda_status(cudaGetLastError(), "tc delta count");
}

}  // namespace gv

using namespace gv;

extern "C" gv_status gv_update_tc(gv_graph *g, const uint32_t *ins_src, const uint32_t *ins_dst, const float *ins_w,
                                  uint64_t n_ins, const uint32_t *del_src, const uint32_t *del_dst, uint64_t n_del,
                                  uint32_t flags, int64_t *delta_total, int64_t *delta_owner, int mem, void *stream) {
    if (!g || !delta_total || (n_ins && (!ins_src || !ins_dst)) || (n_del && (!del_src || !del_dst))) {
        set_error("null argument");
        return GV_ERR_INVALID;
    }
    if (g->parent) { set_error("a view is read-only"); return GV_ERR_STATE; }
    if (g->cfg.directed) { set_error("triangle counting needs an undirected store"); return GV_ERR_STATE; }
    if (mem != GV_MEM_HOST && mem != GV_MEM_DEVICE) { set_error("bad mem flag"); return GV_ERR_INVALID; }
    cudaSetDevice(g->cfg.device);
    cudaStream_t s = (cudaStream_t)stream;
    const uint32_t n = g->d.n;
    // device copies of the pairs (slot 6 is free outside betweenness)
    const uint64_t tot_pairs = n_ins + n_del;
    const bool weighted = g->cfg.weighted && ins_w;
    if (g->cfg.weighted && n_ins && !ins_w) { set_error("weighted store needs weights"); return GV_ERR_INVALID; }
    uint32_t *dp = nullptr;
    const float *iw = ins_w;
    if (mem == GV_MEM_HOST && tot_pairs) {
        dp = (uint32_t *)aux_scratch(g, 6, tot_pairs * 8 + (weighted ? n_ins * 4 : 0) + 256);
        if (!dp) return GV_ERR_NOMEM;
        cudaError_t e = cudaSuccess;
        if (weighted) {
            float *dw = (float *)(dp + 2 * tot_pairs);
            e = cudaMemcpyAsync(dw, ins_w, n_ins * 4, cudaMemcpyHostToDevice, s);
            iw = dw;
        }
        if (n_ins) e = cudaMemcpyAsync(dp, ins_src, n_ins * 4, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && n_ins) e = cudaMemcpyAsync(dp + n_ins, ins_dst, n_ins * 4, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && n_del) e = cudaMemcpyAsync(dp + 2 * n_ins, del_src, n_del * 4, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && n_del)
            e = cudaMemcpyAsync(dp + 2 * n_ins + n_del, del_dst, n_del * 4, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return cuda_status(e, "tc delta input");
    }
    const uint32_t *is = mem == GV_MEM_HOST ? dp : ins_src, *id = mem == GV_MEM_HOST ? dp + n_ins : ins_dst;
    const uint32_t *ds = mem == GV_MEM_HOST ? dp + 2 * n_ins : del_src;
    const uint32_t *dd = mem == GV_MEM_HOST ? dp + 2 * n_ins + n_del : del_dst;
    // words: [0] created, [1] destroyed, [2] error flags
    unsigned long long *words = (unsigned long long *)aux_scratch(g, 3, 64);
    if (!words) return GV_ERR_NOMEM;
    cudaMemsetAsync(words, 0, 24, s);
    uint32_t *err = (uint32_t *)(words + 2);
    long long *owner = nullptr;
    if (delta_owner) {
        owner = (long long *)(mem == GV_MEM_DEVICE ? (void *)delta_owner : aux_scratch(g, 7, (size_t)n * 8));
        if (!owner) return GV_ERR_NOMEM;
        cudaMemsetAsync(owner, 0, (size_t)n * 8, s);
    }
    // inserts: the new pairs A (absent now), then applied; the triangles through
    // A are counted on the graph after the inserts
    unsigned long long *pairs = nullptr;
    uint32_t cnt = 0;
    gv_status st = GV_OK;
    // delete ids are checked before anything changes, so a bad id rejects the whole call
    if (n_del) {
        unsigned long long *unused = nullptr;
        uint32_t unused_cnt = 0;
        st = td_pairs(g, ds, dd, n_del, 1u, &unused, &unused_cnt, s, true);
        if (st != GV_OK) return st;
    }
    st = td_pairs(g, is, id, n_ins, 0u, &pairs, &cnt, s);
    if (st != GV_OK) return st;
    // A moves out of the pair scratch (slot 11), which the deletes' pairs reuse
    unsigned long long *apairs = nullptr;
    const uint32_t acnt = cnt;
    if (acnt) {
        apairs = (unsigned long long *)aux_scratch(g, 11, (size_t)acnt * 8 + 256);
        if (!apairs) return GV_ERR_NOMEM;
        cudaError_t e = cudaMemcpyAsync(apairs, pairs, (size_t)acnt * 8, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return cuda_status(e, "tc delta pairs");
    }
    if (n_ins) {
        st = gv_insert_edges(g, is, id, iw, n_ins, GV_MEM_DEVICE, stream);
        if (st == GV_OK) st = gv_synchronize(g, stream);
        if (st != GV_OK) return st;
    }
    // deletes: the pairs present now R; A and R are counted on this graph with
    // one set of neighbour tables, then the deletes are applied
    uint32_t rcnt = 0;
    unsigned long long *rpairs = nullptr;
    if (n_del) {
        st = td_pairs(g, ds, dd, n_del, 1u, &rpairs, &rcnt, s);
        if (st != GV_OK) return st;
    }
    if (acnt || rcnt) {
        const unsigned long long *lists[2] = {apairs, rpairs};
        const uint32_t counts[2] = {acnt, rcnt};
        TdTables tabs;
        st = td_tables(g, lists, counts, 2, err, &tabs, s);
        if (st == GV_OK) st = td_count(g, apairs, acnt, tabs, words + 0, owner, 1, err, s);
        if (st == GV_OK) st = td_count(g, rpairs, rcnt, tabs, words + 1, owner, -1, err, s);
        if (st != GV_OK) return st;
    }
    if (n_del) {
        st = gv_delete_edges(g, ds, dd, n_del, GV_MEM_DEVICE, stream);
        if (st == GV_OK) st = gv_synchronize(g, stream);
        if (st != GV_OK) return st;
    }
    if (flags & 1u) {
        st = gv_compact(g, stream);
        if (st == GV_OK) st = gv_synchronize(g, stream);
        if (st != GV_OK) return st;
    }
    unsigned long long h[3] = {0, 0, 0};
    cudaError_t e = cudaMemcpyAsync(h, words, 24, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && delta_owner && mem == GV_MEM_HOST)
        e = cudaMemcpyAsync(delta_owner, owner, (size_t)n * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "tc delta out");
    if ((uint32_t)h[2]) {
        set_error("tc delta: a neighbour table overflowed (live counts and stored entries disagree)");
        return GV_ERR_STATE;
    }
    *delta_total = (int64_t)h[0] - (int64_t)h[1];
    return GV_OK;
}
