// Batched edge insert / delete and compaction on the edge-block CBT store.
//
// One batch runs as a stream-ordered pipeline with no host round trip:
//   expand   pairs -> 64-bit keys (src << bits | dst), both directions on an
//            undirected graph; self-loops and out-of-range ids become the
//            sentinel key, which sorts last.  Range errors abort the batch.
//   sort     stable LSD radix sort of the keys (prims.cu) = the batch staged
//            sorted and segmented by source vertex.
//   segment  adjacent-unique compaction: bdst[] (sorted, de-duplicated
//            destinations) and one segment {vertex, start} per touched vertex.
//   member   one lane group per segment (a whole CTA for hubs) streams the
//            vertex's existing blocks with 16-byte loads and binary-searches
//            each entry in the segment: insert marks batch entries that
//            already exist, delete tombstones matching graph entries.
//   plan     blocks each segment needs; warp-aggregated atomics hand out
//            contiguous ranges of the free stack.
//   admit    rejects the whole batch if the pool cannot hold it.
//   apply    writes new entries after the last used slot, links the new
//            blocks into the CBT (children 2k+1 / 2k+2, level-order
//            predecessor) and updates the vertex record.
// Reference pipeline replaced: src/dynamicStructure/graphvine.cu:222-451 with
// kernels src/dynamicStructure/kernels/insert_kernels.cu:3-365 and
// src/dynamicStructure/kernels/delete_kernels.cu:3-48.
#include <algorithm>
#include "store.cuh"
#include "group.cuh"
#include "prims.cuh"
#include "launch.hpp"
#include "prof.hpp"

namespace gv {

unsigned grid_for(uint64_t work_items, unsigned per_cta, unsigned max_ctas) {
    uint64_t g = (work_items + per_cta - 1) / per_cta;
    if (g < 1) g = 1;
    if (g > max_ctas) g = max_ctas;
    return (unsigned)g;
}

namespace {

constexpr int UPD_THREADS = 256;
constexpr int SEG_THREADS = 256;
constexpr int SEG_ITEMS = 8;
constexpr int SEG_TILE = SEG_THREADS * SEG_ITEMS;
constexpr int BIG_TAB = 1024;  // block-table chunk of the CTA-per-vertex paths

__device__ __forceinline__ bool is_big(uint32_t nb, uint32_t len) {
    return nb > BIG_BLOCKS || len > BIG_SEGMENT;
}

// ------------------------------------------------------------------ expand
__global__ void k_expand(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
                         uint64_t k, int sym, uint32_t n, uint32_t bitsn,
                         unsigned long long *__restrict__ keys, uint32_t *__restrict__ vals,
                         Ctl *ctl) {
    const unsigned long long sent = (bitsn >= 32) ? ~0ull : ((1ull << (2 * bitsn)) - 1ull);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < k;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = src[i], d = dst[i];
        const bool bad = (s >= n) || (d >= n);
        if (bad) {
            atomicOr(&ctl->status, GV_DEV_ERR_RANGE);
            ctl->batch_abort = 1;
        }
        const bool drop = bad || (s == d);
        if (sym) {
            keys[2 * i] = drop ? sent : (((unsigned long long)s << bitsn) | d);
            keys[2 * i + 1] = drop ? sent : (((unsigned long long)d << bitsn) | s);
            if (vals) {
                vals[2 * i] = (uint32_t)(2 * i);
                vals[2 * i + 1] = (uint32_t)(2 * i + 1);
            }
        } else {
            keys[i] = drop ? sent : (((unsigned long long)s << bitsn) | d);
            if (vals) vals[i] = (uint32_t)i;
        }
    }
}

// ----------------------------------------------------------------- segment
__device__ __forceinline__ void seg_flags(const unsigned long long *K, uint64_t i, uint64_t N,
                                          unsigned long long sent, uint32_t bitsn, bool &uniq,
                                          bool &head) {
    uniq = head = false;
    if (i >= N) return;
    const unsigned long long key = K[i];
    if (key == sent) return;
    if (i == 0) {
        uniq = head = true;
        return;
    }
    const unsigned long long prev = K[i - 1];
    uniq = key != prev;
    head = uniq && ((key >> bitsn) != (prev >> bitsn));
}

__global__ void __launch_bounds__(SEG_THREADS) k_seg_count(const unsigned long long *__restrict__ K,
                                                           uint64_t N, unsigned long long sent,
                                                           uint32_t bitsn,
                                                           unsigned long long *__restrict__ tile_cnt) {
    __shared__ unsigned long long wt[33];
    const uint64_t base = (uint64_t)blockIdx.x * SEG_TILE + (uint64_t)threadIdx.x * SEG_ITEMS;
    unsigned long long c = 0;
#pragma unroll
    for (int j = 0; j < SEG_ITEMS; ++j) {
        bool u, h;
        seg_flags(K, base + j, N, sent, bitsn, u, h);
        c += ((unsigned long long)u << 32) | (unsigned long long)h;
    }
    unsigned long long tot = cta_sum<unsigned long long, SEG_THREADS>(c, wt);
    if (threadIdx.x == 0) tile_cnt[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(SEG_THREADS) k_seg_write(
    const unsigned long long *__restrict__ K, const uint32_t *__restrict__ V, uint64_t N,
    unsigned long long sent, uint32_t bitsn, int sym_shift,
    const unsigned long long *__restrict__ tile_off, const float *__restrict__ in_w,
    uint32_t *__restrict__ bdst, float *__restrict__ bw, uint8_t *__restrict__ found,
    uint32_t *__restrict__ seg_vertex, uint32_t *__restrict__ seg_start, uint8_t *affected,
    Ctl *ctl) {
    __shared__ unsigned long long wt[33];
    const uint64_t base = (uint64_t)blockIdx.x * SEG_TILE + (uint64_t)threadIdx.x * SEG_ITEMS;
    const unsigned long long dmask = (1ull << bitsn) - 1ull;
    unsigned long long c = 0;
    bool uf[SEG_ITEMS], hf[SEG_ITEMS];
#pragma unroll
    for (int j = 0; j < SEG_ITEMS; ++j) {
        seg_flags(K, base + j, N, sent, bitsn, uf[j], hf[j]);
        c += ((unsigned long long)uf[j] << 32) | (unsigned long long)hf[j];
    }
    unsigned long long tot;
    unsigned long long pre = cta_excl_scan<unsigned long long, SEG_THREADS>(c, wt, tot) + tile_off[blockIdx.x];
    uint32_t up = (uint32_t)(pre >> 32), hp = (uint32_t)(pre & 0xFFFFFFFFull);
#pragma unroll
    for (int j = 0; j < SEG_ITEMS; ++j) {
        if (!uf[j]) continue;
        const unsigned long long key = K[base + j];
        const uint32_t s = (uint32_t)(key >> bitsn), d = (uint32_t)(key & dmask);
        bdst[up] = d;
        found[up] = 0;
        if (bw) bw[up] = in_w[V[base + j] >> sym_shift];
        affected[s] = 1;
        affected[d] = 1;
        if (hf[j]) {
            seg_vertex[hp] = s;
            seg_start[hp] = up;
            ++hp;
        }
        ++up;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // The scan wrote the packed grand total into ctl->scratch0.
        const unsigned long long t = ctl->scratch0;
        const uint32_t nuniq = (uint32_t)(t >> 32), nseg = (uint32_t)(t & 0xFFFFFFFFull);
        ctl->nuniq = nuniq;
        ctl->nseg = nseg;
        seg_start[nseg] = nuniq;
    }
}

// ------------------------------------------------------------------ member
template <int TPV, bool DEL>
__global__ void __launch_bounds__(UPD_THREADS) k_member(DevGraph g,
                                                        const uint32_t *__restrict__ seg_vertex,
                                                        const uint32_t *__restrict__ seg_start,
                                                        const uint32_t *__restrict__ bdst,
                                                        uint8_t *__restrict__ found,
                                                        uint32_t *__restrict__ seg_found,
                                                        uint32_t *__restrict__ big_list) {
    constexpr int GPC = UPD_THREADS / TPV;
    __shared__ uint32_t tabs[GPC][BIG_BLOCKS];
    if (DEL && g.ctl->batch_abort) return;
    const uint32_t nseg = (uint32_t)g.ctl->nseg;
    Group<TPV> G;
    const uint32_t gcta = threadIdx.x / TPV;
    uint32_t *tab = tabs[gcta];
    const uint32_t ngroups = gridDim.x * GPC;
    for (uint32_t s = blockIdx.x * GPC + gcta; s < nseg; s += ngroups) {
        const uint32_t u = seg_vertex[s];
        const uint32_t st = seg_start[s], len = seg_start[s + 1] - st;
        const uint4 rec = g.vtx[u];
        const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB);
        if (is_big(nb, len)) {
            if (G.gl == 0) big_list[atomicAdd(&g.ctl->nbig, 1ull)] = s;
            continue;
        }
        fill_block_table(g, rec.x, 0, nb, tab, G.gl, TPV);
        G.sync();
        const uint32_t *D = bdst + st;
        uint32_t cnt = 0;
        const uint32_t nq = (fill + 3) >> 2;
        for (uint32_t q = G.gl; q < nq; q += TPV) {
            const uint32_t e = q << 2;
            const uint32_t b = tab[e >> g.logB];
            uint32_t *slot = g.pool + ((size_t)b << g.logB) + (e & (g.B - 1));
            const uint4 v = *reinterpret_cast<const uint4 *>(slot);
            const uint32_t ev[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (e + j < fill && ev[j] != GV_TOMB) {
                    const uint32_t idx = lower_bound_u32(D, len, ev[j]);
                    if (idx < len && D[idx] == ev[j]) {
                        ++cnt;
                        found[st + idx] = 1;
                        if (DEL) slot[j] = GV_TOMB;
                    }
                }
            }
        }
        cnt = G.sum(cnt);
        if (G.gl == 0) {
            seg_found[s] = cnt;
            if (DEL && cnt) {
                g.vtx[u].z = rec.z - cnt;
                atomicAdd(&g.ctl->live_edges, (unsigned long long)(-(long long)cnt));
                if (!g.dirty[u]) {
                    g.dirty[u] = 1;
                    g.dirty_list[atomicAdd(&g.ctl->ndirty, 1ull)] = u;
                }
            }
        }
        G.sync();
    }
}

template <bool DEL>
__global__ void __launch_bounds__(BIG_THREADS) k_member_big(DevGraph g,
                                                            const uint32_t *__restrict__ seg_vertex,
                                                            const uint32_t *__restrict__ seg_start,
                                                            const uint32_t *__restrict__ bdst,
                                                            uint8_t *__restrict__ found,
                                                            uint32_t *__restrict__ seg_found,
                                                            const uint32_t *__restrict__ big_list) {
    __shared__ uint32_t tab[BIG_TAB];
    __shared__ uint32_t wt[33];
    if (DEL && g.ctl->batch_abort) return;
    const uint32_t nbig = (uint32_t)g.ctl->nbig;
    for (uint32_t i = blockIdx.x; i < nbig; i += gridDim.x) {
        const uint32_t s = big_list[i];
        const uint32_t u = seg_vertex[s];
        const uint32_t st = seg_start[s], len = seg_start[s + 1] - st;
        const uint4 rec = g.vtx[u];
        const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB);
        const uint32_t *D = bdst + st;
        uint32_t cnt = 0;
        for (uint32_t k0 = 0; k0 < nb; k0 += BIG_TAB) {
            const uint32_t kc = min((uint32_t)BIG_TAB, nb - k0);
            fill_block_table(g, rec.x, k0, kc, tab, threadIdx.x, BIG_THREADS);
            __syncthreads();
            const uint32_t e0 = k0 << g.logB;
            const uint32_t e1 = min(fill, (k0 + kc) << g.logB);
            const uint32_t nq = (e1 - e0 + 3) >> 2;
            for (uint32_t q = threadIdx.x; q < nq; q += BIG_THREADS) {
                const uint32_t e = e0 + (q << 2);
                const uint32_t b = tab[(e >> g.logB) - k0];
                uint32_t *slot = g.pool + ((size_t)b << g.logB) + (e & (g.B - 1));
                const uint4 v = *reinterpret_cast<const uint4 *>(slot);
                const uint32_t ev[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (e + j < fill && ev[j] != GV_TOMB) {
                        const uint32_t idx = lower_bound_u32(D, len, ev[j]);
                        if (idx < len && D[idx] == ev[j]) {
                            ++cnt;
                            found[st + idx] = 1;
                            if (DEL) slot[j] = GV_TOMB;
                        }
                    }
                }
            }
            __syncthreads();
        }
        cnt = cta_sum<uint32_t, BIG_THREADS>(cnt, wt);
        if (threadIdx.x == 0) {
            seg_found[s] = cnt;
            if (DEL && cnt) {
                g.vtx[u].z = rec.z - cnt;
                atomicAdd(&g.ctl->live_edges, (unsigned long long)(-(long long)cnt));
                if (!g.dirty[u]) {
                    g.dirty[u] = 1;
                    g.dirty_list[atomicAdd(&g.ctl->ndirty, 1ull)] = u;
                }
            }
        }
        __syncthreads();
    }
}

// -------------------------------------------------------------- plan/admit
__global__ void __launch_bounds__(UPD_THREADS) k_plan(DevGraph g, const uint32_t *__restrict__ seg_vertex,
                                                      const uint32_t *__restrict__ seg_start,
                                                      const uint32_t *__restrict__ seg_found,
                                                      uint32_t *__restrict__ seg_newblocks,
                                                      uint32_t *__restrict__ seg_blkbase) {
    if (g.ctl->batch_abort) return;
    const uint32_t nseg = (uint32_t)g.ctl->nseg;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < nseg; base += stride) {
        const uint32_t s = base + threadIdx.x;
        uint32_t need = 0;
        if (s < nseg) {
            const uint32_t u = seg_vertex[s];
            const uint32_t newcnt = (seg_start[s + 1] - seg_start[s]) - seg_found[s];
            const uint32_t fill = g.vtx[u].y;
            const uint32_t cap = blocks_for(fill, g.logB) << g.logB;
            const uint32_t room = cap - fill;
            const uint32_t extra = newcnt > room ? newcnt - room : 0u;
            need = (extra + g.B - 1) >> g.logB;
            seg_newblocks[s] = need;
        }
        const unsigned long long off = warp_agg_alloc(&g.ctl->alloc_cursor, need);
        if (s < nseg) seg_blkbase[s] = (uint32_t)off;
    }
}

__global__ void k_admit(Ctl *ctl) {
    if (!ctl->batch_abort && ctl->alloc_cursor > ctl->free_top) {
        ctl->batch_abort = 1;
        ctl->status |= GV_DEV_ERR_NOMEM;
    }
}

__global__ void k_finish(Ctl *ctl) {
    if (!ctl->batch_abort) ctl->free_top -= ctl->alloc_cursor;
    ctl->alloc_cursor = 0;
    ctl->nbig = 0;
    ctl->batch_abort = 0;
}

// Commits one stage of a multi-stage window but keeps the abort flag, so a
// window rejected in an earlier stage skips the later ones too.
__global__ void k_commit_keep_abort(Ctl *ctl) {
    if (!ctl->batch_abort) ctl->free_top -= ctl->alloc_cursor;
    ctl->alloc_cursor = 0;
    ctl->nbig = 0;
}

// ------------------------------------------------------------------- apply
// Pool index of new block t of a segment (popped from the top of the stack).
__device__ __forceinline__ uint32_t new_block(const DevGraph &g, unsigned long long top, uint32_t base,
                                              uint32_t t) {
    return g.free_stack[top - 1ull - (unsigned long long)(base + t)];
}

// Initialises the new blocks, then links them into the tree (two passes so
// a parent that is itself new is initialised before its child pointer is set).
template <typename SyncF>
__device__ __forceinline__ void link_new_blocks(const DevGraph &g, uint32_t u, uint4 rec, uint32_t nb_old,
                                                uint32_t nnew, uint32_t newfill,
                                                unsigned long long top, uint32_t base,
                                                uint32_t t0, uint32_t nt, SyncF sync) {
    for (uint32_t t = t0; t < nnew; t += nt) {
        const uint32_t k = nb_old + t;
        const uint32_t b = new_block(g, top, base, t);
        g.left[b] = GV_NIL;
        g.right[b] = GV_NIL;
        g.owner[b] = u;
        g.bcount[b] = min(g.B, newfill - (k << g.logB));
        g.pred[b] = (k == 0) ? GV_NIL : (t == 0 ? rec.w : new_block(g, top, base, t - 1));
    }
    sync();
    for (uint32_t t = t0; t < nnew; t += nt) {
        const uint32_t k = nb_old + t;
        if (k == 0) continue;
        const uint32_t b = new_block(g, top, base, t);
        const uint32_t pk = (k - 1) >> 1;
        const uint32_t pb = (pk >= nb_old) ? new_block(g, top, base, pk - nb_old)
                                           : cbt_block(g.left, g.right, rec.x, pk);
        if (k & 1u) g.left[pb] = b; else g.right[pb] = b;
    }
}

template <int TPV>
__global__ void __launch_bounds__(UPD_THREADS) k_apply(DevGraph g, const uint32_t *__restrict__ seg_vertex,
                                                       const uint32_t *__restrict__ seg_start,
                                                       const uint32_t *__restrict__ bdst,
                                                       const float *__restrict__ bw,
                                                       const uint8_t *__restrict__ found,
                                                       const uint32_t *__restrict__ seg_found,
                                                       const uint32_t *__restrict__ seg_newblocks,
                                                       const uint32_t *__restrict__ seg_blkbase) {
    constexpr int GPC = UPD_THREADS / TPV;
    if (g.ctl->batch_abort) return;
    const uint32_t nseg = (uint32_t)g.ctl->nseg;
    const unsigned long long top = g.ctl->free_top;
    Group<TPV> G;
    const uint32_t ngroups = gridDim.x * GPC;
    for (uint32_t s = blockIdx.x * GPC + threadIdx.x / TPV; s < nseg; s += ngroups) {
        const uint32_t u = seg_vertex[s];
        const uint32_t st = seg_start[s], len = seg_start[s + 1] - st;
        const uint4 rec = g.vtx[u];
        const uint32_t fill = rec.y, nb_old = blocks_for(fill, g.logB);
        if (is_big(nb_old, len)) continue;
        const uint32_t newcnt = len - seg_found[s];
        if (newcnt == 0) continue;
        const uint32_t nnew = seg_newblocks[s], base = seg_blkbase[s];
        const uint32_t newfill = fill + newcnt;
        uint32_t j0 = 0;
        for (uint32_t c = 0; c < len; c += TPV) {
            const uint32_t i = c + G.gl;
            const uint32_t isnew = (i < len && !found[st + i]) ? 1u : 0u;
            uint32_t tot;
            const uint32_t pre = G.excl_scan(isnew, tot);
            if (isnew) {
                const uint32_t p = fill + j0 + pre;
                const uint32_t k = p >> g.logB;
                const uint32_t b = (k < nb_old) ? rec.w : new_block(g, top, base, k - nb_old);
                const size_t at = ((size_t)b << g.logB) + (p & (g.B - 1));
                g.pool[at] = bdst[st + i];
                if (bw) g.wpool[at] = bw[st + i];
            }
            j0 += tot;
        }
        link_new_blocks(g, u, rec, nb_old, nnew, newfill, top, base, G.gl, TPV, [&] { G.sync(); });
        if (G.gl == 0) {
            if (nb_old > 0) g.bcount[rec.w] = min(g.B, newfill - ((nb_old - 1) << g.logB));
            uint4 nrec;
            nrec.x = nb_old ? rec.x : new_block(g, top, base, 0);
            nrec.y = newfill;
            nrec.z = rec.z + newcnt;
            nrec.w = nnew ? new_block(g, top, base, nnew - 1) : rec.w;
            g.vtx[u] = nrec;
            atomicAdd(&g.ctl->live_edges, (unsigned long long)newcnt);
        }
        G.sync();
    }
}

__global__ void __launch_bounds__(BIG_THREADS) k_apply_big(DevGraph g, const uint32_t *__restrict__ seg_vertex,
                                                           const uint32_t *__restrict__ seg_start,
                                                           const uint32_t *__restrict__ bdst,
                                                           const float *__restrict__ bw,
                                                           const uint8_t *__restrict__ found,
                                                           const uint32_t *__restrict__ seg_found,
                                                           const uint32_t *__restrict__ seg_newblocks,
                                                           const uint32_t *__restrict__ seg_blkbase,
                                                           const uint32_t *__restrict__ big_list) {
    __shared__ uint32_t wt[33];
    if (g.ctl->batch_abort) return;
    const uint32_t nbig = (uint32_t)g.ctl->nbig;
    const unsigned long long top = g.ctl->free_top;
    for (uint32_t bi = blockIdx.x; bi < nbig; bi += gridDim.x) {
        const uint32_t s = big_list[bi];
        const uint32_t u = seg_vertex[s];
        const uint32_t st = seg_start[s], len = seg_start[s + 1] - st;
        const uint4 rec = g.vtx[u];
        const uint32_t fill = rec.y, nb_old = blocks_for(fill, g.logB);
        const uint32_t newcnt = len - seg_found[s];
        if (newcnt == 0) continue;  // uniform across the CTA
        const uint32_t nnew = seg_newblocks[s], base = seg_blkbase[s];
        const uint32_t newfill = fill + newcnt;
        uint32_t j0 = 0;
        for (uint32_t c = 0; c < len; c += BIG_THREADS) {
            const uint32_t i = c + threadIdx.x;
            const uint32_t isnew = (i < len && !found[st + i]) ? 1u : 0u;
            uint32_t tot;
            const uint32_t pre = cta_excl_scan<uint32_t, BIG_THREADS>(isnew, wt, tot);
            if (isnew) {
                const uint32_t p = fill + j0 + pre;
                const uint32_t k = p >> g.logB;
                const uint32_t b = (k < nb_old) ? rec.w : new_block(g, top, base, k - nb_old);
                const size_t at = ((size_t)b << g.logB) + (p & (g.B - 1));
                g.pool[at] = bdst[st + i];
                if (bw) g.wpool[at] = bw[st + i];
            }
            j0 += tot;
        }
        link_new_blocks(g, u, rec, nb_old, nnew, newfill, top, base, threadIdx.x, BIG_THREADS,
                        [] { __syncthreads(); });
        __syncthreads();
        if (threadIdx.x == 0) {
            if (nb_old > 0) g.bcount[rec.w] = min(g.B, newfill - ((nb_old - 1) << g.logB));
            uint4 nrec;
            nrec.x = nb_old ? rec.x : new_block(g, top, base, 0);
            nrec.y = newfill;
            nrec.z = rec.z + newcnt;
            nrec.w = nnew ? new_block(g, top, base, nnew - 1) : rec.w;
            g.vtx[u] = nrec;
            atomicAdd(&g.ctl->live_edges, (unsigned long long)newcnt);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ window apply
// A window's net updates in one persistent launch.  The window has been
// reduced to the last operation per pair, so every touched vertex u has one
// segment: its destinations sorted, each marked insert or delete, and no
// pair appears twice.  Units of work are segments, taken from a device
// queue: first the big ones (more than BIG_BLOCKS blocks or BIG_SEGMENT
// entries), one per CTA, then chunks of WIN_CHUNK small ones per warp, a
// lane group per segment.  A unit scans u's blocks once: an entry found
// among the segment's deletes becomes a tombstone, one found among its
// inserts marks that insert as already present.  The remaining inserts are
// appended after the last used slot into blocks popped from the free stack
// (warp-aggregated atomics), the new blocks are linked into the CBT and the
// vertex record is rewritten.  The caller has checked that the free stack
// holds the window's worst case (one block per segment plus one per B
// inserts), so no unit can run out; a unit that would still overrun the
// stack records GV_DEV_ERR_NOMEM and writes nothing past it.
constexpr uint32_t WIN_CHUNK = 64;

struct WinSegs {
    const uint32_t *seg_vertex, *seg_start, *bdst;
    const uint32_t *btype;       // per entry: 1 insert, 0 delete
    uint8_t *found;              // per entry: the insert is already stored
    uint32_t *big_list;          // big segments
    unsigned long long *queue;   // [0] next big unit, [1] next small chunk, [2] big units
};

__device__ __forceinline__ uint32_t win_new_blocks(uint32_t fill, uint32_t nb_old, uint32_t newcnt, uint32_t logB) {
    const uint32_t room = (nb_old << logB) - fill;
    const uint32_t extra = newcnt > room ? newcnt - room : 0u;
    return (extra + (1u << logB) - 1u) >> logB;
}

// Rewrites u's record after a unit (one thread).
__device__ __forceinline__ void win_record(const DevGraph &g, uint32_t u, uint4 rec, uint32_t nb_old, uint32_t newcnt,
                                           uint32_t nnew, uint32_t ndel, unsigned long long top, uint32_t base) {
    if (!newcnt && !ndel) return;
    uint4 nrec = rec;
    if (newcnt) {
        const uint32_t newfill = rec.y + newcnt;
        if (nb_old > 0) g.bcount[rec.w] = min(g.B, newfill - ((nb_old - 1) << g.logB));
        nrec.x = nb_old ? rec.x : new_block(g, top, base, 0);
        nrec.y = newfill;
        nrec.w = nnew ? new_block(g, top, base, nnew - 1) : rec.w;
    }
    nrec.z = rec.z - ndel + newcnt;
    g.vtx[u] = nrec;
    atomicAdd(&g.ctl->live_edges, (unsigned long long)((long long)newcnt - (long long)ndel));
    if (ndel && !g.dirty[u]) {
        g.dirty[u] = 1;
        g.dirty_list[atomicAdd(&g.ctl->ndirty, 1ull)] = u;
    }
}

__global__ void k_window_classify(DevGraph g, WinSegs w) {
    const uint32_t nseg = (uint32_t)g.ctl->nseg;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x) {
        const uint32_t len = w.seg_start[s + 1] - w.seg_start[s];
        const uint32_t nb = blocks_for(g.vtx[w.seg_vertex[s]].y, g.logB);
        if (is_big(nb, len)) w.big_list[atomicAdd(&w.queue[2], 1ull)] = s;
    }
}

template <int TPV>
__global__ void __launch_bounds__(BIG_THREADS) k_window_apply(DevGraph g, WinSegs w) {
    constexpr int GPC = BIG_THREADS / TPV;
    constexpr int GPW = 32 / TPV;
    __shared__ uint32_t tab[BIG_TAB];
    __shared__ uint32_t tabs[GPC][BIG_BLOCKS];
    __shared__ uint32_t wt[33];
    __shared__ uint32_t unit_s;
    __shared__ unsigned long long base_s;
    if (g.ctl->batch_abort) return;
    const unsigned long long top = g.ctl->free_top;
    const uint32_t nbig = (uint32_t)w.queue[2];
    // ---- big segments: one CTA each
    for (;;) {
        if (threadIdx.x == 0) unit_s = (uint32_t)min(atomicAdd(&w.queue[0], 1ull), 0xFFFFFFFFull);
        __syncthreads();
        const uint32_t bi = unit_s;
        __syncthreads();
        if (bi >= nbig) break;
        const uint32_t s = w.big_list[bi];
        const uint32_t u = w.seg_vertex[s];
        const uint32_t st = w.seg_start[s], len = w.seg_start[s + 1] - st;
        const uint4 rec = g.vtx[u];
        const uint32_t fill = rec.y, nb_old = blocks_for(fill, g.logB);
        const uint32_t *D = w.bdst + st;
        const uint32_t *T = w.btype + st;
        uint32_t ndel = 0;
        for (uint32_t k0 = 0; k0 < nb_old; k0 += BIG_TAB) {
            const uint32_t kc = min((uint32_t)BIG_TAB, nb_old - k0);
            fill_block_table(g, rec.x, k0, kc, tab, threadIdx.x, BIG_THREADS);
            __syncthreads();
            const uint32_t e0 = k0 << g.logB;
            const uint32_t e1 = min(fill, (k0 + kc) << g.logB);
            const uint32_t nq = (e1 - e0 + 3) >> 2;
            for (uint32_t q = threadIdx.x; q < nq; q += BIG_THREADS) {
                const uint32_t e = e0 + (q << 2);
                uint32_t *slot = g.pool + ((size_t)tab[(e >> g.logB) - k0] << g.logB) + (e & (g.B - 1));
                const uint4 v = *reinterpret_cast<const uint4 *>(slot);
                const uint32_t ev[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (e + j < e1 && ev[j] != GV_TOMB) {
                        const uint32_t idx = lower_bound_u32(D, len, ev[j]);
                        if (idx < len && D[idx] == ev[j]) {
                            if (T[idx]) w.found[st + idx] = 1;
                            else {
                                slot[j] = GV_TOMB;
                                ++ndel;
                            }
                        }
                    }
                }
            }
            __syncthreads();
        }
        ndel = cta_sum<uint32_t, BIG_THREADS>(ndel, wt);
        uint32_t c = 0;
        for (uint32_t i = threadIdx.x; i < len; i += BIG_THREADS) c += (T[i] && !w.found[st + i]) ? 1u : 0u;
        const uint32_t newcnt = cta_sum<uint32_t, BIG_THREADS>(c, wt);
        uint32_t nnew = win_new_blocks(fill, nb_old, newcnt, g.logB);
        if (threadIdx.x == 0) base_s = nnew ? atomicAdd(&g.ctl->alloc_cursor, (unsigned long long)nnew) : 0ull;
        __syncthreads();
        const unsigned long long b64 = base_s;
        uint32_t ins = newcnt;
        if (b64 + nnew > top) {  // unreachable after the host's admission check; never write past the stack
            if (threadIdx.x == 0) atomicOr(&g.ctl->status, GV_DEV_ERR_NOMEM);
            ins = 0;
            nnew = 0;
        }
        const uint32_t base = (uint32_t)b64;
        if (ins) {
            uint32_t j0 = 0;
            for (uint32_t c0 = 0; c0 < len; c0 += BIG_THREADS) {
                const uint32_t i = c0 + threadIdx.x;
                const uint32_t isnew = (i < len && T[i] && !w.found[st + i]) ? 1u : 0u;
                uint32_t tot;
                const uint32_t pre = cta_excl_scan<uint32_t, BIG_THREADS>(isnew, wt, tot);
                if (isnew) {
                    const uint32_t p = fill + j0 + pre;
                    const uint32_t k = p >> g.logB;
                    const uint32_t b = (k < nb_old) ? rec.w : new_block(g, top, base, k - nb_old);
                    g.pool[((size_t)b << g.logB) + (p & (g.B - 1))] = D[i];
                }
                j0 += tot;
            }
            link_new_blocks(g, u, rec, nb_old, nnew, fill + ins, top, base, threadIdx.x, BIG_THREADS,
                            [] { __syncthreads(); });
            __syncthreads();
        }
        if (threadIdx.x == 0) win_record(g, u, rec, nb_old, ins, nnew, ndel, top, base);
        __syncthreads();
    }
    // ---- small segments: chunks per warp, a lane group per segment
    Group<TPV> G;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t gw = lane / TPV;
    uint32_t *mytab = tabs[threadIdx.x / TPV];
    const uint32_t nseg = (uint32_t)g.ctl->nseg;
    for (;;) {
        unsigned long long c0 = 0;
        if (lane == 0) c0 = atomicAdd(&w.queue[1], (unsigned long long)WIN_CHUNK);
        c0 = __shfl_sync(GV_FULL_MASK, c0, 0);
        if (c0 >= nseg) break;
        const uint32_t cend = (uint32_t)min((unsigned long long)nseg, c0 + WIN_CHUNK);
        for (uint32_t r = (uint32_t)c0; r < cend; r += GPW) {  // warp-uniform rounds
            const uint32_t s = r + gw;
            bool active = s < cend;
            uint32_t u = 0, st = 0, len = 0, fill = 0, nb_old = 0;
            uint4 rec = make_uint4(0, 0, 0, 0);
            if (active) {
                u = w.seg_vertex[s];
                st = w.seg_start[s];
                len = w.seg_start[s + 1] - st;
                rec = g.vtx[u];
                fill = rec.y;
                nb_old = blocks_for(fill, g.logB);
                active = !is_big(nb_old, len);
            }
            const uint32_t *D = w.bdst + st;
            const uint32_t *T = w.btype + st;
            uint32_t ndel = 0;
            if (active) {
                fill_block_table(g, rec.x, 0, nb_old, mytab, G.gl, TPV);
                G.sync();
                const uint32_t nq = (fill + 3) >> 2;
                for (uint32_t q = G.gl; q < nq; q += TPV) {
                    const uint32_t e = q << 2;
                    uint32_t *slot = g.pool + ((size_t)mytab[e >> g.logB] << g.logB) + (e & (g.B - 1));
                    const uint4 v = *reinterpret_cast<const uint4 *>(slot);
                    const uint32_t ev[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        if (e + j < fill && ev[j] != GV_TOMB) {
                            const uint32_t idx = lower_bound_u32(D, len, ev[j]);
                            if (idx < len && D[idx] == ev[j]) {
                                if (T[idx]) w.found[st + idx] = 1;
                                else {
                                    slot[j] = GV_TOMB;
                                    ++ndel;
                                }
                            }
                        }
                    }
                }
            }
            ndel = G.sum(ndel);
            G.sync();
            uint32_t c = 0;
            if (active)
                for (uint32_t i = G.gl; i < len; i += TPV) c += (T[i] && !w.found[st + i]) ? 1u : 0u;
            const uint32_t newcnt = G.sum(c);
            uint32_t nnew = active ? win_new_blocks(fill, nb_old, newcnt, g.logB) : 0u;
            const unsigned long long off = warp_agg_alloc(&g.ctl->alloc_cursor, (G.gl == 0) ? nnew : 0u);
            const unsigned long long b64 = G.bcast(off, 0);
            uint32_t ins = active ? newcnt : 0u;
            if (b64 + nnew > top) {  // see the admission note above
                if (active && G.gl == 0) atomicOr(&g.ctl->status, GV_DEV_ERR_NOMEM);
                ins = 0;
                nnew = 0;
            }
            const uint32_t base = (uint32_t)b64;
            if (ins) {
                uint32_t j0 = 0;
                for (uint32_t cc = 0; cc < len; cc += TPV) {
                    const uint32_t i = cc + G.gl;
                    const uint32_t isnew = (i < len && T[i] && !w.found[st + i]) ? 1u : 0u;
                    uint32_t tot;
                    const uint32_t pre = G.excl_scan(isnew, tot);
                    if (isnew) {
                        const uint32_t p = fill + j0 + pre;
                        const uint32_t k = p >> g.logB;
                        const uint32_t b = (k < nb_old) ? rec.w : new_block(g, top, base, k - nb_old);
                        g.pool[((size_t)b << g.logB) + (p & (g.B - 1))] = D[i];
                    }
                    j0 += tot;
                }
                link_new_blocks(g, u, rec, nb_old, nnew, fill + ins, top, base, G.gl, TPV, [&] { G.sync(); });
            }
            G.sync();
            if (active && G.gl == 0) win_record(g, u, rec, nb_old, ins, nnew, ndel, top, base);
            G.sync();
        }
    }
}

// -------------------------------------------------------------- compaction
// Stable in-place compaction of one vertex: live entries keep their order,
// tail blocks that end up empty go back to the free stack and are unlinked
// from their parents.  Replaces compactionVertexCentric
// (src/dynamicStructure/kernels/delete_kernels.cu:50-261), which fills holes
// from the tail and can drop live entries when a hole and the tail entry
// meet in the same block.
template <int TPV>
__global__ void __launch_bounds__(UPD_THREADS) k_compact(DevGraph g, uint32_t *__restrict__ big_list) {
    constexpr int GPC = UPD_THREADS / TPV;
    __shared__ uint32_t tabs[GPC][BIG_BLOCKS];
    const uint32_t nd = (uint32_t)g.ctl->ndirty;
    Group<TPV> G;
    uint32_t *tab = tabs[threadIdx.x / TPV];
    const uint32_t ngroups = gridDim.x * GPC;
    for (uint32_t di = blockIdx.x * GPC + threadIdx.x / TPV; di < nd; di += ngroups) {
        const uint32_t u = g.dirty_list[di];
        const uint4 rec = g.vtx[u];
        const uint32_t fill = rec.y, live = rec.z, nb = blocks_for(fill, g.logB);
        if (nb > BIG_BLOCKS) {
            if (G.gl == 0) big_list[atomicAdd(&g.ctl->nbig, 1ull)] = u;
            continue;
        }
        fill_block_table(g, rec.x, 0, nb, tab, G.gl, TPV);
        G.sync();
        uint32_t wpos = 0;
        const uint32_t nq = (fill + 3) >> 2;
        for (uint32_t q0 = 0; q0 < nq; q0 += TPV) {
            const uint32_t q = q0 + G.gl;
            uint32_t ev[4] = {GV_TOMB, GV_TOMB, GV_TOMB, GV_TOMB};
            float wv[4] = {0.f, 0.f, 0.f, 0.f};
            uint32_t c = 0;
            if (q < nq) {
                const uint32_t e = q << 2;
                const size_t at = ((size_t)tab[e >> g.logB] << g.logB) + (e & (g.B - 1));
                const uint4 v = *reinterpret_cast<const uint4 *>(g.pool + at);
                ev[0] = v.x; ev[1] = v.y; ev[2] = v.z; ev[3] = v.w;
                if (g.weighted) {
                    const float4 w = *reinterpret_cast<const float4 *>(g.wpool + at);
                    wv[0] = w.x; wv[1] = w.y; wv[2] = w.z; wv[3] = w.w;
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (e + j >= fill) ev[j] = GV_TOMB;
                    c += (ev[j] != GV_TOMB);
                }
            }
            uint32_t tot;
            uint32_t p = wpos + G.excl_scan(c, tot);
            G.sync();
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (ev[j] != GV_TOMB) {
                    const size_t at = ((size_t)tab[p >> g.logB] << g.logB) + (p & (g.B - 1));
                    g.pool[at] = ev[j];
                    if (g.weighted) g.wpool[at] = wv[j];
                    ++p;
                }
            }
            wpos += tot;
        }
        G.sync();
        const uint32_t nb_new = blocks_for(live, g.logB);
        const uint32_t nfree = nb - nb_new;
        unsigned long long fbase = 0;
        if (G.gl == 0 && nfree) fbase = atomicAdd(&g.ctl->free_top, (unsigned long long)nfree);
        fbase = G.bcast(fbase, 0);
        for (uint32_t t = G.gl; t < nfree; t += TPV) {
            const uint32_t k = nb_new + t;
            g.free_stack[fbase + t] = tab[k];
            const uint32_t pk = (k - 1) >> 1;
            if (k > 0 && pk < nb_new) {
                if (k & 1u) g.left[tab[pk]] = GV_NIL; else g.right[tab[pk]] = GV_NIL;
            }
        }
        if (G.gl == 0) {
            if (nb_new) g.bcount[tab[nb_new - 1]] = live - ((nb_new - 1) << g.logB);
            g.vtx[u] = make_uint4(nb_new ? rec.x : GV_NIL, live, live, nb_new ? tab[nb_new - 1] : GV_NIL);
            g.dirty[u] = 0;
        }
        G.sync();
    }
}

__global__ void __launch_bounds__(BIG_THREADS) k_compact_big(DevGraph g, const uint32_t *__restrict__ big_list) {
    __shared__ uint32_t tab[BIG_TAB];
    __shared__ uint32_t wt[33];
    __shared__ unsigned long long fbase_s;
    const uint32_t nbig = (uint32_t)g.ctl->nbig;
    for (uint32_t bi = blockIdx.x; bi < nbig; bi += gridDim.x) {
        const uint32_t u = big_list[bi];
        const uint4 rec = g.vtx[u];
        const uint32_t fill = rec.y, live = rec.z, nb = blocks_for(fill, g.logB);
        uint32_t wpos = 0;
        for (uint32_t k0 = 0; k0 < nb; k0 += BIG_TAB) {
            const uint32_t kc = min((uint32_t)BIG_TAB, nb - k0);
            fill_block_table(g, rec.x, k0, kc, tab, threadIdx.x, BIG_THREADS);
            __syncthreads();
            const uint32_t e0 = k0 << g.logB;
            const uint32_t e1 = min(fill, (k0 + kc) << g.logB);
            const uint32_t nq = (e1 - e0 + 3) >> 2;
            for (uint32_t q0 = 0; q0 < nq; q0 += BIG_THREADS) {
                const uint32_t q = q0 + threadIdx.x;
                uint32_t ev[4] = {GV_TOMB, GV_TOMB, GV_TOMB, GV_TOMB};
                float wv[4] = {0.f, 0.f, 0.f, 0.f};
                uint32_t c = 0;
                if (q < nq) {
                    const uint32_t e = e0 + (q << 2);
                    const size_t at = ((size_t)tab[(e >> g.logB) - k0] << g.logB) + (e & (g.B - 1));
                    const uint4 v = *reinterpret_cast<const uint4 *>(g.pool + at);
                    ev[0] = v.x; ev[1] = v.y; ev[2] = v.z; ev[3] = v.w;
                    if (g.weighted) {
                        const float4 w = *reinterpret_cast<const float4 *>(g.wpool + at);
                        wv[0] = w.x; wv[1] = w.y; wv[2] = w.z; wv[3] = w.w;
                    }
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        if (e + j >= fill) ev[j] = GV_TOMB;
                        c += (ev[j] != GV_TOMB);
                    }
                }
                uint32_t tot;
                uint32_t p = wpos + cta_excl_scan<uint32_t, BIG_THREADS>(c, wt, tot);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (ev[j] != GV_TOMB) {
                        const uint32_t kd = p >> g.logB;
                        const uint32_t b = (kd >= k0) ? tab[kd - k0] : cbt_block(g.left, g.right, rec.x, kd);
                        const size_t at = ((size_t)b << g.logB) + (p & (g.B - 1));
                        g.pool[at] = ev[j];
                        if (g.weighted) g.wpool[at] = wv[j];
                        ++p;
                    }
                }
                wpos += tot;
                __syncthreads();
            }
        }
        // Free the tail blocks.  Walks only touch surviving ancestors, whose
        // links to other survivors are not modified here.
        const uint32_t nb_new = blocks_for(live, g.logB);
        const uint32_t nfree = nb - nb_new;
        if (threadIdx.x == 0) fbase_s = nfree ? atomicAdd(&g.ctl->free_top, (unsigned long long)nfree) : 0ull;
        __syncthreads();
        const unsigned long long fbase = fbase_s;
        for (uint32_t t = threadIdx.x; t < nfree; t += BIG_THREADS) {
            const uint32_t k = nb_new + t;
            g.free_stack[fbase + t] = cbt_block(g.left, g.right, rec.x, k);
        }
        __syncthreads();
        for (uint32_t t = threadIdx.x; t < nfree; t += BIG_THREADS) {
            const uint32_t k = nb_new + t;
            const uint32_t pk = (k - 1) >> 1;
            if (k > 0 && pk < nb_new) {
                const uint32_t pb = cbt_block(g.left, g.right, rec.x, pk);
                if (k & 1u) g.left[pb] = GV_NIL; else g.right[pb] = GV_NIL;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const uint32_t lb = nb_new ? cbt_block(g.left, g.right, rec.x, nb_new - 1) : GV_NIL;
            if (nb_new) g.bcount[lb] = live - ((nb_new - 1) << g.logB);
            g.vtx[u] = make_uint4(nb_new ? rec.x : GV_NIL, live, live, lb);
            g.dirty[u] = 0;
        }
        __syncthreads();
    }
}

__global__ void k_compact_done(Ctl *ctl) {
    ctl->ndirty = 0;
    ctl->nbig = 0;
}

// --------------------------------------------------------- vertex delete
// Every entry of a flagged vertex, and every entry pointing at one, becomes
// a tombstone; live counts, the control block and the dirty list change as a
// batch delete changes them, so gv_compact reclaims the blocks.
template <int TPV>
__global__ void __launch_bounds__(UPD_THREADS) k_vertex_delete(DevGraph g, const uint8_t *__restrict__ del) {
    Group<TPV> G;
    constexpr int GPC = UPD_THREADS / TPV;
    const uint32_t ngroups = gridDim.x * GPC;
    for (uint32_t u = blockIdx.x * GPC + threadIdx.x / TPV; u < g.n; u += ngroups) {
        const uint4 rec = g.vtx[u];
        const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB);
        if (rec.z == 0) continue;
        const bool all = del[u] != 0;
        uint32_t cnt = 0;
        for (uint32_t k = 0; k < nb; ++k) {
            const uint32_t b = (k == 0) ? rec.x : cbt_block(g.left, g.right, rec.x, k);
            const uint32_t slots = min(g.B, fill - (k << g.logB));
            uint32_t *blk = g.pool + ((size_t)b << g.logB);
            for (uint32_t i = G.gl; i < slots; i += TPV) {
                const uint32_t v = blk[i];
                if (v != GV_TOMB && (all || del[v])) {
                    blk[i] = GV_TOMB;
                    g.affected[v] = 1;
                    ++cnt;
                }
            }
        }
        cnt = G.sum(cnt);
        if (G.gl == 0 && cnt) {
            g.vtx[u].z = rec.z - cnt;
            g.affected[u] = 1;
            atomicAdd(&g.ctl->live_edges, (unsigned long long)(-(long long)cnt));
            if (!g.dirty[u]) {
                g.dirty[u] = 1;
                g.dirty_list[atomicAdd(&g.ctl->ndirty, 1ull)] = u;
            }
        }
    }
}

// ------------------------------------------------------------------ export
template <int TPV>
__global__ void __launch_bounds__(UPD_THREADS) k_export(DevGraph g, const unsigned long long *__restrict__ off,
                                                        uint32_t *__restrict__ out, float *__restrict__ wout) {
    Group<TPV> G;
    constexpr int GPC = UPD_THREADS / TPV;
    const uint32_t ngroups = gridDim.x * GPC;
    for (uint32_t u = blockIdx.x * GPC + threadIdx.x / TPV; u < g.n; u += ngroups) {
        const uint4 rec = g.vtx[u];
        const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB);
        unsigned long long w = off[u];
        const unsigned long long wend = off[u + 1];  // bounds every write of this vertex
        for (uint32_t k = 0; k < nb; ++k) {
            const uint32_t b = (k == 0) ? rec.x : cbt_block(g.left, g.right, rec.x, k);
            const uint32_t slots = min(g.B, fill - (k << g.logB));
            for (uint32_t c = 0; c < slots; c += TPV) {
                const uint32_t i = c + G.gl;
                const size_t at = ((size_t)b << g.logB) + i;
                const uint32_t v = (i < slots) ? g.pool[at] : GV_TOMB;
                const uint32_t keep = v != GV_TOMB;
                uint32_t tot;
                const uint32_t pre = G.excl_scan(keep, tot);
                if (keep && w + pre < wend) {
                    out[w + pre] = v;
                    if (wout) wout[w + pre] = g.wpool[at];
                }
                w += tot;
            }
        }
    }
}

__global__ void k_live_degrees(DevGraph g, uint32_t *__restrict__ deg) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < g.n; u += gridDim.x * blockDim.x)
        deg[u] = g.vtx[u].z;
}

// ------------------------------------------------------------------- check
// Codes: 1 root/fill mismatch, 2 live > fill, 3 bad block index, 4 owner,
// 5 block count, 6 predecessor, 7 left child, 8 right child, 9 last block,
// 10 live count, 11 block used twice or lost, 12 bad free entry, 13 totals.
__device__ void report(unsigned long long *viol, uint32_t *first, uint32_t code, uint32_t u) {
    if (atomicAdd(viol, 1ull) == 0) {
        first[0] = code;
        first[1] = u;
    }
}

__global__ void k_check_vertices(DevGraph g, uint32_t *__restrict__ mark, unsigned long long *viol,
                                 uint32_t *first, unsigned long long *used_blocks) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < g.n; u += gridDim.x * blockDim.x) {
        const uint4 rec = g.vtx[u];
        const uint32_t fill = rec.y, live = rec.z, nb = blocks_for(fill, g.logB);
        if ((fill == 0) != (rec.x == GV_NIL)) { report(viol, first, 1, u); continue; }
        if (live > fill) report(viol, first, 2, u);
        if (nb == 0) continue;
        atomicAdd(used_blocks, (unsigned long long)nb);
        uint32_t prev = GV_NIL, cnt = 0;
        bool ok = true;
        for (uint32_t k = 0; k < nb && ok; ++k) {
            // walk with bounds checks
            uint32_t p = k + 1, b = rec.x;
            int d = 31 - __clz(p);
            for (int i = d - 1; i >= 0; --i) {
                if (b >= g.P) break;
                b = ((p >> i) & 1u) ? g.right[b] : g.left[b];
            }
            if (b >= g.P) { report(viol, first, 3, u); ok = false; break; }
            atomicAdd(&mark[b], 1u);
            if (g.owner[b] != u) report(viol, first, 4, u);
            const uint32_t want = (k + 1 < nb) ? g.B : fill - ((nb - 1) << g.logB);
            if (g.bcount[b] != want) report(viol, first, 5, u);
            if (k > 0 && g.pred[b] != prev) report(viol, first, 6, u);
            const bool hl = 2 * k + 1 < nb, hr = 2 * k + 2 < nb;
            if (hl != (g.left[b] != GV_NIL)) report(viol, first, 7, u);
            if (hr != (g.right[b] != GV_NIL)) report(viol, first, 8, u);
            const uint32_t slots = min(g.B, fill - (k << g.logB));
            for (uint32_t i = 0; i < slots; ++i) cnt += (g.pool[((size_t)b << g.logB) + i] != GV_TOMB);
            prev = b;
        }
        if (ok && prev != rec.w) report(viol, first, 9, u);
        if (ok && cnt != live) report(viol, first, 10, u);
    }
}

__global__ void k_check_free(DevGraph g, uint32_t *__restrict__ mark, unsigned long long *viol, uint32_t *first) {
    unsigned long long top = g.ctl->free_top;
    if (top > g.P) {
        if (blockIdx.x == 0 && threadIdx.x == 0) report(viol, first, 13, 0);
        top = g.P;
    }
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < top;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const uint32_t b = g.free_stack[i];
        if (b >= g.P) { report(viol, first, 12, 0); continue; }
        atomicAdd(&mark[b], 1u);
    }
}

__global__ void k_check_marks(DevGraph g, const uint32_t *__restrict__ mark, unsigned long long *viol,
                              uint32_t *first, const unsigned long long *used_blocks) {
    for (unsigned long long b = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; b < g.P;
         b += (unsigned long long)gridDim.x * blockDim.x)
        if (mark[b] != 1u) report(viol, first, 11, (uint32_t)b);
    if (blockIdx.x == 0 && threadIdx.x == 0 && *used_blocks + g.ctl->free_top != g.P)
        report(viol, first, 13, 0);
}

}  // namespace

// ====================================================================== host
gv_status run_update(gv_graph *g, const uint32_t *dsrc, const uint32_t *ddst, const float *dw,
                     uint64_t k, bool symmetric, bool is_delete, cudaStream_t s) {
    BatchScratch &bs = g->bs;
    const uint64_t E = symmetric ? 2 * k : k;
    const bool vals = (dw != nullptr) && !is_delete;
    int which = 0;
    {
        ProfScope ps(PROF_RADIX, s);
        GV_LAUNCH(k_expand, grid_for(k, 256), 256, 0, s, dsrc, ddst, k, symmetric ? 1 : 0, g->d.n,
                  g->bitsn, bs.keys, vals ? bs.vals : nullptr, g->d.ctl);
        which = radix_sort_u64(bs.keys, bs.keys_alt, vals ? bs.vals : nullptr, vals ? bs.vals_alt : nullptr,
                               E, 2 * (int)g->bitsn, bs.rs_counts, bs.scan_tmp, s);
    }
    const unsigned long long *K = which ? bs.keys_alt : bs.keys;
    const uint32_t *V = which ? bs.vals_alt : bs.vals;
    return apply_sorted(g, K, vals ? V : nullptr, E, symmetric, dw, is_delete, true, s);
}

void launch_commit_keep_abort(gv_graph *g, cudaStream_t s) {
    GV_LAUNCH(k_commit_keep_abort, 1, 1, 0, s, g->d.ctl);
}

void launch_finish(gv_graph *g, cudaStream_t s) { GV_LAUNCH(k_finish, 1, 1, 0, s, g->d.ctl); }

gv_status launch_window_apply(gv_graph *g, const uint32_t *seg_vertex, const uint32_t *seg_start,
                              const uint32_t *bdst, const uint32_t *btype, uint8_t *found, uint32_t *big_list,
                              unsigned long long *queue, cudaStream_t s) {
    DevGraph d = g->d;
    WinSegs w{seg_vertex, seg_start, bdst, btype, found, big_list, queue};
    {
        ProfScope ps(PROF_MEMBER, s);
        GV_LAUNCH(k_window_classify, 148 * 4, 256, 0, s, d, w);
    }
    {
        ProfScope ps(PROF_APPLY, s);
        dispatch_tpv(g->cfg.threads_per_vertex, [&](auto t) {
            constexpr int T = decltype(t)::value;
            GV_LAUNCH((k_window_apply<T>), 148 * 2, BIG_THREADS, 0, s, d, w);
        });
    }
    GV_LAUNCH(k_finish, 1, 1, 0, s, d.ctl);
    return cuda_status(cudaGetLastError(), "window apply launch");
}

gv_status apply_sorted(gv_graph *g, const unsigned long long *K, const uint32_t *V, uint64_t E, bool symmetric,
                       const float *dw, bool is_delete, bool finish, cudaStream_t s) {
    BatchScratch &bs = g->bs;
    const bool vals = (V != nullptr) && (dw != nullptr) && !is_delete;
    const unsigned long long sent = (g->bitsn >= 32) ? ~0ull : ((1ull << (2 * g->bitsn)) - 1ull);
    const unsigned ntiles = (unsigned)((E + SEG_TILE - 1) / SEG_TILE);
    {
        ProfScope ps(PROF_SEGMENT, s);
        GV_LAUNCH(k_seg_count, ntiles, SEG_THREADS, 0, s, K, E, sent, g->bitsn, bs.tile_cnt);
        scan_exclusive_u64(bs.tile_cnt, bs.tile_cnt, ntiles, &g->d.ctl->scratch0, bs.scan_tmp, s);
        GV_LAUNCH(k_seg_write, ntiles, SEG_THREADS, 0, s, K, V, E, sent, g->bitsn, symmetric ? 1 : 0,
                  (const unsigned long long *)bs.tile_cnt, dw, bs.bdst, vals ? bs.bw : nullptr, bs.found,
                  bs.seg_vertex, bs.seg_start, g->d.affected, g->d.ctl);
    }
    // Segments <= unique entries <= E.
    const unsigned gsmall = grid_for(E, 64);
    const unsigned gbig = 148 * 2;
    const uint32_t tpv = g->cfg.threads_per_vertex;
    DevGraph d = g->d;
    {
        ProfScope ps(PROF_MEMBER, s);
        dispatch_tpv(tpv, [&](auto t) {
            constexpr int T = decltype(t)::value;
            if (is_delete)
                GV_LAUNCH((k_member<T, true>), gsmall, UPD_THREADS, 0, s, d, bs.seg_vertex, bs.seg_start,
                          bs.bdst, bs.found, bs.seg_found, bs.big_list);
            else
                GV_LAUNCH((k_member<T, false>), gsmall, UPD_THREADS, 0, s, d, bs.seg_vertex, bs.seg_start,
                          bs.bdst, bs.found, bs.seg_found, bs.big_list);
        });
        if (is_delete)
            GV_LAUNCH(k_member_big<true>, gbig, BIG_THREADS, 0, s, d, bs.seg_vertex, bs.seg_start, bs.bdst,
                      bs.found, bs.seg_found, bs.big_list);
        else
            GV_LAUNCH(k_member_big<false>, gbig, BIG_THREADS, 0, s, d, bs.seg_vertex, bs.seg_start, bs.bdst,
                      bs.found, bs.seg_found, bs.big_list);
    }
    if (!is_delete) {
        ProfScope ps(PROF_APPLY, s);
        GV_LAUNCH(k_plan, grid_for(E, UPD_THREADS), UPD_THREADS, 0, s, d, bs.seg_vertex, bs.seg_start,
                  bs.seg_found, bs.seg_newblocks, bs.seg_blkbase);
        GV_LAUNCH(k_admit, 1, 1, 0, s, d.ctl);
        dispatch_tpv(tpv, [&](auto t) {
            constexpr int T = decltype(t)::value;
            GV_LAUNCH((k_apply<T>), gsmall, UPD_THREADS, 0, s, d, bs.seg_vertex, bs.seg_start, bs.bdst,
                      vals ? bs.bw : nullptr, bs.found, bs.seg_found, bs.seg_newblocks, bs.seg_blkbase);
        });
        GV_LAUNCH(k_apply_big, gbig, BIG_THREADS, 0, s, d, bs.seg_vertex, bs.seg_start, bs.bdst,
                  vals ? bs.bw : nullptr, bs.found, bs.seg_found, bs.seg_newblocks, bs.seg_blkbase,
                  bs.big_list);
    }
    if (finish) GV_LAUNCH(k_finish, 1, 1, 0, s, d.ctl);
    else GV_LAUNCH(k_commit_keep_abort, 1, 1, 0, s, d.ctl);
    return cuda_status(cudaGetLastError(), "update launch");
}

gv_status run_compact(gv_graph *g, cudaStream_t s) {
    DevGraph d = g->d;
    ProfScope ps(PROF_COMPACT, s);
    // The dirty list holds at most n vertices; size the grid for it.
    const unsigned grid = grid_for(g->d.n, 64);
    dispatch_tpv(g->cfg.threads_per_vertex, [&](auto t) {
        constexpr int T = decltype(t)::value;
        GV_LAUNCH((k_compact<T>), grid, UPD_THREADS, 0, s, d, d.vbig_list);
    });
    GV_LAUNCH(k_compact_big, 148 * 2, BIG_THREADS, 0, s, d, (const uint32_t *)d.vbig_list);
    GV_LAUNCH(k_compact_done, 1, 1, 0, s, d.ctl);
    return cuda_status(cudaGetLastError(), "compact launch");
}

gv_status run_export(gv_graph *g, unsigned long long *offsets, uint32_t *dst, float *w, cudaStream_t s) {
    DevGraph d = g->d;
    dispatch_tpv(g->cfg.threads_per_vertex, [&](auto t) {
        constexpr int T = decltype(t)::value;
        GV_LAUNCH((k_export<T>), grid_for(g->d.n, UPD_THREADS / T), UPD_THREADS, 0, s, d, offsets, dst, w);
    });
    return cuda_status(cudaGetLastError(), "export launch");
}

gv_status run_vertex_delete(gv_graph *g, const uint8_t *del, cudaStream_t s) {
    DevGraph d = g->d;
    dispatch_tpv(g->cfg.threads_per_vertex, [&](auto t) {
        constexpr int T = decltype(t)::value;
        GV_LAUNCH((k_vertex_delete<T>), grid_for(g->d.n, UPD_THREADS / T), UPD_THREADS, 0, s, d, del);
    });
    return cuda_status(cudaGetLastError(), "vertex delete launch");
}

void launch_degrees(gv_graph *g, uint32_t *deg, cudaStream_t s) {
    GV_LAUNCH(k_live_degrees, grid_for(g->d.n, 256), 256, 0, s, g->d, deg);
}

gv_status run_check(gv_graph *g, uint64_t *violations, uint32_t *code, uint32_t *vertex) {
    DevGraph d = g->d;
    uint32_t *mark = nullptr;
    unsigned long long *cnt = nullptr;
    cudaError_t e = cudaMalloc(&mark, d.P * sizeof(uint32_t));
    if (e != cudaSuccess) return cuda_status(e, "check alloc");
    e = cudaMalloc(&cnt, 4 * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        cudaFree(mark);
        return cuda_status(e, "check alloc");
    }
    cudaMemset(mark, 0, d.P * sizeof(uint32_t));
    cudaMemset(cnt, 0, 4 * sizeof(unsigned long long));
    unsigned long long *viol = cnt, *used = cnt + 1;
    uint32_t *first = reinterpret_cast<uint32_t *>(cnt + 2);
    GV_LAUNCH(k_check_vertices, grid_for(d.n, 256), 256, 0, 0, d, mark, viol, first, used);
    GV_LAUNCH(k_check_free, grid_for(d.P, 256), 256, 0, 0, d, mark, viol, first);
    GV_LAUNCH(k_check_marks, grid_for(d.P, 256), 256, 0, 0, d, (const uint32_t *)mark, viol, first,
              (const unsigned long long *)used);
    unsigned long long h[4] = {0, 0, 0, 0};
    e = cudaMemcpy(h, cnt, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(mark);
    cudaFree(cnt);
    if (e != cudaSuccess) return cuda_status(e, "check");
    *violations = h[0];
    const uint32_t *f = reinterpret_cast<const uint32_t *>(&h[2]);
    if (code) *code = f[0];
    if (vertex) *vertex = f[1];
    return GV_OK;
}

}  // namespace gv
