// Betweenness centrality (Brandes) and single-source BFS path counts over the
// edge-block store, 32 or 64 sources per pass, sources spread over the lanes.
//
// Replaces the reference's bc (src/algorithm/bc/bc.cu:3-88) and its kernels
// initializeArrays / initbfsKernel / bfsKernel / dependencyKernel
// (src/algorithm/bc/bc_kernel.cu:3-119), which run one source per host loop
// and one level per launch with int path counts and an unordered dependency
// pass.  Here the sources of a pass share every adjacency read.  A pass keeps
// NW 32-bit words of source bits per vertex (NW = 1: 32 sources, NW = 2: 64);
// source slot s sits in lane s % 32, half s / 32.
//
//   forward, level L -> L+1, push (top-down over the union frontier): a warp takes
//   a vertex u at level L for the sources in mask F = masks[L][u]; each lane
//   holds sigma_s(u) of its NW sources.  For each neighbour w (ids read 32 at
//   a time, coalesced), want = F & ~vis[w] are the sources that reach w first
//   through this level; the neighbours with want != 0 are packed and visited:
//   one atomicOr marks want in nxt[w], each source in want adds sigma_s(u)
//   into sigma_s(w) (exact uint64 adds, so the order does not matter).
//
//   forward, pull (bottom-up, chosen per level on the device when the level
//   holds many entries; 64-source passes only): a warp takes a vertex w that
//   some source has not reached, sums sigma_s(u) over its neighbours u at level
//   L for those sources and writes its row and nxt[w] once, without atomics.
//
//   backward, level L (pull, no atomics): a warp takes v at level L for the
//   sources in A = masks[L][v]; for each neighbour w, the sources in
//   A & masks[L+1][w] (w one level deeper for them) add
//   coef_s(w) = (1 + delta_s(w)) / sigma_s(w).  Then delta_s(v) =
//   sigma_s(v) * acc_s, coef_s(v) replaces sigma_s(v) in the same 8-byte slot,
//   and each half of the pass adds the sum of its 32 deltas (fixed shuffle
//   order, fp64) into its own output row, so one pass can serve two requests.
//
// Level masks stay resident for the backward pass; sigma / coef rows are
// vertex-major ([v][32 NW] x 8 bytes), so the lanes of one vertex and half
// touch one 256-byte segment.  Vertices with more than MS_HEAVY_FILL entries
// are expanded by a whole CTA (block table in shared memory, warps over
// blocks); the backward partials of a CTA are combined in warp order, so
// results are bit-for-bit repeatable.
#include <algorithm>
#include <cstdlib>
#include <string>
#include <vector>
#include "store.cuh"
#include "launch.hpp"
#include "prof.hpp"

namespace gv {
namespace {

constexpr int MS_THREADS = 256;
constexpr int MS_WARPS = MS_THREADS / 32;
constexpr uint32_t MS_HEAVY_FILL = 1024;  // entries; above: one CTA per vertex
constexpr uint32_t MS_TAB = 2048;         // blocks per shared-memory table window
// CTAs of a level launch: many small shares, so the block scheduler evens
// out the heavy-tailed work per vertex.  BC at R-MAT scale 25 (32 / 64
// sources): 283 / 382 ms with 148 * (8 + 2) CTAs, 241 / 339 with twice as
// many, 214 / 284 with 8 times, 207 / 287 with 16 times (this), 204 / 282
// with 32 times.
constexpr unsigned MS_LIGHT_GRID = 148 * 128;
constexpr unsigned MS_HEAVY_GRID = 148 * 32;
constexpr uint32_t MS_MAX_LEVELS = 1u << 16;
constexpr uint32_t MS_MAX_NW = 2;

template <int NW> struct MaskOf;
template <> struct MaskOf<1> { using type = uint32_t; };
template <> struct MaskOf<2> { using type = unsigned long long; };

template <int NW>
struct MsBufs {
    using M = typename MaskOf<NW>::type;
    unsigned long long *row;  // [n][32 NW] sigma (u64); after its level's backward step: coef (f64 bits)
    M *vis;                   // [n] sources that reached v at a finished level
    M *nxt;                   // [n] sources that reach v at the level being built
    M *masks;                 // [levels][n]
    uint32_t *light;          // vertices of the current level, fill <= MS_HEAVY_FILL
    uint32_t *heavy;          // the rest
    uint32_t *cnt;            // [0] light, [1] heavy, [2] light candidates, [3] heavy candidates
    uint32_t *flags;          // [levels] level non-empty
    double *bc;               // [outputs][n]; half k of the pass adds into row out[k]
    uint32_t *clight;         // pull levels: vertices some source has not reached, fill <= MS_HEAVY_FILL
    uint32_t *cheavy;         // the rest of them
    unsigned long long *esum; // [0] entries of the level's vertices; [1] entries of the vertices some
                              // source has not reached (counted down by k_ms_close as vertices fill up)
    M full;                   // the pass's sources
    uint32_t alpha;           // pull when alpha * esum[0] > esum[1] (0: always push)
    uint32_t n;
    uint32_t out[2];
};

// Scratch of one call, carved once for the widest pass it runs.
struct MsArena {
    unsigned long long *row;
    void *vis, *nxt;
    uint32_t *light, *heavy, *clight, *cheavy, *cnt, *flags, *dsrc, *hflags;
    unsigned long long *esum;
    double *bc;
    uint32_t n;

    template <int NW>
    MsBufs<NW> bufs(gv_graph *g) const {
        using M = typename MaskOf<NW>::type;
        MsBufs<NW> b;
        b.row = row;
        b.vis = (M *)vis;
        b.nxt = (M *)nxt;
        b.masks = (M *)g->aux[6];
        b.light = light;
        b.heavy = heavy;
        b.cnt = cnt;
        b.flags = flags;
        b.bc = bc;
        b.clight = clight;
        b.cheavy = cheavy;
        b.esum = esum;
        b.full = 0;
        b.alpha = 0;
        b.n = n;
        b.out[0] = b.out[1] = 0;
        return b;
    }
};

template <int NW>
struct alignas(8) Packed {
    uint32_t w;
    typename MaskOf<NW>::type m;
};

__device__ __forceinline__ double as_f64(unsigned long long x) { return __longlong_as_double((long long)x); }
__device__ __forceinline__ unsigned long long as_u64(double x) { return (unsigned long long)__double_as_longlong(x); }

// Source bit of lane `lane`, half k.
template <typename M>
__device__ __forceinline__ bool has_src(M m, uint32_t lane, int k) {
    return (m >> (lane + 32u * (uint32_t)k)) & 1u;
}

__device__ __forceinline__ uint32_t ms_block(const DevGraph &g, uint32_t root, uint32_t k) {
    return k == 0 ? root : cbt_block(g.left, g.right, root, k);
}

// Walks the entries of one block 32 at a time: lane j loads entry e0 + j and
// its source mask pre(w) (0: nothing to do for any source); the entries with
// a non-zero mask are packed into the warp's shared slots, and body(w, mask)
// runs for each of them with the whole warp.  In most levels few entries need
// work, so the warp skips the rest without touching them.
template <int NW, typename Pre, typename Body>
__device__ __forceinline__ void ms_block_entries(const DevGraph &g, uint32_t b, uint32_t slots, Pre &&pre,
                                                 Body &&body) {
    using M = typename MaskOf<NW>::type;
    __shared__ Packed<NW> pack_all[MS_WARPS][32];  // one row of slots per warp (MS_THREADS threads)
    const uint32_t lane = threadIdx.x & 31u;
    Packed<NW> *pack = pack_all[threadIdx.x >> 5];
    const uint32_t *bp = g.pool + ((size_t)b << g.logB);
    for (uint32_t e0 = 0; e0 < slots; e0 += 32) {
        const uint32_t e = e0 + lane;
        uint32_t w = GV_TOMB;
        M pv = 0;
        if (e < slots) {
            w = bp[e];
            if (w != GV_TOMB) pv = pre(w);
        }
        const uint32_t bal = __ballot_sync(GV_FULL_MASK, pv != 0);
        if (!bal) continue;  // warp-uniform
        if (pv) pack[__popc(bal & ((1u << lane) - 1u))] = Packed<NW>{w, pv};
        __syncwarp();
        const uint32_t c = __popc(bal);
        for (uint32_t j = 0; j < c; ++j) {
            const Packed<NW> x = pack[j];
            body(x.w, x.m);
        }
        __syncwarp();
    }
}

// Light vertex: the warp's lanes hold its (at most 32) block indices.
template <int NW, typename Pre, typename Body>
__device__ __forceinline__ void ms_walk_light(const DevGraph &g, uint4 rec, Pre &&pre, Body &&body) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB);
    const uint32_t blk = lane < nb ? ms_block(g, rec.x, lane) : GV_NIL;
    for (uint32_t k = 0; k < nb; ++k) {
        const uint32_t b = __shfl_sync(GV_FULL_MASK, blk, k);
        ms_block_entries<NW>(g, b, min(g.B, fill - (k << g.logB)), pre, body);
    }
}

// Heavy vertex: the CTA fills a shared block table window by window; warps
// take blocks w, w + MS_WARPS, ...
template <int NW, typename Pre, typename Body>
__device__ __forceinline__ void ms_walk_heavy(const DevGraph &g, uint4 rec, uint32_t *tab, Pre &&pre, Body &&body) {
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB);
    for (uint32_t k0 = 0; k0 < nb; k0 += MS_TAB) {
        const uint32_t cnt = min(MS_TAB, nb - k0);
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) tab[i] = ms_block(g, rec.x, k0 + i);
        __syncthreads();
        for (uint32_t i = warp; i < cnt; i += MS_WARPS) {
            const uint32_t k = k0 + i;
            ms_block_entries<NW>(g, tab[i], min(g.B, fill - (k << g.logB)), pre, body);
        }
    }
}

// Places the pass's sources: slot s (< 32 NW) holds src[s], GV_NIL for none.
template <int NW>
__global__ void k_ms_init(MsBufs<NW> b, const uint32_t *__restrict__ src) {
    using M = typename MaskOf<NW>::type;
    const uint32_t s = threadIdx.x;
    if (s >= 32u * NW) return;
    const uint32_t v = src[s];
    if (v == GV_NIL) return;
    atomicOr(&b.masks[v], (M)1 << s);
    atomicOr(&b.vis[v], (M)1 << s);
    b.row[(size_t)v * 32 * NW + s] = 1ull;
}

// Vertices of level L into the light / heavy lists (warp-aggregated appends).
template <int NW>
__global__ void k_ms_split(DevGraph g, MsBufs<NW> b, const typename MaskOf<NW>::type *__restrict__ mask) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t n = b.n;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint32_t v = base + threadIdx.x;
        bool on = false, heavy = false;
        uint32_t fill = 0;
        if (v < n && mask[v]) {
            on = true;
            fill = g.vtx[v].y;
            heavy = fill > MS_HEAVY_FILL;
        }
        const uint32_t bl = __ballot_sync(GV_FULL_MASK, on && !heavy), bh = __ballot_sync(GV_FULL_MASK, on && heavy);
        const unsigned long long es = warp_sum((unsigned long long)fill);
        uint32_t ol = 0, oh = 0;
        if (lane == 0) {
            if (bl) ol = atomicAdd(&b.cnt[0], __popc(bl));
            if (bh) oh = atomicAdd(&b.cnt[1], __popc(bh));
            if (es) atomicAdd(&b.esum[0], es);
        }
        ol = __shfl_sync(GV_FULL_MASK, ol, 0);
        oh = __shfl_sync(GV_FULL_MASK, oh, 0);
        const uint32_t below = (1u << lane) - 1u;
        if (on && !heavy) b.light[ol + __popc(bl & below)] = v;
        if (on && heavy) b.heavy[oh + __popc(bh & below)] = v;
    }
}

// Pull levels choose themselves on the device: the level's own entries
// (esum[0], what a push level reads) against the entries of the vertices some
// source has not reached (esum[1], what a pull level reads).
template <int NW>
__device__ __forceinline__ bool ms_pull_level(const MsBufs<NW> &b) {
    return b.alpha && (unsigned long long)b.alpha * b.esum[0] > b.esum[1];
}

// Candidates of a pull level: vertices with entries that some source of the
// pass has not reached (warp-aggregated appends); nothing on push levels.
template <int NW>
__global__ void k_ms_cand(DevGraph g, MsBufs<NW> b) {
    using M = typename MaskOf<NW>::type;
    if (!ms_pull_level(b)) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t n = b.n;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t v = base + threadIdx.x;
        bool on = false, heavy = false;
        uint32_t fill = 0;
        if (v < n) {
            const M need = b.full & ~b.vis[v];
            if (need) {
                fill = g.vtx[v].y;
                on = fill > 0;
                heavy = fill > MS_HEAVY_FILL;
            }
        }
        const uint32_t bl = __ballot_sync(GV_FULL_MASK, on && !heavy), bh = __ballot_sync(GV_FULL_MASK, on && heavy);
        uint32_t ol = 0, oh = 0;
        if (lane == 0) {
            if (bl) ol = atomicAdd(&b.cnt[2], __popc(bl));
            if (bh) oh = atomicAdd(&b.cnt[3], __popc(bh));
        }
        ol = __shfl_sync(GV_FULL_MASK, ol, 0);
        oh = __shfl_sync(GV_FULL_MASK, oh, 0);
        const uint32_t below = (1u << lane) - 1u;
        if (on && !heavy) b.clight[ol + __popc(bl & below)] = v;
        if (on && heavy) b.cheavy[oh + __popc(bh & below)] = v;
    }
}

// Entries of every vertex, the pull levels' starting count of entries of
// vertices some source has not reached.
__global__ void k_ms_total_fill(DevGraph g, unsigned long long *__restrict__ out) {
    unsigned long long t = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < g.n; v += gridDim.x * blockDim.x) t += g.vtx[v].y;
    t = warp_sum(t);
    if ((threadIdx.x & 31u) == 0 && t) atomicAdd(out, t);
}

template <typename M>
__device__ __forceinline__ M warp_or_mask(M x) {
    if (sizeof(M) == 8) {
        const uint32_t lo = __reduce_or_sync(GV_FULL_MASK, (uint32_t)x);
        const uint32_t hi = __reduce_or_sync(GV_FULL_MASK, (uint32_t)((unsigned long long)x >> 32));
        return (M)(((unsigned long long)hi << 32) | lo);
    }
    return (M)__reduce_or_sync(GV_FULL_MASK, (uint32_t)x);
}

// Pull over one block of candidate w's entries: the neighbours u at level L
// for some source that has not reached w (F = mask[u] & need) are packed,
// then each lane adds sigma_s(u) of its sources for them (exact uint64 sums)
// and ORs F into the sources that reach w at level L + 1.
template <int NW>
__device__ __forceinline__ void ms_pull_block(const DevGraph &g, const MsBufs<NW> &b,
                                              const typename MaskOf<NW>::type *__restrict__ mask, uint32_t blk,
                                              uint32_t slots, typename MaskOf<NW>::type need,
                                              unsigned long long (&acc)[NW], typename MaskOf<NW>::type &reach) {
    using M = typename MaskOf<NW>::type;
    __shared__ Packed<NW> pack_all[MS_WARPS][32];
    const uint32_t lane = threadIdx.x & 31u;
    Packed<NW> *pack = pack_all[threadIdx.x >> 5];
    const uint32_t *bp = g.pool + ((size_t)blk << g.logB);
    const unsigned long long *row = b.row;
    for (uint32_t e0 = 0; e0 < slots; e0 += 32) {
        const uint32_t e = e0 + lane;
        uint32_t u = 0;
        M f = 0;
        if (e < slots) {
            u = bp[e];
            if (u != GV_TOMB) f = mask[u] & need;
            else u = 0;
        }
        reach |= f;
        const uint32_t bal = __ballot_sync(GV_FULL_MASK, f != 0);
        if (!bal) continue;  // warp-uniform
        if (f) pack[__popc(bal & ((1u << lane) - 1u))] = Packed<NW>{u, f};
        __syncwarp();
        const uint32_t c = __popc(bal);
        constexpr int GB = NW == 1 ? 8 : 4;
        for (uint32_t j0 = 0; j0 < c; j0 += GB) {
            Packed<NW> x[GB];
#pragma unroll
            for (int t = 0; t < GB; ++t) x[t] = (j0 + t < c) ? pack[j0 + t] : Packed<NW>{0u, (M)0};
            unsigned long long v[NW][GB];
#pragma unroll
            for (int k = 0; k < NW; ++k)
#pragma unroll
                for (int t = 0; t < GB; ++t)
                    v[k][t] = has_src(x[t].m, lane, k) ? __ldg(row + (size_t)x[t].w * 32 * NW + lane + 32 * k) : 0ull;
#pragma unroll
            for (int k = 0; k < NW; ++k)
#pragma unroll
                for (int t = 0; t < GB; ++t) acc[k] += v[k][t];
        }
        __syncwarp();
    }
}

// Writes w's sigma for the sources that reach it at this level, and nxt[w].
template <int NW>
__device__ __forceinline__ void ms_pull_finish(const MsBufs<NW> &b, uint32_t w, typename MaskOf<NW>::type reach,
                                               const unsigned long long (&acc)[NW]) {
    const uint32_t lane = threadIdx.x & 31u;
    if (!reach) return;  // warp-uniform
#pragma unroll
    for (int k = 0; k < NW; ++k)
        if (has_src(reach, lane, k)) b.row[(size_t)w * 32 * NW + lane + 32 * k] = acc[k];
    if (lane == 0) b.nxt[w] = reach;
}

template <int NW>
__device__ __forceinline__ void ms_pull_light(const DevGraph &g, const MsBufs<NW> &b,
                                              const typename MaskOf<NW>::type *__restrict__ mask, uint32_t vb,
                                              uint32_t vg) {
    using M = typename MaskOf<NW>::type;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nl = b.cnt[2];
    for (uint32_t i = vb * MS_WARPS + (threadIdx.x >> 5); i < nl; i += vg * MS_WARPS) {
        const uint32_t w = b.clight[i];
        const M need = b.full & ~b.vis[w];
        unsigned long long acc[NW];
#pragma unroll
        for (int k = 0; k < NW; ++k) acc[k] = 0ull;
        M reach = 0;
        const uint4 rec = g.vtx[w];
        const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB);
        const uint32_t blk = lane < nb ? ms_block(g, rec.x, lane) : GV_NIL;
        for (uint32_t k = 0; k < nb; ++k) {
            const uint32_t bk = __shfl_sync(GV_FULL_MASK, blk, k);
            ms_pull_block<NW>(g, b, mask, bk, min(g.B, fill - (k << g.logB)), need, acc, reach);
        }
        ms_pull_finish<NW>(b, w, warp_or_mask(reach), acc);
    }
}

template <int NW>
__device__ __forceinline__ void ms_pull_heavy(const DevGraph &g, const MsBufs<NW> &b,
                                              const typename MaskOf<NW>::type *__restrict__ mask, uint32_t vb,
                                              uint32_t vg) {
    using M = typename MaskOf<NW>::type;
    __shared__ uint32_t tab[MS_TAB];
    __shared__ unsigned long long red[MS_WARPS][NW][32];
    __shared__ M rred[MS_WARPS];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t nh = b.cnt[3];
    for (uint32_t i = vb; i < nh; i += vg) {
        const uint32_t w = b.cheavy[i];
        const M need = b.full & ~b.vis[w];
        unsigned long long acc[NW];
#pragma unroll
        for (int k = 0; k < NW; ++k) acc[k] = 0ull;
        M reach = 0;
        const uint4 rec = g.vtx[w];
        const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB);
        for (uint32_t k0 = 0; k0 < nb; k0 += MS_TAB) {
            const uint32_t cnt = min(MS_TAB, nb - k0);
            __syncthreads();
            for (uint32_t t = threadIdx.x; t < cnt; t += blockDim.x) tab[t] = ms_block(g, rec.x, k0 + t);
            __syncthreads();
            for (uint32_t t = warp; t < cnt; t += MS_WARPS)
                ms_pull_block<NW>(g, b, mask, tab[t], min(g.B, fill - ((k0 + t) << g.logB)), need, acc, reach);
        }
#pragma unroll
        for (int k = 0; k < NW; ++k) red[warp][k][lane] = acc[k];
        reach = warp_or_mask(reach);
        if (lane == 0) rred[warp] = reach;
        __syncthreads();
        if (warp == 0) {
            unsigned long long tot[NW];
            M r = 0;
#pragma unroll
            for (int k = 0; k < NW; ++k) {
                tot[k] = 0ull;
                for (int x = 0; x < MS_WARPS; ++x) tot[k] += red[x][k][lane];
            }
            for (int x = 0; x < MS_WARPS; ++x) r |= rred[x];
            ms_pull_finish<NW>(b, w, r, tot);
        }
        __syncthreads();
    }
}

template <int NW>
struct FwdBody {
    using M = typename MaskOf<NW>::type;
    MsBufs<NW> b;
    M F;
    unsigned long long sig[NW];
    __device__ __forceinline__ void load(uint32_t u) {
        const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
        for (int k = 0; k < NW; ++k) sig[k] = has_src(F, lane, k) ? b.row[(size_t)u * 32 * NW + lane + 32 * k] : 0ull;
    }
    // sources that reach w first through this level
    __device__ __forceinline__ M operator()(uint32_t w) const { return F & ~b.vis[w]; }
    __device__ __forceinline__ void visit(uint32_t w, M want) const {
        const uint32_t lane = threadIdx.x & 31u;
        if (lane == 0) atomicOr(&b.nxt[w], want);
#pragma unroll
        for (int k = 0; k < NW; ++k)
            if (has_src(want, lane, k)) atomicAdd(&b.row[(size_t)w * 32 * NW + lane + 32 * k], sig[k]);
    }
};

template <int NW>
__device__ __forceinline__ void ms_fwd_light(const DevGraph &g, const MsBufs<NW> &b,
                                             const typename MaskOf<NW>::type *__restrict__ mask, uint32_t vb,
                                             uint32_t vg) {
    using M = typename MaskOf<NW>::type;
    const uint32_t nl = b.cnt[0];
    for (uint32_t i = vb * MS_WARPS + (threadIdx.x >> 5); i < nl; i += vg * MS_WARPS) {
        const uint32_t u = b.light[i];
        FwdBody<NW> f{b, mask[u], {}};
        f.load(u);
        ms_walk_light<NW>(g, g.vtx[u], f, [&](uint32_t w, M want) { f.visit(w, want); });
    }
}

template <int NW>
__device__ __forceinline__ void ms_fwd_heavy(const DevGraph &g, const MsBufs<NW> &b,
                                             const typename MaskOf<NW>::type *__restrict__ mask, uint32_t vb,
                                             uint32_t vg) {
    using M = typename MaskOf<NW>::type;
    __shared__ uint32_t tab[MS_TAB];
    const uint32_t nh = b.cnt[1];
    for (uint32_t i = vb; i < nh; i += vg) {
        const uint32_t u = b.heavy[i];
        FwdBody<NW> f{b, mask[u], {}};
        f.load(u);
        ms_walk_heavy<NW>(g, g.vtx[u], tab, f, [&](uint32_t w, M want) { f.visit(w, want); });
    }
}

// One launch per level and direction: CTA i runs the heavy-vertex part when
// i % 5 == 4, the light part otherwise, so hub CTAs and light warps share
// every wave.
__device__ __forceinline__ bool ms_split_cta(uint32_t &vb, uint32_t &vg_light, uint32_t &vg_heavy) {
    const uint32_t bi = blockIdx.x;
    vg_heavy = gridDim.x / 5;
    vg_light = gridDim.x - vg_heavy;
    if (bi % 5 == 4) {
        vb = bi / 5;
        return true;
    }
    vb = (bi / 5) * 4 + bi % 5;
    return false;
}

template <int NW>
__global__ void __launch_bounds__(MS_THREADS) k_ms_fwd(DevGraph g, MsBufs<NW> b,
                                                       const typename MaskOf<NW>::type *__restrict__ mask) {
    if (ms_pull_level(b)) return;  // k_ms_pull does this level
    uint32_t vb, vgl, vgh;
    if (ms_split_cta(vb, vgl, vgh)) ms_fwd_heavy<NW>(g, b, mask, vb, vgh);
    else ms_fwd_light<NW>(g, b, mask, vb, vgl);
}

// Pull (bottom-up) forward level: each candidate gathers the path counts of
// its neighbours at level L; no atomics, one write of its row.
// Five resident CTAs (48 registers, a few spilled) for the pull and the
// dependency pass: at R-MAT scale 25, 64 sources, 290 -> 268 ms (two
// requests in one pass 317 -> 302 ms) against four CTAs at 56-64 registers;
// six (40 registers) were slower.
template <int NW>
__global__ void __launch_bounds__(MS_THREADS, 5) k_ms_pull(DevGraph g, MsBufs<NW> b,
                                                           const typename MaskOf<NW>::type *__restrict__ mask) {
    if (!ms_pull_level(b)) return;  // k_ms_fwd does this level
    uint32_t vb, vgl, vgh;
    if (ms_split_cta(vb, vgl, vgh)) ms_pull_heavy<NW>(g, b, mask, vb, vgh);
    else ms_pull_light<NW>(g, b, mask, vb, vgl);
}

// Closes level L: masks[L+1] = nxt, vis |= nxt, flags[L+1] = any.
template <int NW>
__global__ void k_ms_close(DevGraph g, MsBufs<NW> b, typename MaskOf<NW>::type *__restrict__ next_mask,
                           uint32_t *flag) {
    using M = typename MaskOf<NW>::type;
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    bool mine = false;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < b.n; v += gridDim.x * blockDim.x) {
        const M x = b.nxt[v];
        next_mask[v] = x;
        if (x) {
            const M old = b.vis[v];
            b.vis[v] = old | x;
            b.nxt[v] = 0;
            mine = true;
            // every source has reached v: its entries leave the pull levels' count
            if (b.alpha && (old | x) == b.full && old != b.full)
                atomicAdd(&b.esum[1], 0ull - (unsigned long long)g.vtx[v].y);
        }
    }
    if (mine) any = 1;
    __syncthreads();
    if (threadIdx.x == 0 && any) atomicOr(flag, 1u);
}

// Backward sum over one block's entries for the sources in A: the entries one
// level deeper for some of them are packed, then every lane gathers coef of
// its sources for eight (one word) or four (two words) entries at a time,
// eight predicated gathers in flight per lane, and adds them in entry order.
template <int NW>
__device__ __forceinline__ void ms_bwd_block(const DevGraph &g, const MsBufs<NW> &b,
                                             const typename MaskOf<NW>::type *__restrict__ deeper, uint32_t blk,
                                             uint32_t slots, typename MaskOf<NW>::type A, double (&acc)[NW]) {
    using M = typename MaskOf<NW>::type;
    __shared__ Packed<NW> pack_all[MS_WARPS][32];
    const uint32_t lane = threadIdx.x & 31u;
    Packed<NW> *pack = pack_all[threadIdx.x >> 5];
    const uint32_t *bp = g.pool + ((size_t)blk << g.logB);
    const unsigned long long *row = b.row;
    for (uint32_t e0 = 0; e0 < slots; e0 += 32) {
        const uint32_t e = e0 + lane;
        uint32_t w = 0;
        M mw = 0;
        if (e < slots) {
            w = bp[e];
            if (w != GV_TOMB) mw = deeper[w] & A;
            else w = 0;
        }
        const uint32_t bal = __ballot_sync(GV_FULL_MASK, mw != 0);
        if (!bal) continue;  // warp-uniform
        if (mw) pack[__popc(bal & ((1u << lane) - 1u))] = Packed<NW>{w, mw};
        __syncwarp();
        const uint32_t c = __popc(bal);
        constexpr int GB = NW == 1 ? 8 : 4;  // entries per batch: 8 gathers in flight per lane either way
        for (uint32_t j0 = 0; j0 < c; j0 += GB) {
            Packed<NW> x[GB];
#pragma unroll
            for (int t = 0; t < GB; ++t) x[t] = (j0 + t < c) ? pack[j0 + t] : Packed<NW>{0u, (M)0};
            unsigned long long v[NW][GB];
#pragma unroll
            for (int k = 0; k < NW; ++k)
#pragma unroll
                for (int t = 0; t < GB; ++t)
                    v[k][t] = has_src(x[t].m, lane, k) ? __ldg(row + (size_t)x[t].w * 32 * NW + lane + 32 * k) : 0ull;
#pragma unroll
            for (int k = 0; k < NW; ++k)
#pragma unroll
                for (int t = 0; t < GB; ++t) acc[k] += as_f64(v[k][t]);
        }
        __syncwarp();
    }
}

template <int NW>
__device__ __forceinline__ void ms_load_sig(const MsBufs<NW> &b, uint32_t v, typename MaskOf<NW>::type A,
                                            unsigned long long (&sig)[NW]) {
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (int k = 0; k < NW; ++k) sig[k] = has_src(A, lane, k) ? b.row[(size_t)v * 32 * NW + lane + 32 * k] : 0ull;
}

// Finishes (v, sources in A): delta = sigma * acc, coef replaces sigma, and
// each half with a source here adds the sum of its deltas over the lanes into
// its output row (lane 0, halves in order).
template <int NW>
__device__ __forceinline__ void ms_finish(const MsBufs<NW> &b, uint32_t v, typename MaskOf<NW>::type A,
                                          const unsigned long long (&sig)[NW], const double (&acc)[NW]) {
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (int k = 0; k < NW; ++k) {
        if (NW > 1 && !(uint32_t)(A >> (32u * (uint32_t)k))) continue;  // warp-uniform: no source of this half here
        double delta = 0.0;
        if (has_src(A, lane, k)) {
            const double sv = (double)sig[k];
            delta = sv * acc[k];
            b.row[(size_t)v * 32 * NW + lane + 32 * k] = as_u64((1.0 + delta) / sv);
        }
        delta = warp_sum(delta);
        if (lane == 0) b.bc[(size_t)b.out[k] * b.n + v] += delta;
    }
}

template <int NW>
__device__ __forceinline__ void ms_bwd_light(const DevGraph &g, const MsBufs<NW> &b,
                                             const typename MaskOf<NW>::type *__restrict__ mask,
                                             const typename MaskOf<NW>::type *__restrict__ deeper, uint32_t vb,
                                             uint32_t vg) {
    using M = typename MaskOf<NW>::type;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nl = b.cnt[0];
    const uint32_t stride = vg * MS_WARPS;
    // A two-stage prefetch: while a vertex runs, the id of the vertex after
    // next and the source mask and record of the next one are in flight, and
    // the next one's sigma row is loaded before this one finishes, so a
    // vertex starts with its header at hand.  (Rows read here belong to
    // vertices of this level, which only their own warp writes.)
    uint32_t i = vb * MS_WARPS + (threadIdx.x >> 5);
    uint32_t v1 = i < nl ? b.light[i] : 0u;
    uint32_t v2 = i + stride < nl ? b.light[i + stride] : 0u;
    M A1 = i < nl ? mask[v1] : (M)0;
    uint2 rec1 = make_uint2(0u, 0u);
    if (i < nl) {
        const uint4 r = g.vtx[v1];
        rec1 = make_uint2(r.x, r.y);
    }
    unsigned long long sig1[NW];
    ms_load_sig<NW>(b, v1, A1, sig1);
    for (; i < nl; i += stride) {
        const bool has2 = i + stride < nl;
        const uint32_t v3 = i + 2 * stride < nl ? b.light[i + 2 * stride] : 0u;
        const M A2 = has2 ? mask[v2] : (M)0;
        uint2 rec2 = make_uint2(0u, 0u);
        if (has2) {
            const uint4 r = g.vtx[v2];
            rec2 = make_uint2(r.x, r.y);
        }
        double acc[NW];
#pragma unroll
        for (int k = 0; k < NW; ++k) acc[k] = 0.0;
        const uint32_t fill = rec1.y, nb = blocks_for(fill, g.logB);
        const uint32_t blk = lane < nb ? ms_block(g, rec1.x, lane) : GV_NIL;
        for (uint32_t k = 0; k < nb; ++k) {
            const uint32_t bk = __shfl_sync(GV_FULL_MASK, blk, k);
            ms_bwd_block<NW>(g, b, deeper, bk, min(g.B, fill - (k << g.logB)), A1, acc);
        }
        unsigned long long sig2[NW];
        ms_load_sig<NW>(b, v2, A2, sig2);
        ms_finish<NW>(b, v1, A1, sig1, acc);
        v1 = v2;
        v2 = v3;
        A1 = A2;
        rec1 = rec2;
#pragma unroll
        for (int k = 0; k < NW; ++k) sig1[k] = sig2[k];
    }
}

template <int NW>
__device__ __forceinline__ void ms_bwd_heavy(const DevGraph &g, const MsBufs<NW> &b,
                                             const typename MaskOf<NW>::type *__restrict__ mask,
                                             const typename MaskOf<NW>::type *__restrict__ deeper, uint32_t vb,
                                             uint32_t vg) {
    __shared__ uint32_t tab[MS_TAB];
    __shared__ double red[MS_WARPS][NW][32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t nh = b.cnt[1];
    for (uint32_t i = vb; i < nh; i += vg) {
        const uint32_t v = b.heavy[i];
        const typename MaskOf<NW>::type A = mask[v];
        unsigned long long sig[NW];
        ms_load_sig<NW>(b, v, A, sig);
        double acc[NW];
#pragma unroll
        for (int k = 0; k < NW; ++k) acc[k] = 0.0;
        const uint4 rec = g.vtx[v];
        const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB);
        for (uint32_t k0 = 0; k0 < nb; k0 += MS_TAB) {
            const uint32_t cnt = min(MS_TAB, nb - k0);
            __syncthreads();
            for (uint32_t t = threadIdx.x; t < cnt; t += blockDim.x) tab[t] = ms_block(g, rec.x, k0 + t);
            __syncthreads();
            for (uint32_t t = warp; t < cnt; t += MS_WARPS)
                ms_bwd_block<NW>(g, b, deeper, tab[t], min(g.B, fill - ((k0 + t) << g.logB)), A, acc);
        }
#pragma unroll
        for (int k = 0; k < NW; ++k) red[warp][k][lane] = acc[k];
        __syncthreads();
        if (warp == 0) {
            double tot[NW];
#pragma unroll
            for (int k = 0; k < NW; ++k) {
                tot[k] = 0.0;
                for (int w = 0; w < MS_WARPS; ++w) tot[k] += red[w][k][lane];
            }
            ms_finish<NW>(b, v, A, sig, tot);
        }
        __syncthreads();
    }
}

template <int NW>
__global__ void __launch_bounds__(MS_THREADS, 5) k_ms_bwd(DevGraph g, MsBufs<NW> b,
                                                       const typename MaskOf<NW>::type *__restrict__ mask,
                                                       const typename MaskOf<NW>::type *__restrict__ deeper) {
    uint32_t vb, vgl, vgh;
    if (ms_split_cta(vb, vgl, vgh)) ms_bwd_heavy<NW>(g, b, mask, deeper, vb, vgh);
    else ms_bwd_light<NW>(g, b, mask, deeper, vb, vgl);
}

__global__ void k_ms_to_f32(const double *__restrict__ x, float *__restrict__ y, uint32_t n) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) y[v] = (float)x[v];
}

// dist / sigma of slot 0 after a one-source forward pass.
__global__ void k_ms_extract(MsBufs<1> b, uint32_t depth, int32_t *__restrict__ dist,
                             unsigned long long *__restrict__ sigma) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < b.n; v += gridDim.x * blockDim.x) {
        int32_t d = -1;
        for (uint32_t L = 0; L <= depth; ++L)
            if (b.masks[(size_t)L * b.n + v] & 1u) {
                d = (int32_t)L;
                break;
            }
        dist[v] = d;
        sigma[v] = b.row[(size_t)v * 32];
    }
}

// Level masks live in auxiliary slot 6 and grow (keeping the first
// keep_levels levels) when a BFS runs deeper than the levels allocated.
template <int NW>
gv_status masks_reserve(gv_graph *g, MsBufs<NW> &b, uint32_t levels, uint32_t keep_levels, cudaStream_t s) {
    using M = typename MaskOf<NW>::type;
    const size_t level_bytes = (size_t)b.n * sizeof(M);
    const uint32_t cap = (uint32_t)std::min<size_t>(g->aux[6] ? g->aux_bytes[6] / level_bytes : 0, MS_MAX_LEVELS);
    b.masks = (M *)g->aux[6];
    if (levels <= cap) return GV_OK;
    uint32_t want = std::max<uint32_t>(32, cap);
    while (want < levels) want *= 2;
    if (want > MS_MAX_LEVELS) {
        set_error("BFS deeper than the level table");
        return GV_ERR_UNSUPPORTED;
    }
    const size_t bytes = (size_t)want * level_bytes;
    void *nb = nullptr;
    if (cudaMalloc(&nb, bytes) != cudaSuccess) {
        cudaGetLastError();
        set_error("level masks allocation of " + std::to_string(bytes) + " B failed");
        return GV_ERR_NOMEM;
    }
    if (keep_levels && g->aux[6]) {
        cudaError_t e = cudaMemcpyAsync(nb, g->aux[6], (size_t)keep_levels * level_bytes, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            cudaFree(nb);
            return cuda_status(e, "level masks copy");
        }
    }
    if (g->aux[6]) cudaFree(g->aux[6]);
    g->aux[6] = nb;
    g->aux_bytes[6] = bytes;
    b.masks = (M *)nb;
    return GV_OK;
}

// Forward pass for the sources placed in dsrc (32 NW slots); returns the
// deepest non-empty level.
template <int NW>
gv_status ms_forward(gv_graph *g, MsBufs<NW> &b, const uint32_t *dsrc, uint32_t *h_flags, uint32_t *depth_out,
                     cudaStream_t s) {
    using M = typename MaskOf<NW>::type;
    const DevGraph d = g->d;
    const uint32_t n = b.n;
    gv_status st = masks_reserve<NW>(g, b, 8, 0, s);
    if (st != GV_OK) return st;
    cudaMemsetAsync(b.row, 0, (size_t)n * 256 * NW, s);
    cudaMemsetAsync(b.vis, 0, (size_t)n * sizeof(M), s);
    cudaMemsetAsync(b.nxt, 0, (size_t)n * sizeof(M), s);
    cudaMemsetAsync(b.masks, 0, (size_t)n * sizeof(M), s);
    GV_LAUNCH(k_ms_init<NW>, 1, 32 * NW, 0, s, b, dsrc);
    if (b.alpha) {
        cudaMemsetAsync(b.esum + 1, 0, 8, s);
        GV_LAUNCH(k_ms_total_fill, grid_for(n, 256), 256, 0, s, d, b.esum + 1);
    }
    const uint32_t chunk = 4;
    uint32_t L = 0;
    for (;;) {
        st = masks_reserve<NW>(g, b, L + chunk + 2, L + 1, s);
        if (st != GV_OK) return st;
        cudaMemsetAsync(b.flags + L + 1, 0, chunk * 4, s);
        for (uint32_t i = 0; i < chunk; ++i, ++L) {
            const M *mask = b.masks + (size_t)L * n;
            ProfScope ps(PROF_BFS_LEVEL, s);
            cudaMemsetAsync(b.cnt, 0, 16, s);
            cudaMemsetAsync(b.esum, 0, 8, s);
            GV_LAUNCH(k_ms_split<NW>, grid_for(n, 256), 256, 0, s, d, b, mask);
            static_assert(MS_LIGHT_GRID == 4 * MS_HEAVY_GRID, "the fused launch interleaves 4 light CTAs per heavy one");
            if (b.alpha) {
                GV_LAUNCH(k_ms_cand<NW>, grid_for(n, 256), 256, 0, s, d, b);
                GV_LAUNCH(k_ms_pull<NW>, MS_LIGHT_GRID + MS_HEAVY_GRID, MS_THREADS, 0, s, d, b, mask);
            }
            GV_LAUNCH(k_ms_fwd<NW>, MS_LIGHT_GRID + MS_HEAVY_GRID, MS_THREADS, 0, s, d, b, mask);
            GV_LAUNCH(k_ms_close<NW>, grid_for(n, 256), 256, 0, s, d, b, b.masks + (size_t)(L + 1) * n, b.flags + L + 1);
        }
        cudaError_t e = cudaMemcpyAsync(h_flags, b.flags + L - chunk + 1, chunk * 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e, "bfs levels");
        for (uint32_t i = 0; i < chunk; ++i)
            if (!h_flags[i]) {
                *depth_out = L - chunk + i;  // level L - chunk + 1 + i is empty
                return GV_OK;
            }
    }
}

template <int NW>
gv_status ms_backward(gv_graph *g, MsBufs<NW> &b, uint32_t depth, cudaStream_t s) {
    using M = typename MaskOf<NW>::type;
    const DevGraph d = g->d;
    const uint32_t n = b.n;
    for (uint32_t L = depth; L >= 1; --L) {
        const M *mask = b.masks + (size_t)L * n;
        const M *deeper = b.masks + (size_t)(L + 1) * n;
        ProfScope ps(PROF_BC_DEP, s);
        cudaMemsetAsync(b.cnt, 0, 8, s);
        GV_LAUNCH(k_ms_split<NW>, grid_for(n, 256), 256, 0, s, d, b, mask);
        GV_LAUNCH(k_ms_bwd<NW>, MS_LIGHT_GRID + MS_HEAVY_GRID, MS_THREADS, 0, s, d, b, mask, deeper);
    }
    return cuda_status(cudaGetLastError(), "bc dependencies");
}

size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

// Carves the buffers of passes up to nw mask words wide and `outputs` score
// rows from the analytics scratch.
gv_status ms_setup(gv_graph *g, uint32_t nw, uint32_t outputs, MsArena &a) {
    const uint32_t n = g->d.n;
    a.n = n;
    const size_t o_row = 0, o_vis = o_row + al256((size_t)n * 256 * nw), o_nxt = o_vis + al256((size_t)n * 4 * nw);
    const size_t o_light = o_nxt + al256((size_t)n * 4 * nw), o_heavy = o_light + al256((size_t)n * 4);
    const size_t o_clight = o_heavy + al256((size_t)n * 4), o_cheavy = o_clight + al256((size_t)n * 4);
    const size_t o_cnt = o_cheavy + al256((size_t)n * 4), o_flags = o_cnt + 256;
    const size_t o_src = o_flags + al256((size_t)MS_MAX_LEVELS * 4 + 4), o_bc = o_src + 256;
    const size_t bytes = o_bc + al256((size_t)n * 8 * outputs);
    char *p = (char *)analytics_scratch(g, bytes);
    if (!p) return GV_ERR_NOMEM;
    a.row = (unsigned long long *)(p + o_row);
    a.vis = p + o_vis;
    a.nxt = p + o_nxt;
    a.light = (uint32_t *)(p + o_light);
    a.heavy = (uint32_t *)(p + o_heavy);
    a.cnt = (uint32_t *)(p + o_cnt);
    a.esum = (unsigned long long *)(p + o_cnt + 64);
    a.clight = (uint32_t *)(p + o_clight);
    a.cheavy = (uint32_t *)(p + o_cheavy);
    a.flags = (uint32_t *)(p + o_flags);
    a.dsrc = (uint32_t *)(p + o_src);
    a.bc = (double *)(p + o_bc);
    if (!g->host_pinned) {
        if (cudaMallocHost(&g->host_pinned, 256) != cudaSuccess) {
            cudaGetLastError();
            set_error("pinned host word allocation failed");
            return GV_ERR_NOMEM;
        }
        g->host_pinned_bytes = 256;
    }
    a.hflags = (uint32_t *)g->host_pinned;
    return GV_OK;
}

// Pull levels: a forward level of a 64-source pass pulls when MS_PULL_ALPHA
// times its own entries exceed the entries of the vertices some source has
// not reached; GV_BC_PULL=<alpha> overrides it (0: push every level).  On
// R-MAT scale 22 this takes the forward of 64 sources from 21.1 to 15.2 ms;
// 32-source passes push every level (pull levels made them slower: their
// push adds touch half the row bytes).
constexpr uint32_t MS_PULL_ALPHA = 2;
template <int NW>
uint32_t ms_pull_alpha() {
    const char *env = std::getenv("GV_BC_PULL");
    if (env) return (uint32_t)std::strtoul(env, nullptr, 10);
    return NW == 2 ? MS_PULL_ALPHA : 0;
}

// A whole pass (forward, then dependencies) over 32 NW source slots.
template <int NW>
gv_status ms_pass(gv_graph *g, const MsArena &a, const uint32_t *slots, uint32_t out0, uint32_t out1,
                  cudaStream_t s) {
    using M = typename MaskOf<NW>::type;
    MsBufs<NW> b = a.bufs<NW>(g);
    b.out[0] = out0;
    b.out[1] = out1;
    for (uint32_t i = 0; i < 32u * NW; ++i)
        if (slots[i] != GV_NIL) b.full |= (M)1 << i;
    b.alpha = ms_pull_alpha<NW>();
    cudaError_t e = cudaMemcpyAsync(a.dsrc, slots, 32 * NW * 4, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_status(e, "bc sources");
    uint32_t depth = 0;
    gv_status st = ms_forward<NW>(g, b, a.dsrc, a.hflags, &depth, s);
    if (st != GV_OK) return st;
    return ms_backward<NW>(g, b, depth, s);
}

struct Group {
    uint32_t req;
    uint64_t first;
    uint32_t count;
};

}  // namespace

// Scores of nreq requests: request r holds hs[off[r] .. off[r+1]) (empty:
// every vertex) and adds into score row r.  Requests are cut into groups of
// up to 32 sources; consecutive groups are paired into 64-source passes (the
// last group alone runs a 32-source pass), so two requests of up to 32
// sources share every adjacency read of their BFS.
gv_status bc_requests(gv_graph *g, std::vector<uint32_t> &hs, std::vector<uint64_t> &off, uint32_t nreq,
                      float *out, int mem, cudaStream_t s) {
    const uint32_t n = g->d.n;
    for (uint32_t v : hs)
        if (v >= n) { set_error("BC source out of range"); return GV_ERR_INVALID; }
    std::vector<Group> groups;
    std::vector<uint32_t> all;
    for (uint32_t r = 0; r < nreq; ++r) {
        uint64_t lo = off[r], hi = off[r + 1];
        if (lo == hi) {  // every vertex
            if (all.empty()) {
                all.resize(n);
                for (uint32_t i = 0; i < n; ++i) all[i] = i;
            }
            lo = hs.size();
            hs.insert(hs.end(), all.begin(), all.end());
            hi = hs.size();
        }
        for (uint64_t i = lo; i < hi; i += 32) groups.push_back({r, i, (uint32_t)std::min<uint64_t>(32, hi - i)});
    }
    MsArena a;
    gv_status st = ms_setup(g, groups.size() > 1 ? 2 : 1, nreq, a);
    if (st != GV_OK) return st;
    cudaMemsetAsync(a.bc, 0, (size_t)n * 8 * nreq, s);
    std::vector<uint32_t> slots(64);
    for (size_t i = 0; i < groups.size() && st == GV_OK; i += 2) {
        std::fill(slots.begin(), slots.end(), GV_NIL);
        const Group &x = groups[i];
        std::copy(hs.begin() + x.first, hs.begin() + x.first + x.count, slots.begin());
        if (i + 1 < groups.size()) {
            const Group &y = groups[i + 1];
            std::copy(hs.begin() + y.first, hs.begin() + y.first + y.count, slots.begin() + 32);
            st = ms_pass<2>(g, a, slots.data(), x.req, y.req, s);
        } else {
            st = ms_pass<1>(g, a, slots.data(), x.req, x.req, s);
        }
    }
    if (st != GV_OK) return st;
    float *tmp = (float *)a.row;  // the sigma rows are free once every pass is done
    for (uint32_t r = 0; r < nreq; ++r) {
        float *dst = out + (size_t)r * n;
        GV_LAUNCH(k_ms_to_f32, grid_for(n, 256), 256, 0, s, (const double *)(a.bc + (size_t)r * n),
                  mem == GV_MEM_DEVICE ? dst : tmp, n);
        if (mem != GV_MEM_DEVICE) {
            cudaError_t e = cudaMemcpyAsync(dst, tmp, (size_t)n * 4, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // tmp is reused by the next row
            if (e != cudaSuccess) return cuda_status(e, "bc out");
        }
    }
    return cuda_status(cudaStreamSynchronize(s), "bc out");
}

gv_status bfs_sigma_impl(gv_graph *g, uint32_t source, int32_t *dist, uint64_t *sigma, int mem, cudaStream_t s) {
    const uint32_t n = g->d.n;
    MsArena a;
    gv_status st = ms_setup(g, 1, 1, a);
    if (st != GV_OK) return st;
    MsBufs<1> b = a.bufs<1>(g);
    uint32_t slots[32];
    std::fill(slots, slots + 32, GV_NIL);
    slots[0] = source;
    cudaError_t e = cudaMemcpyAsync(a.dsrc, slots, sizeof(slots), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // slots is a stack array
    if (e != cudaSuccess) return cuda_status(e, "bfs source");
    uint32_t depth = 0;
    st = ms_forward<1>(g, b, a.dsrc, a.hflags, &depth, s);
    if (st != GV_OK) return st;
    // dist (int32) and sigma (u64) staged in light and the score row (n * 4 and n * 8 bytes)
    int32_t *ddist = (int32_t *)a.light;
    unsigned long long *dsig = (unsigned long long *)a.bc;
    GV_LAUNCH(k_ms_extract, grid_for(n, 256), 256, 0, s, b, depth, ddist, dsig);
    const cudaMemcpyKind k = mem == GV_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    e = cudaMemcpyAsync(dist, ddist, (size_t)n * 4, k, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sigma, dsig, (size_t)n * 8, k, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return cuda_status(e, "bfs sigma");
}

// Sources from host or device memory into a host vector.
gv_status bc_host_sources(const uint32_t *sources, uint64_t ns, int mem, cudaStream_t s, std::vector<uint32_t> &hs) {
    hs.resize(ns);
    if (!ns) return GV_OK;
    if (mem == GV_MEM_DEVICE) {
        cudaError_t e = cudaMemcpyAsync(hs.data(), sources, ns * 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        return cuda_status(e, "bc sources");
    }
    std::copy(sources, sources + ns, hs.begin());
    return GV_OK;
}

}  // namespace gv

using namespace gv;

extern "C" gv_status gv_bc(gv_graph *g, const uint32_t *sources, uint64_t ns, float *bc_out, int mem, void *stream) {
    if (!g || !bc_out) return GV_ERR_INVALID;
    if (!sources) ns = 0;  // every vertex
    const cudaStream_t s = (cudaStream_t)stream;
    std::vector<uint32_t> hs;
    gv_status st = bc_host_sources(sources, ns, mem, s, hs);
    if (st != GV_OK) return st;
    std::vector<uint64_t> off{0, hs.size()};
    return bc_requests(g, hs, off, 1, bc_out, mem, s);
}

extern "C" gv_status gv_bc_multi(gv_graph *g, const uint32_t *sources, const uint64_t *offsets, uint32_t nreq,
                                 float *bc_out, int mem, void *stream) {
    if (!g || !bc_out || !offsets || nreq == 0) return GV_ERR_INVALID;
    if ((uint64_t)nreq * std::max<uint32_t>(g->d.n, 1) > (1ull << 40)) {  // fp64 score rows in device scratch
        set_error("too many BC requests for one call");
        return GV_ERR_INVALID;
    }
    for (uint32_t r = 0; r < nreq; ++r)
        if (offsets[r + 1] < offsets[r]) { set_error("request offsets must not decrease"); return GV_ERR_INVALID; }
    if (offsets[0] != 0) { set_error("request offsets start at 0"); return GV_ERR_INVALID; }
    if (offsets[nreq] && !sources) return GV_ERR_INVALID;
    const cudaStream_t s = (cudaStream_t)stream;
    std::vector<uint32_t> hs;
    gv_status st = bc_host_sources(sources, offsets[nreq], mem, s, hs);
    if (st != GV_OK) return st;
    std::vector<uint64_t> off(offsets, offsets + nreq + 1);
    return bc_requests(g, hs, off, nreq, bc_out, mem, s);
}

extern "C" gv_status gv_bfs_sigma(gv_graph *g, uint32_t source, int32_t *dist, uint64_t *sigma, int mem, void *stream) {
    if (!g || !dist || !sigma || source >= g->d.n) return GV_ERR_INVALID;
    return bfs_sigma_impl(g, source, dist, sigma, mem, (cudaStream_t)stream);
}
