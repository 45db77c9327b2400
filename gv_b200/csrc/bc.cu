// Betweenness centrality (Brandes) and single-source BFS path counts over the
// edge-block store, 32 sources at a time, one source per lane.
//
// Replaces the reference's bc (src/algorithm/bc/bc.cu:3-88) and its kernels
// initializeArrays / initbfsKernel / bfsKernel / dependencyKernel
// (src/algorithm/bc/bc_kernel.cu:3-119), which run one source per host loop
// and one level per launch with int path counts and an unordered dependency
// pass.  Here the 32 sources of a batch share every adjacency read:
//
//   forward, level L -> L+1 (top-down over the union frontier): a warp takes
//   a vertex u that is at level L for the sources in mask F = masks[L][u];
//   lane s holds sigma_s(u).  For each neighbour w (ids read 32 at a time,
//   coalesced, with vis[w] prefetched per lane), want = F & ~vis[w]: the
//   sources that reach w first through this level.  One atomicOr marks them
//   in nxt[w]; the lanes in `want` add sigma_s(u) into sigma_s(w) (exact
//   uint64 adds, so the order does not matter).
//
//   backward, level L (pull, no atomics): a warp takes v at level L for the
//   sources in A = masks[L][v]; for each neighbour w, the lanes in
//   A & masks[L+1][w] (w one level deeper for that source) add
//   coef_s(w) = (1 + delta_s(w)) / sigma_s(w).  Then delta_s(v) =
//   sigma_s(v) * acc_s, coef_s(v) replaces sigma_s(v) in the same 8-byte slot,
//   and bc[v] += sum over lanes of delta_s(v) (fixed shuffle order, fp64).
//
// Level masks (32 bits per vertex per level) stay resident for the backward
// pass and are small enough to be gathered from L2; sigma / coef rows are
// vertex-major ([v][32] x 8 bytes), so the lanes of one vertex touch one
// 256-byte row.  Vertices with more than MS_HEAVY_FILL entries are expanded by
// a whole CTA (block table in shared memory, warps over blocks); the backward
// partials of a CTA are combined in warp order, so results are bit-for-bit
// repeatable.
#include <algorithm>
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
constexpr unsigned MS_LIGHT_GRID = 148 * 8;
constexpr unsigned MS_HEAVY_GRID = 148 * 2;
constexpr uint32_t MS_MAX_LEVELS = 1u << 16;

struct MsBufs {
    unsigned long long *row;  // [n][32] sigma (u64); after its level's backward step: coef (f64 bits)
    uint32_t *vis;            // [n] sources that reached v at a finished level
    uint32_t *nxt;            // [n] sources that reach v at the level being built
    uint32_t *masks;          // [levels][n]
    uint32_t *light;          // vertices of the current level, fill <= MS_HEAVY_FILL
    uint32_t *heavy;          // the rest
    uint32_t *cnt;            // [0] light, [1] heavy
    uint32_t *flags;          // [levels] level non-empty
    double *bc;               // [n]
    uint32_t n;
};

__device__ __forceinline__ double as_f64(unsigned long long x) { return __longlong_as_double((long long)x); }
__device__ __forceinline__ unsigned long long as_u64(double x) { return (unsigned long long)__double_as_longlong(x); }

__device__ __forceinline__ uint32_t ms_block(const DevGraph &g, uint32_t root, uint32_t k) {
    return k == 0 ? root : cbt_block(g.left, g.right, root, k);
}

// Walks the entries of one block 32 at a time: lane j loads entry e0 + j and
// its source mask pre(w) (0: nothing to do for any source); the entries with
// a non-zero mask are packed into the warp's shared slots, and body(w, mask)
// runs for each of them with the whole warp (lane = source).  In most levels
// few entries need work, so the warp skips the rest without touching them.
__shared__ uint2 ms_pack[MS_WARPS][32];  // one row of slots per warp (the kernels run MS_THREADS threads)

template <typename Pre, typename Body>
__device__ __forceinline__ void ms_block_entries(const DevGraph &g, uint32_t b, uint32_t slots, Pre &&pre,
                                                 Body &&body) {
    const uint32_t lane = threadIdx.x & 31u;
    uint2 *pack = ms_pack[threadIdx.x >> 5];
    const uint32_t *bp = g.pool + ((size_t)b << g.logB);
    for (uint32_t e0 = 0; e0 < slots; e0 += 32) {
        const uint32_t e = e0 + lane;
        uint32_t w = GV_TOMB, pv = 0;
        if (e < slots) {
            w = bp[e];
            if (w != GV_TOMB) pv = pre(w);
        }
        const uint32_t bal = __ballot_sync(GV_FULL_MASK, pv != 0);
        if (!bal) continue;  // warp-uniform
        if (pv) pack[__popc(bal & ((1u << lane) - 1u))] = make_uint2(w, pv);
        __syncwarp();
        const uint32_t c = __popc(bal);
        for (uint32_t j = 0; j < c; ++j) {
            const uint2 x = pack[j];
            body(x.x, x.y);
        }
        __syncwarp();
    }
}

// Light vertex: the warp's lanes hold its (at most 32) block indices.
template <typename Pre, typename Body>
__device__ __forceinline__ void ms_walk_light(const DevGraph &g, uint4 rec, Pre &&pre, Body &&body) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB);
    const uint32_t blk = lane < nb ? ms_block(g, rec.x, lane) : GV_NIL;
    for (uint32_t k = 0; k < nb; ++k) {
        const uint32_t b = __shfl_sync(GV_FULL_MASK, blk, k);
        ms_block_entries(g, b, min(g.B, fill - (k << g.logB)), pre, body);
    }
}

// Heavy vertex: the CTA fills a shared block table window by window; warps
// take blocks w, w + MS_WARPS, ...
template <typename Pre, typename Body>
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
            ms_block_entries(g, tab[i], min(g.B, fill - (k << g.logB)), pre, body);
        }
    }
}

__global__ void k_ms_init(MsBufs b, const uint32_t *__restrict__ src, uint32_t nsrc) {
    const uint32_t s = threadIdx.x;
    if (s >= nsrc) return;
    const uint32_t v = src[s];
    atomicOr(&b.masks[v], 1u << s);
    atomicOr(&b.vis[v], 1u << s);
    b.row[(size_t)v * 32 + s] = 1ull;
}

// Vertices of level L into the light / heavy lists (warp-aggregated appends).
__global__ void k_ms_split(DevGraph g, MsBufs b, const uint32_t *__restrict__ mask) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t n = b.n;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint32_t v = base + threadIdx.x;
        bool on = false, heavy = false;
        if (v < n && mask[v]) {
            on = true;
            heavy = g.vtx[v].y > MS_HEAVY_FILL;
        }
        const uint32_t bl = __ballot_sync(GV_FULL_MASK, on && !heavy), bh = __ballot_sync(GV_FULL_MASK, on && heavy);
        uint32_t ol = 0, oh = 0;
        if (lane == 0) {
            if (bl) ol = atomicAdd(&b.cnt[0], __popc(bl));
            if (bh) oh = atomicAdd(&b.cnt[1], __popc(bh));
        }
        ol = __shfl_sync(GV_FULL_MASK, ol, 0);
        oh = __shfl_sync(GV_FULL_MASK, oh, 0);
        const uint32_t below = (1u << lane) - 1u;
        if (on && !heavy) b.light[ol + __popc(bl & below)] = v;
        if (on && heavy) b.heavy[oh + __popc(bh & below)] = v;
    }
}

struct FwdBody {
    MsBufs b;
    uint32_t F;
    unsigned long long sig;
    // sources that reach w first through this level
    __device__ __forceinline__ uint32_t operator()(uint32_t w) const { return F & ~b.vis[w]; }
    __device__ __forceinline__ void visit(uint32_t w, uint32_t want) const {
        const uint32_t lane = threadIdx.x & 31u;
        if (lane == 0) atomicOr(&b.nxt[w], want);
        if ((want >> lane) & 1u) atomicAdd(&b.row[(size_t)w * 32 + lane], sig);
    }
};

__device__ __forceinline__ void ms_fwd_light(const DevGraph &g, const MsBufs &b, const uint32_t *__restrict__ mask,
                                             uint32_t vb, uint32_t vg) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nl = b.cnt[0];
    for (uint32_t i = vb * MS_WARPS + (threadIdx.x >> 5); i < nl; i += vg * MS_WARPS) {
        const uint32_t u = b.light[i];
        FwdBody f{b, mask[u], 0ull};
        if ((f.F >> lane) & 1u) f.sig = b.row[(size_t)u * 32 + lane];
        ms_walk_light(g, g.vtx[u], f, [&](uint32_t w, uint32_t vw) { f.visit(w, vw); });
    }
}

__device__ __forceinline__ void ms_fwd_heavy(const DevGraph &g, const MsBufs &b, const uint32_t *__restrict__ mask,
                                             uint32_t vb, uint32_t vg) {
    __shared__ uint32_t tab[MS_TAB];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nh = b.cnt[1];
    for (uint32_t i = vb; i < nh; i += vg) {
        const uint32_t u = b.heavy[i];
        FwdBody f{b, mask[u], 0ull};
        if ((f.F >> lane) & 1u) f.sig = b.row[(size_t)u * 32 + lane];
        ms_walk_heavy(g, g.vtx[u], tab, f, [&](uint32_t w, uint32_t vw) { f.visit(w, vw); });
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

__global__ void __launch_bounds__(MS_THREADS) k_ms_fwd(DevGraph g, MsBufs b, const uint32_t *__restrict__ mask) {
    uint32_t vb, vgl, vgh;
    if (ms_split_cta(vb, vgl, vgh)) ms_fwd_heavy(g, b, mask, vb, vgh);
    else ms_fwd_light(g, b, mask, vb, vgl);
}

// Closes level L: masks[L+1] = nxt, vis |= nxt, flags[L+1] = any.
__global__ void k_ms_close(MsBufs b, uint32_t *__restrict__ next_mask, uint32_t *flag) {
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    bool mine = false;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < b.n; v += gridDim.x * blockDim.x) {
        const uint32_t x = b.nxt[v];
        next_mask[v] = x;
        if (x) {
            b.vis[v] |= x;
            b.nxt[v] = 0;
            mine = true;
        }
    }
    if (mine) any = 1;
    __syncthreads();
    if (threadIdx.x == 0 && any) atomicOr(flag, 1u);
}


// Backward sum over one block's entries for the lanes in A: entries 32 at a
// time, lane j loads entry j and masks[L+1] of it; then every lane adds
// coef(w_j) for the entries one level deeper for its source.  The gathers are
// predicated and unrolled so a warp keeps several in flight.
__device__ __forceinline__ double ms_bwd_block(const DevGraph &g, const MsBufs &b, const uint32_t *__restrict__ deeper,
                                               uint32_t blk, uint32_t slots, uint32_t A) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t *bp = g.pool + ((size_t)blk << g.logB);
    const unsigned long long *row = b.row;
    double acc = 0.0;
    for (uint32_t e0 = 0; e0 < slots; e0 += 32) {
        const uint32_t e = e0 + lane;
        uint32_t w = 0, mw = 0;
        if (e < slots) {
            w = bp[e];
            if (w != GV_TOMB) mw = deeper[w] & A;
            else w = 0;
        }
        const uint32_t bal = __ballot_sync(GV_FULL_MASK, mw != 0);
        if (!bal) continue;  // warp-uniform
        uint2 *pack = ms_pack[threadIdx.x >> 5];
        if (mw) pack[__popc(bal & ((1u << lane) - 1u))] = make_uint2(w, mw);
        __syncwarp();
        const uint32_t c = __popc(bal);
        for (uint32_t j0 = 0; j0 < c; j0 += 8) {  // eight gathers in flight, summed in entry order
            uint2 x[8];
#pragma unroll
            for (int t = 0; t < 8; ++t) x[t] = (j0 + t < c) ? pack[j0 + t] : make_uint2(0u, 0u);
            unsigned long long v[8];
#pragma unroll
            for (int t = 0; t < 8; ++t) v[t] = ((x[t].y >> lane) & 1u) ? __ldg(row + (size_t)x[t].x * 32 + lane) : 0ull;
#pragma unroll
            for (int t = 0; t < 8; ++t) acc += as_f64(v[t]);
        }
        __syncwarp();
    }
    return acc;
}

// Backward walk of a light vertex (lanes hold its block indices).
__device__ __forceinline__ double ms_bwd_light(const DevGraph &g, const MsBufs &b, const uint32_t *__restrict__ deeper,
                                               uint4 rec, uint32_t A) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB);
    const uint32_t blk = lane < nb ? ms_block(g, rec.x, lane) : GV_NIL;
    double acc = 0.0;
    for (uint32_t k = 0; k < nb; ++k) {
        const uint32_t bk = __shfl_sync(GV_FULL_MASK, blk, k);
        acc += ms_bwd_block(g, b, deeper, bk, min(g.B, fill - (k << g.logB)), A);
    }
    return acc;
}

// Finishes (v, lanes in A) from acc: delta = sigma * acc, coef replaces
// sigma, returns the lane's delta (0 outside A).
__device__ __forceinline__ double ms_finish(MsBufs &b, uint32_t v, uint32_t A, unsigned long long sig, double acc) {
    const uint32_t lane = threadIdx.x & 31u;
    if (!((A >> lane) & 1u)) return 0.0;
    const double sv = (double)sig;
    const double delta = sv * acc;
    b.row[(size_t)v * 32 + lane] = as_u64((1.0 + delta) / sv);
    return delta;
}

__device__ __forceinline__ void ms_bwd_light_v(const DevGraph &g, MsBufs b, const uint32_t *__restrict__ mask,
                                               const uint32_t *__restrict__ deeper, uint32_t vb, uint32_t vg) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nl = b.cnt[0];
    for (uint32_t i = vb * MS_WARPS + (threadIdx.x >> 5); i < nl; i += vg * MS_WARPS) {
        const uint32_t v = b.light[i];
        const uint32_t A = mask[v];
        const unsigned long long sig = ((A >> lane) & 1u) ? b.row[(size_t)v * 32 + lane] : 0ull;
        const double acc = ms_bwd_light(g, b, deeper, g.vtx[v], A);
        double d = ms_finish(b, v, A, sig, acc);
        d = warp_sum(d);
        if (lane == 0) b.bc[v] += d;
    }
}

__device__ __forceinline__ void ms_bwd_heavy_v(const DevGraph &g, MsBufs b, const uint32_t *__restrict__ mask,
                                               const uint32_t *__restrict__ deeper, uint32_t vb, uint32_t vg) {
    __shared__ uint32_t tab[MS_TAB];
    __shared__ double red[MS_WARPS][32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t nh = b.cnt[1];
    for (uint32_t i = vb; i < nh; i += vg) {
        const uint32_t v = b.heavy[i];
        const uint32_t A = mask[v];
        const unsigned long long sig = ((A >> lane) & 1u) ? b.row[(size_t)v * 32 + lane] : 0ull;
        double acc = 0.0;
        const uint4 rec = g.vtx[v];
        const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB);
        for (uint32_t k0 = 0; k0 < nb; k0 += MS_TAB) {
            const uint32_t cnt = min(MS_TAB, nb - k0);
            __syncthreads();
            for (uint32_t t = threadIdx.x; t < cnt; t += blockDim.x) tab[t] = ms_block(g, rec.x, k0 + t);
            __syncthreads();
            for (uint32_t t = warp; t < cnt; t += MS_WARPS)
                acc += ms_bwd_block(g, b, deeper, tab[t], min(g.B, fill - ((k0 + t) << g.logB)), A);
        }
        red[warp][lane] = acc;
        __syncthreads();
        if (warp == 0) {
            double t = 0.0;
            for (int w = 0; w < MS_WARPS; ++w) t += red[w][lane];
            double d = ms_finish(b, v, A, sig, t);
            d = warp_sum(d);
            if (lane == 0) b.bc[v] += d;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(MS_THREADS) k_ms_bwd(DevGraph g, MsBufs b, const uint32_t *__restrict__ mask,
                                                       const uint32_t *__restrict__ deeper) {
    uint32_t vb, vgl, vgh;
    if (ms_split_cta(vb, vgl, vgh)) ms_bwd_heavy_v(g, b, mask, deeper, vb, vgh);
    else ms_bwd_light_v(g, b, mask, deeper, vb, vgl);
}

__global__ void k_ms_to_f32(const double *__restrict__ x, float *__restrict__ y, uint32_t n) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) y[v] = (float)x[v];
}

// dist / sigma of lane 0 after a one-source forward pass.
__global__ void k_ms_extract(MsBufs b, uint32_t depth, int32_t *__restrict__ dist, unsigned long long *__restrict__ sigma) {
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

// Level masks live in auxiliary slot 6 and grow (keeping their contents)
// when a BFS runs deeper than the levels allocated.
gv_status masks_reserve(gv_graph *g, MsBufs &b, uint32_t levels, uint32_t keep_levels, uint32_t &cap, cudaStream_t s) {
    if (levels <= cap) return GV_OK;
    uint32_t want = std::max<uint32_t>(32, cap);
    while (want < levels) want *= 2;
    if (want > MS_MAX_LEVELS) {
        set_error("BFS deeper than the level table");
        return GV_ERR_UNSUPPORTED;
    }
    const size_t bytes = (size_t)want * b.n * 4;
    if (bytes <= g->aux_bytes[6]) {
        cap = (uint32_t)(g->aux_bytes[6] / ((size_t)b.n * 4));
        b.masks = (uint32_t *)g->aux[6];
        return GV_OK;
    }
    void *nb = nullptr;
    if (cudaMalloc(&nb, bytes) != cudaSuccess) {
        cudaGetLastError();
        set_error("level masks allocation of " + std::to_string(bytes) + " B failed");
        return GV_ERR_NOMEM;
    }
    if (keep_levels && g->aux[6]) {
        cudaError_t e = cudaMemcpyAsync(nb, g->aux[6], (size_t)keep_levels * b.n * 4, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            cudaFree(nb);
            return cuda_status(e, "level masks copy");
        }
    }
    if (g->aux[6]) cudaFree(g->aux[6]);
    g->aux[6] = nb;
    g->aux_bytes[6] = bytes;
    b.masks = (uint32_t *)nb;
    cap = want;
    return GV_OK;
}

// Forward pass for the sources already placed by k_ms_init; returns the
// deepest non-empty level.
gv_status ms_forward(gv_graph *g, MsBufs &b, uint32_t &cap, uint32_t *h_flags, uint32_t *depth_out, cudaStream_t s) {
    const DevGraph d = g->d;
    const uint32_t n = b.n;
    const uint32_t chunk = 4;
    uint32_t L = 0;
    for (;;) {
        gv_status st = masks_reserve(g, b, L + chunk + 2, L + 1, cap, s);
        if (st != GV_OK) return st;
        cudaMemsetAsync(b.flags + L + 1, 0, chunk * 4, s);
        for (uint32_t i = 0; i < chunk; ++i, ++L) {
            const uint32_t *mask = b.masks + (size_t)L * n;
            ProfScope ps(PROF_BFS_LEVEL, s);
            cudaMemsetAsync(b.cnt, 0, 8, s);
            GV_LAUNCH(k_ms_split, grid_for(n, 256), 256, 0, s, d, b, mask);
            static_assert(MS_LIGHT_GRID == 4 * MS_HEAVY_GRID, "the fused launch interleaves 4 light CTAs per heavy one");
            GV_LAUNCH(k_ms_fwd, MS_LIGHT_GRID + MS_HEAVY_GRID, MS_THREADS, 0, s, d, b, mask);
            GV_LAUNCH(k_ms_close, grid_for(n, 256), 256, 0, s, b, b.masks + (size_t)(L + 1) * n, b.flags + L + 1);
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

gv_status ms_backward(gv_graph *g, MsBufs &b, uint32_t depth, cudaStream_t s) {
    const DevGraph d = g->d;
    const uint32_t n = b.n;
    for (uint32_t L = depth; L >= 1; --L) {
        const uint32_t *mask = b.masks + (size_t)L * n;
        const uint32_t *deeper = b.masks + (size_t)(L + 1) * n;
        ProfScope ps(PROF_BC_DEP, s);
        cudaMemsetAsync(b.cnt, 0, 8, s);
        GV_LAUNCH(k_ms_split, grid_for(n, 256), 256, 0, s, d, b, mask);
        GV_LAUNCH(k_ms_bwd, MS_LIGHT_GRID + MS_HEAVY_GRID, MS_THREADS, 0, s, d, b, mask, deeper);
    }
    return cuda_status(cudaGetLastError(), "bc dependencies");
}

size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

// Carves the per-batch buffers from the analytics scratch.
gv_status ms_setup(gv_graph *g, MsBufs &b, uint32_t **dsrc, uint32_t **hflags) {
    const uint32_t n = g->d.n;
    b.n = n;
    const size_t o_row = 0, o_vis = o_row + al256((size_t)n * 256), o_nxt = o_vis + al256((size_t)n * 4);
    const size_t o_light = o_nxt + al256((size_t)n * 4), o_heavy = o_light + al256((size_t)n * 4);
    const size_t o_cnt = o_heavy + al256((size_t)n * 4), o_flags = o_cnt + 256;
    const size_t o_bc = o_flags + al256((size_t)MS_MAX_LEVELS * 4 + 4), o_src = o_bc + al256((size_t)n * 8);
    const size_t bytes = o_src + 256;
    char *p = (char *)analytics_scratch(g, bytes);
    if (!p) return GV_ERR_NOMEM;
    b.row = (unsigned long long *)(p + o_row);
    b.vis = (uint32_t *)(p + o_vis);
    b.nxt = (uint32_t *)(p + o_nxt);
    b.light = (uint32_t *)(p + o_light);
    b.heavy = (uint32_t *)(p + o_heavy);
    b.cnt = (uint32_t *)(p + o_cnt);
    b.flags = (uint32_t *)(p + o_flags);
    b.bc = (double *)(p + o_bc);
    *dsrc = (uint32_t *)(p + o_src);
    b.masks = (uint32_t *)g->aux[6];
    if (hflags && !g->host_pinned) {
        if (cudaMallocHost(&g->host_pinned, 256) != cudaSuccess) {
            cudaGetLastError();
            set_error("pinned host word allocation failed");
            return GV_ERR_NOMEM;
        }
        g->host_pinned_bytes = 256;
    }
    if (hflags) *hflags = (uint32_t *)g->host_pinned;
    return GV_OK;
}

// One batch of up to 32 sources (device array dsrc, already filled).
gv_status ms_batch(gv_graph *g, MsBufs &b, const uint32_t *dsrc, uint32_t nsrc, uint32_t &cap, uint32_t *hflags,
                   uint32_t *depth, cudaStream_t s) {
    const uint32_t n = b.n;
    gv_status st = masks_reserve(g, b, 8, 0, cap, s);
    if (st != GV_OK) return st;
    cudaMemsetAsync(b.row, 0, (size_t)n * 256, s);
    cudaMemsetAsync(b.vis, 0, (size_t)n * 4, s);
    cudaMemsetAsync(b.nxt, 0, (size_t)n * 4, s);
    cudaMemsetAsync(b.masks, 0, (size_t)n * 4, s);
    GV_LAUNCH(k_ms_init, 1, 32, 0, s, b, dsrc, nsrc);
    return ms_forward(g, b, cap, hflags, depth, s);
}

}  // namespace

gv_status bc_impl(gv_graph *g, const uint32_t *sources, uint64_t ns, float *bc_out, int mem, cudaStream_t s) {
    const uint32_t n = g->d.n;
    std::vector<uint32_t> src_all;
    const uint32_t *hs = sources;
    if (!sources || ns == 0) {
        src_all.resize(n);
        for (uint32_t i = 0; i < n; ++i) src_all[i] = i;
        hs = src_all.data();
        ns = n;
    } else if (mem == GV_MEM_DEVICE) {
        src_all.resize(ns);
        cudaError_t e = cudaMemcpyAsync(src_all.data(), sources, ns * 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e, "bc sources");
        hs = src_all.data();
    }
    for (uint64_t i = 0; i < ns; ++i)
        if (hs[i] >= n) { set_error("BC source out of range"); return GV_ERR_INVALID; }
    MsBufs b;
    uint32_t *dsrc = nullptr, *hflags = nullptr;
    gv_status st = ms_setup(g, b, &dsrc, &hflags);
    if (st != GV_OK) return st;
    uint32_t cap = g->aux[6] ? (uint32_t)(g->aux_bytes[6] / ((size_t)n * 4)) : 0;
    cudaMemsetAsync(b.bc, 0, (size_t)n * 8, s);
    for (uint64_t s0 = 0; s0 < ns; s0 += 32) {
        const uint32_t nsrc = (uint32_t)std::min<uint64_t>(32, ns - s0);
        cudaError_t e = cudaMemcpyAsync(dsrc, hs + s0, nsrc * 4, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return cuda_status(e, "bc sources");
        uint32_t depth = 0;
        st = ms_batch(g, b, dsrc, nsrc, cap, hflags, &depth, s);
        if (st != GV_OK) return st;
        st = ms_backward(g, b, depth, s);
        if (st != GV_OK) return st;
    }
    float *tmp = (float *)b.vis;  // n floats fit in vis + nxt
    GV_LAUNCH(k_ms_to_f32, grid_for(n, 256), 256, 0, s, (const double *)b.bc, tmp, n);
    cudaError_t e = cudaMemcpyAsync(bc_out, tmp, (size_t)n * 4,
                                    mem == GV_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return cuda_status(e, "bc out");
}

gv_status bfs_sigma_impl(gv_graph *g, uint32_t source, int32_t *dist, uint64_t *sigma, int mem, cudaStream_t s) {
    const uint32_t n = g->d.n;
    MsBufs b;
    uint32_t *dsrc = nullptr, *hflags = nullptr;
    gv_status st = ms_setup(g, b, &dsrc, &hflags);
    if (st != GV_OK) return st;
    uint32_t cap = g->aux[6] ? (uint32_t)(g->aux_bytes[6] / ((size_t)n * 4)) : 0;
    cudaError_t e = cudaMemcpyAsync(dsrc, &source, 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // &source is a stack word
    if (e != cudaSuccess) return cuda_status(e, "bfs source");
    uint32_t depth = 0;
    st = ms_batch(g, b, dsrc, 1, cap, hflags, &depth, s);
    if (st != GV_OK) return st;
    // dist (int32) and sigma (u64) staged in light / heavy + bc (n * 4 and n * 8 bytes)
    int32_t *ddist = (int32_t *)b.light;
    unsigned long long *dsig = (unsigned long long *)b.bc;
    GV_LAUNCH(k_ms_extract, grid_for(n, 256), 256, 0, s, b, depth, ddist, dsig);
    const cudaMemcpyKind k = mem == GV_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    e = cudaMemcpyAsync(dist, ddist, (size_t)n * 4, k, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sigma, dsig, (size_t)n * 8, k, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return cuda_status(e, "bfs sigma");
}

}  // namespace gv

using namespace gv;

extern "C" gv_status gv_bc(gv_graph *g, const uint32_t *sources, uint64_t ns, float *bc_out, int mem, void *stream) {
    if (!g || !bc_out) return GV_ERR_INVALID;
    return bc_impl(g, sources, ns, bc_out, mem, (cudaStream_t)stream);
}

extern "C" gv_status gv_bfs_sigma(gv_graph *g, uint32_t source, int32_t *dist, uint64_t *sigma, int mem, void *stream) {
    if (!g || !dist || !sigma || source >= g->d.n) return GV_ERR_INVALID;
    return bfs_sigma_impl(g, source, dist, sigma, mem, (cudaStream_t)stream);
}
