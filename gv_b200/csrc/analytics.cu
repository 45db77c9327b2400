// Analytics that traverse the edge-block CBT store directly: PageRank,
// personalised PageRank, exact triangle counting and weighted PageRank with
// its adjoint (betweenness centrality: bc.cu; subset triangles: tc_local.cu).
//
// Reference kernels replaced:
//   PageRank   src/algorithm/pagerank/pr_kernel.cu:3-103, pagerank.cu:3-132
//              (push + float atomics + host reduce per sweep) -> pull over
//              the symmetric store, deterministic, residual reduced on the
//              device, no host round trip per sweep;
//   TC         src/algorithm/tc/tc_kernel.cu:3-147 (triple linear scans,
//              float counts) -> degree-oriented sorted snapshot + merge-path
//              intersection (packed hash probe behind GV_TC_PACKED=1),
//              uint64 counts;
#include <algorithm>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>
#include "../../include/gv_batch.h"
#include "store.cuh"
#include "group.cuh"
#include "prims.cuh"
#include "launch.hpp"
#include "prof.hpp"

namespace gv {
namespace {

constexpr int AN_THREADS = 256;
// What a triangle count credits: the smallest id of each triangle (per-vertex
// counts as the reference keeps them), all three vertices, or only the total.
constexpr int TC_OWNER = 0, TC_INCIDENT = 1, TC_TOTAL = 2;
constexpr int BIG_TAB_A = 1024;
// Pull sweeps route vertices by used slots: lane groups up to LIGHT_FILL,
// one CTA per vertex up to HUB_FILL, the whole grid above.
constexpr uint32_t LIGHT_FILL = 256;
constexpr uint32_t TINY_FILL = 32;  // thread-per-vertex tier of the pull sweeps
constexpr unsigned FIN_GRID = 148;
// The fused sweep runs SWEEP_WAVES rounds of SWEEP_PERIOD CTAs; of each
// round, the tiers get CTAs in proportion to their estimated work, so no
// tier's CTAs carry the tail.  Residual slots: lane-group tier [0,
// SWEEP_GRID), item finish [SWEEP_GRID, + FIN_GRID), thread-per-vertex tier
// [SWEEP_GRID + FIN_GRID, + SWEEP_GRID).
constexpr unsigned SWEEP_PERIOD = 16;
constexpr unsigned SWEEP_WAVES = 148 * 24 / SWEEP_PERIOD;
constexpr unsigned SWEEP_GRID = SWEEP_PERIOD * SWEEP_WAVES;
constexpr unsigned SWEEP_PARTS = SWEEP_GRID + FIN_GRID + SWEEP_GRID;
constexpr uint32_t HUB_FILL = 16384;

// Lanes per block and blocks per warp step for the grid-cooperative paths.
struct WarpBlocks {
    uint32_t lpb, bpw, sub, sl;
    __device__ __forceinline__ explicit WarpBlocks(uint32_t B) {
        const uint32_t lane = threadIdx.x & 31u;
        lpb = min(32u, B >> 2);
        bpw = 32u / lpb;
        sub = lane / lpb;
        sl = lane % lpb;
    }
};

// ----------------------------------------------------------- pull sweeps
// out[v] = base(v) + alpha * scale(v) * sum_{u in N(v)} w(v,u) * gather[u]
struct PullArgs {
    const float *gather;
    float alpha;
    float base_all;       // added to every vertex
    uint32_t base_src;    // vertex that also gets base_src_val (GV_NIL: none)
    float base_src_val;
    const float *cvec;    // per-vertex additive term (nullable)
    const float *rscale;  // per-vertex multiplier of the sum (nullable)
    const float *xold;    // previous iterate (residual)
    float *xnew;
    float *contrib;       // xnew / deg (nullable)
    double *partial;      // one slot per CTA (+ heavy kernel slots)
    const int *state;     // [0] done flag
};

__device__ __forceinline__ float pull_finish(const PullArgs &a, uint32_t v, float sum, uint32_t deg,
                                             double &res) {
    float base = a.base_all + (v == a.base_src ? a.base_src_val : 0.f);
    if (a.cvec) base += a.cvec[v];
    const float sc = a.rscale ? a.rscale[v] : 1.f;
    const float xv = base + a.alpha * (sc * sum);
    a.xnew[v] = xv;
    if (a.contrib) a.contrib[v] = deg ? xv / (float)deg : 0.f;
    res += (double)fabsf(xv - a.xold[v]);
    return xv;
}

// Adds the gathered values of the live entries among four (entries at or past
// `limit` and tombstones skipped).
template <bool W>
__device__ __forceinline__ float pull_gather4(const PullArgs &a, uint4 q, float4 wq, uint32_t e, uint32_t limit) {
    const uint32_t ev[4] = {q.x, q.y, q.z, q.w};
    const float wv[4] = {wq.x, wq.y, wq.z, wq.w};
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (e + j < limit && ev[j] != GV_TOMB) s += W ? wv[j] * __ldg(a.gather + ev[j]) : __ldg(a.gather + ev[j]);
    return s;
}

// Vertices with at most TINY_FILL entries: one thread per vertex issues all
// of its (at most 8) 16-byte loads and gathers at once, so the dependent
// chain vertex -> block -> neighbours is paid once per thread instead of
// once per vertex by a whole lane group.
template <bool W>
__device__ __forceinline__ void pull_tiny_body(const DevGraph &g, const PullArgs &a, const uint32_t *__restrict__ list,
                                               uint32_t cnt, uint32_t part_base, uint32_t vb, uint32_t vg) {
    __shared__ double red[AN_THREADS / 32];
    if (a.state[0]) return;
    double res = 0.0;
    for (uint32_t i = vb * blockDim.x + threadIdx.x; i < cnt; i += vg * blockDim.x) {
        const uint32_t v = list[i];  // the vertices with at most TINY_FILL entries, in id order
        const uint4 rec = g.vtx[v];
        const uint32_t fill = rec.y;
        float sum = 0.f;
        if (fill) {
            const size_t base = (size_t)rec.x << g.logB;  // fill <= 32 <= B: one block
#pragma unroll
            for (uint32_t e = 0; e < TINY_FILL; e += 4) {
                if (e < fill) {
                    const uint4 q = __ldcs(reinterpret_cast<const uint4 *>(g.pool + base + e));
                    float4 wq = make_float4(1.f, 1.f, 1.f, 1.f);
                    if (W) wq = __ldcs(reinterpret_cast<const float4 *>(g.wpool + base + e));
                    const uint32_t ev[4] = {q.x, q.y, q.z, q.w};
                    const float wv[4] = {wq.x, wq.y, wq.z, wq.w};
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        if (e + j < fill && ev[j] != GV_TOMB)
                            sum += W ? wv[j] * __ldg(a.gather + ev[j]) : __ldg(a.gather + ev[j]);
                }
            }
        }
        pull_finish(a, v, sum, rec.z, res);
    }
    res = warp_sum(res);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = res;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < AN_THREADS / 32; ++i) t += red[i];
        a.partial[part_base + vb] = t;
    }
}

template <int TPV, bool W>
__device__ __forceinline__ void pull_body(const DevGraph &g, const PullArgs &a, const uint32_t *__restrict__ list,
                                          uint32_t cnt, uint32_t vb, uint32_t vg) {
    __shared__ double red[AN_THREADS / 32];
    if (a.state[0]) return;
    constexpr int GPC = AN_THREADS / TPV;
    __shared__ uint32_t tabs[GPC][BIG_BLOCKS];
    Group<TPV> G;
    uint32_t *tab = tabs[threadIdx.x / TPV];
    const uint32_t ngroups = vg * GPC;
    double res = 0.0;
    for (uint32_t i = vb * GPC + threadIdx.x / TPV; i < cnt; i += ngroups) {
        const uint32_t v = list[i];  // the vertices with TINY_FILL < fill <= LIGHT_FILL, in id order
        const uint4 rec = g.vtx[v];
        const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB);
        float sum = 0.f;
        if (nb == 1) {
            // two 16-byte loads per lane before their gathers: eight gathers in flight
            const size_t base = (size_t)rec.x << g.logB;
            for (uint32_t e = G.gl * 4; e < fill; e += TPV * 8) {
                const uint32_t e2 = e + TPV * 4;
                const uint4 q = __ldcs(reinterpret_cast<const uint4 *>(g.pool + base + e));
                uint4 q2 = make_uint4(GV_TOMB, GV_TOMB, GV_TOMB, GV_TOMB);
                if (e2 < fill) q2 = __ldcs(reinterpret_cast<const uint4 *>(g.pool + base + e2));
                float4 wq = make_float4(1.f, 1.f, 1.f, 1.f), wq2 = wq;
                if (W) {
                    wq = __ldcs(reinterpret_cast<const float4 *>(g.wpool + base + e));
                    if (e2 < fill) wq2 = __ldcs(reinterpret_cast<const float4 *>(g.wpool + base + e2));
                }
                sum += pull_gather4<W>(a, q, wq, e, fill);
                sum += pull_gather4<W>(a, q2, wq2, e2, fill);
            }
        } else if (nb > 1) {
            fill_block_table(g, rec.x, 0, nb, tab, G.gl, TPV);
            G.sync();
            const uint32_t nq = (fill + 3) >> 2;
            for (uint32_t qi = G.gl; qi < nq; qi += 2 * TPV) {
                const uint32_t e = qi << 2, e2 = (qi + TPV) << 2;
                const size_t at = ((size_t)tab[e >> g.logB] << g.logB) + (e & (g.B - 1));
                const uint4 q = __ldcs(reinterpret_cast<const uint4 *>(g.pool + at));
                uint4 q2 = make_uint4(GV_TOMB, GV_TOMB, GV_TOMB, GV_TOMB);
                size_t at2 = 0;
                if (qi + TPV < nq) {
                    at2 = ((size_t)tab[e2 >> g.logB] << g.logB) + (e2 & (g.B - 1));
                    q2 = __ldcs(reinterpret_cast<const uint4 *>(g.pool + at2));
                }
                float4 wq = make_float4(1.f, 1.f, 1.f, 1.f), wq2 = wq;
                if (W) {
                    wq = __ldcs(reinterpret_cast<const float4 *>(g.wpool + at));
                    if (qi + TPV < nq) wq2 = __ldcs(reinterpret_cast<const float4 *>(g.wpool + at2));
                }
                sum += pull_gather4<W>(a, q, wq, e, fill);
                sum += pull_gather4<W>(a, q2, wq2, e2, fill);
            }
            G.sync();
        }
        sum = G.sum(sum);
        if (G.gl == 0) pull_finish(a, v, sum, rec.z, res);
    }
    res = warp_sum(res);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = res;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < AN_THREADS / 32; ++i) t += red[i];
        a.partial[vb] = t;
    }
}

// ---------------------------------------------------- chunked work items
// Vertices above LIGHT_FILL are cut into items of 32 blocks; one warp takes
// one item, so a hub of a million entries is spread over hundreds of warps
// and every warp gets about the same work.  Items of a vertex are adjacent
// and their partials are combined in item order (deterministic).
struct Items {
    const uint32_t *item_vertex;  // item -> vertex
    const uint32_t *item_first;   // vertex -> its first item (n + 1)
    const uint32_t *multi;        // vertices that have items
    const uint32_t *light;        // vertices with TINY_FILL < fill <= LIGHT_FILL (lane-group tier), id order
    const uint32_t *tiny;         // vertices with fill <= TINY_FILL (thread-per-vertex tier), id order
    uint32_t nitems, nmulti, nlight, ntiny;
    uint32_t split;               // CTAs of the fused sweep per SWEEP_PERIOD: lane-group | tiny << 8 | items << 16
};

// Items per vertex; tier[0..4] (nullable) gets the entries and vertices of
// the thread-per-vertex tier, those of the lane-group tier and the entries
// of the item tier, which size the tiers' shares of the fused sweep.
__global__ void k_item_count(DevGraph g, uint32_t *__restrict__ cnt, uint32_t *__restrict__ multi,
                             unsigned long long *nmulti, unsigned long long *__restrict__ tier) {
    const uint32_t chunk_log = g.logB + 5;  // 32 blocks per item
    unsigned long long t[5] = {0, 0, 0, 0, 0};
    for (uint32_t base = blockIdx.x * blockDim.x; base < g.n; base += gridDim.x * blockDim.x) {
        const uint32_t v = base + threadIdx.x;
        if (v >= g.n) continue;
        const uint32_t fill = g.vtx[v].y;
        uint32_t c = 0;
        if (fill > LIGHT_FILL) {
            c = (fill + (1u << chunk_log) - 1) >> chunk_log;
            multi[atomicAdd(nmulti, 1ull)] = v;
            t[4] += fill;
        } else if (fill > TINY_FILL) {
            t[2] += fill;
            t[3] += 1;
        } else if (fill) {
            t[0] += fill;
            t[1] += 1;
        }
        cnt[v] = c;
    }
    if (!tier) return;
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        const unsigned long long s = warp_sum(t[i]);
        if ((threadIdx.x & 31) == 0 && s) atomicAdd(&tier[i], s);
    }
}

// Tier flags of every vertex: tl[v] = 1 for the lane-group tier, tt[v] = 1
// for the thread-per-vertex tier (scanned into list positions next).
__global__ void k_tier_flags(DevGraph g, uint32_t *__restrict__ tl, uint32_t *__restrict__ tt) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < g.n; v += gridDim.x * blockDim.x) {
        const uint32_t fill = g.vtx[v].y;
        tl[v] = (fill > TINY_FILL && fill <= LIGHT_FILL) ? 1u : 0u;
        tt[v] = fill <= TINY_FILL ? 1u : 0u;
    }
}

// Scatters the tier members into their lists at the scanned positions (id order).
__global__ void k_tier_lists(DevGraph g, const uint32_t *__restrict__ pl, const uint32_t *__restrict__ pt,
                             uint32_t *__restrict__ light, uint32_t *__restrict__ tiny) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < g.n; v += gridDim.x * blockDim.x) {
        if (pl[v + 1] != pl[v]) light[pl[v]] = v;
        if (pt[v + 1] != pt[v]) tiny[pt[v]] = v;
    }
}

__global__ void k_item_fill(uint32_t n, const uint32_t *__restrict__ first, uint32_t *__restrict__ item_vertex) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        for (uint32_t i = first[v]; i < first[v + 1]; ++i) item_vertex[i] = v;
}

// Pool index of block (item block base + lane) for the lanes that have one.
__device__ __forceinline__ uint32_t item_block(const DevGraph &g, uint4 rec, uint32_t kb0, uint32_t nb) {
    const uint32_t k = kb0 + (threadIdx.x & 31u);
    if (k >= nb) return GV_NIL;
    return (k == 0) ? rec.x : cbt_block(g.left, g.right, rec.x, k);
}

template <bool W>
__device__ __forceinline__ void pull_items_body(const DevGraph &g, const PullArgs &a, const Items &it,
                                                float *__restrict__ ipart, uint32_t vb, uint32_t vg) {
    if (a.state[0]) return;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t nw = vg * (AN_THREADS / 32);
    for (uint32_t i = vb * (AN_THREADS / 32) + (threadIdx.x >> 5); i < it.nitems; i += nw) {
        const uint32_t v = it.item_vertex[i];
        const uint32_t c = i - it.item_first[v];
        const uint4 rec = g.vtx[v];
        const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB);
        const uint32_t kb0 = c << 5;
        const uint32_t my_blk = item_block(g, rec, kb0, nb);
        const uint32_t e0 = kb0 << g.logB;
        const uint32_t e1 = min(fill, (kb0 + 32) << g.logB);
        const uint32_t nq = (e1 - e0 + 3) >> 2;
        float sum = 0.f;
        for (uint32_t q0 = 0; q0 < nq; q0 += 64) {  // warp-uniform trip count; two loads per lane in flight
            const uint32_t q = q0 + lane, q2 = q + 32;
            const uint32_t el = q << 2, el2 = q2 << 2;  // entry offsets within the item
            const uint32_t pb = __shfl_sync(GV_FULL_MASK, my_blk, (el >> g.logB) & 31u);
            const uint32_t pb2 = __shfl_sync(GV_FULL_MASK, my_blk, (el2 >> g.logB) & 31u);
            uint4 qv = make_uint4(GV_TOMB, GV_TOMB, GV_TOMB, GV_TOMB), qv2 = qv;
            float4 wq = make_float4(1.f, 1.f, 1.f, 1.f), wq2 = wq;
            const size_t at = ((size_t)pb << g.logB) + (el & (g.B - 1));
            const size_t at2 = ((size_t)pb2 << g.logB) + (el2 & (g.B - 1));
            if (q < nq) {
                qv = __ldcs(reinterpret_cast<const uint4 *>(g.pool + at));
                if (W) wq = __ldcs(reinterpret_cast<const float4 *>(g.wpool + at));
            }
            if (q2 < nq) {
                qv2 = __ldcs(reinterpret_cast<const uint4 *>(g.pool + at2));
                if (W) wq2 = __ldcs(reinterpret_cast<const float4 *>(g.wpool + at2));
            }
            sum += pull_gather4<W>(a, qv, wq, e0 + el, e1);
            sum += pull_gather4<W>(a, qv2, wq2, e0 + el2, e1);
        }
        sum = warp_sum(sum);
        if (lane == 0) ipart[i] = sum;
    }
}

// One launch for the three tiers of a sweep, CTAs interleaved (each round of
// SWEEP_PERIOD CTAs holds the tiers' shares, it.split) so the lane-group,
// thread-per-vertex and hub-item work share every wave instead of running one
// after another.
template <int TPV, bool W>
__global__ void __launch_bounds__(AN_THREADS) k_pull_fused(DevGraph g, PullArgs a, Items it, float *__restrict__ ipart,
                                                           uint32_t tiny_base) {
    const uint32_t t0 = it.split & 0xFFu, t1 = (it.split >> 8) & 0xFFu, t2 = (it.split >> 16) & 0xFFu;
    const uint32_t r = blockIdx.x % SWEEP_PERIOD, w = blockIdx.x / SWEEP_PERIOD, waves = gridDim.x / SWEEP_PERIOD;
    if (r < t0) pull_body<TPV, W>(g, a, it.light, it.nlight, w * t0 + r, waves * t0);
    else if (r < t0 + t1) pull_tiny_body<W>(g, a, it.tiny, it.ntiny, tiny_base, w * t1 + (r - t0), waves * t1);
    else pull_items_body<W>(g, a, it, ipart, w * t2 + (r - t0 - t1), waves * t2);
}

__global__ void __launch_bounds__(AN_THREADS) k_pull_items_fin(DevGraph g, PullArgs a, Items it,
                                                               const float *__restrict__ ipart, uint32_t part_base) {
    __shared__ double red[AN_THREADS / 32];
    if (a.state[0]) return;
    double res = 0.0;
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < it.nmulti; m += gridDim.x * blockDim.x) {
        const uint32_t v = it.multi[m];
        float t = 0.f;
        for (uint32_t i = it.item_first[v]; i < it.item_first[v + 1]; ++i) t += ipart[i];
        pull_finish(a, v, t, g.vtx[v].z, res);
    }
    res = warp_sum(res);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = res;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < AN_THREADS / 32; ++i) s += red[i];
        a.partial[part_base + blockIdx.x] = s;
    }
}

// Sums the per-CTA residuals in a fixed order; latches convergence.
__global__ void k_iter_done(const double *__restrict__ partial, uint32_t nparts, float eps, int *state,
                            double *last_res) {
    __shared__ double red[32];
    if (state[0]) return;
    double t = 0.0;
    for (uint32_t i = threadIdx.x; i < nparts; i += blockDim.x) t += partial[i];
    t = warp_sum(t);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < (int)(blockDim.x / 32); ++i) s += red[i];
        *last_res = s;
        state[1] += 1;
        if (s < (double)eps) state[0] = 1;
    }
}

__global__ void k_fill_f32(float *x, uint32_t n, float val, uint32_t one_at, float one_val) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        x[v] = (v == one_at) ? one_val : val;
}

// contrib[u] = x[u] * scale(u), scale = 1/deg (PageRank) or 1/s_u (weighted)
__global__ void k_contrib(DevGraph g, const float *__restrict__ x, const float *__restrict__ rscale,
                          float *__restrict__ contrib) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < g.n; v += gridDim.x * blockDim.x) {
        if (rscale) contrib[v] = x[v] * rscale[v];
        else {
            const uint32_t d = g.vtx[v].z;
            contrib[v] = d ? x[v] / (float)d : 0.f;
        }
    }
}

// ------------------------------------------------------------ PR driver
struct IterBufs {
    float *x0, *x1, *c0, *c1;
    double *partial;
    int *state;  // [0] done, [1] sweeps
    double *res;
    uint32_t *heavy;
    unsigned long long *nheavy;  // [0] medium count, [1] hub count
    uint32_t *hubs;
};

size_t iter_bytes(uint32_t n, uint32_t parts) {
    return (size_t)n * 4 * 4 + (size_t)parts * 8 + 64 + (size_t)n * 4 * 2 + 64;
}

IterBufs carve_iter(void *base, uint32_t n, uint32_t parts) {
    char *p = static_cast<char *>(base);
    IterBufs b;
    b.x0 = (float *)p; p += (size_t)n * 4;
    b.x1 = (float *)p; p += (size_t)n * 4;
    b.c0 = (float *)p; p += (size_t)n * 4;
    b.c1 = (float *)p; p += (size_t)n * 4;
    b.partial = (double *)p; p += (size_t)parts * 8;
    b.state = (int *)p; p += 16;
    b.res = (double *)p; p += 16;
    b.nheavy = (unsigned long long *)p; p += 32;
    b.heavy = (uint32_t *)p; p += (size_t)n * 4;
    b.hubs = (uint32_t *)p;
    return b;
}

constexpr unsigned PULL_GRID = 148 * 8;
constexpr unsigned HUB_GRID = 148 * 2;

// Tier shares of a round from tier[] of k_item_count: the work of a tier is
// its entries plus a per-vertex cost (the record load, the dependent first
// block load and the finish) of 16 entries.  On R-MAT scale 22 this gives
// 3, 4 and 9 CTAs of 16 to the lane-group, thread-per-vertex and item tiers,
// the best of the splits measured (0.58 ms per sweep; equal thirds 0.69).  A
// tier with work gets at least one CTA per round; GV_SWEEP_SPLIT="a,b,c"
// overrides the split.
uint32_t sweep_split(const unsigned long long *tier) {
    if (const char *env = std::getenv("GV_SWEEP_SPLIT")) {  // "lane-group,tiny,items" CTAs per round
        unsigned x = 0, y = 0, z = 0;
        if (std::sscanf(env, "%u,%u,%u", &x, &y, &z) == 3 && x + y + z == SWEEP_PERIOD && x && y && z)
            return x | (y << 8) | (z << 16);
    }
    const double w[3] = {(double)tier[2] + 16.0 * tier[3], (double)tier[0] + 16.0 * tier[1], (double)tier[4]};
    const double tot = w[0] + w[1] + w[2];
    uint32_t t[3] = {0, 0, 0};
    if (tot <= 0) return 1u | (1u << 8) | (1u << 16);
    uint32_t sum = 0;
    for (int i = 0; i < 3; ++i) {
        t[i] = w[i] > 0 ? std::max<uint32_t>(1, (uint32_t)(SWEEP_PERIOD * w[i] / tot + 0.5)) : 0;
        sum += t[i];
    }
    // settle the rounding on the tier with the most CTAs
    int big = 0;
    for (int i = 1; i < 3; ++i)
        if (t[i] > t[big]) big = i;
    while (sum > SWEEP_PERIOD) { --t[big]; --sum; }
    while (sum < SWEEP_PERIOD) { ++t[big]; ++sum; }
    return t[0] | (t[1] << 8) | (t[2] << 16);
}

// Builds the chunked item list of the current graph (aux scratch slots 1, 2);
// *ipart gets one 4-byte slot per item.
gv_status build_items(gv_graph *g, cudaStream_t s, unsigned long long *nmulti, Items *it, float **ipart,
                      bool tiers = true) {
    DevGraph d = g->d;
    const uint32_t n = d.n;
    // first, multi, the two tier position arrays (n + 1 each), the two tier lists (n each), counters
    uint32_t *first = (uint32_t *)aux_scratch(g, 1, ((size_t)n + 1) * 4 * 4 + (size_t)n * 4 * 2 + 128);
    if (!first) return GV_ERR_NOMEM;
    uint32_t *multi = first + (n + 1);
    uint32_t *pl = multi + (n + 1), *pt = pl + (n + 1), *light = pt + (n + 1), *tiny = light + n;
    unsigned long long *tier = (unsigned long long *)(((uintptr_t)(tiny + n) + 7) & ~(uintptr_t)7);
    if (tiers) {  // the sweeps' tier lists (the triangle snapshot needs only the items)
        GV_LAUNCH(k_tier_flags, grid_for(n, 256), 256, 0, s, d, pl, pt);
        scan_exclusive_u32(pl, pl, n, pl + n, g->bs.scan_tmp, s);
        scan_exclusive_u32(pt, pt, n, pt + n, g->bs.scan_tmp, s);
        GV_LAUNCH(k_tier_lists, grid_for(n, 256), 256, 0, s, d, (const uint32_t *)pl, (const uint32_t *)pt, light, tiny);
    } else {
        cudaMemsetAsync(pl + n, 0, 4, s);
        cudaMemsetAsync(pt + n, 0, 4, s);
    }
    cudaMemsetAsync(nmulti, 0, 8, s);
    cudaMemsetAsync(tier, 0, 5 * 8, s);
    GV_LAUNCH(k_item_count, grid_for(n, 256), 256, 0, s, d, first, multi, nmulti, tier);
    scan_exclusive_u32(first, first, n, first + n, g->bs.scan_tmp, s);
    uint32_t nitems = 0, nl = 0, nt = 0;
    unsigned long long nm = 0, ht[5] = {0, 0, 0, 0, 0};
    cudaMemcpyAsync(&nitems, first + n, 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&nl, pl + n, 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&nt, pt + n, 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&nm, nmulti, 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(ht, tier, 5 * 8, cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "items");
    uint32_t *item_vertex = nullptr;
    float *ip = nullptr;
    if (nitems) {
        item_vertex = (uint32_t *)aux_scratch(g, 2, (size_t)nitems * 8);
        if (!item_vertex) return GV_ERR_NOMEM;
        ip = (float *)(item_vertex + nitems);
        GV_LAUNCH(k_item_fill, grid_for(n, 256), 256, 0, s, n, (const uint32_t *)first, item_vertex);
    }
    it->item_vertex = item_vertex;
    it->item_first = first;
    it->multi = multi;
    it->nitems = nitems;
    it->nmulti = (uint32_t)nm;
    it->light = light;
    it->tiny = tiny;
    it->nlight = nl;
    it->ntiny = nt;
    it->split = sweep_split(ht);
    *ipart = ip;
    return GV_OK;
}

// Runs pull sweeps until convergence or max_iter.  Result in *result (one of
// x0/x1).  `weighted_rscale` non-null selects the weighted gather (adjoint).
gv_status run_sweeps(gv_graph *g, cudaStream_t s, IterBufs &b, PullArgs proto, bool weighted,
                     const float *weighted_rscale, float eps, int max_iter, bool contrib_pr,
                     int *sweeps_out, float **result) {
    DevGraph d = g->d;
    Items it{};
    float *ipart = nullptr;
    gv_status st = build_items(g, s, b.nheavy, &it, &ipart);
    if (st != GV_OK) return st;
    cudaMemsetAsync(b.state, 0, 16, s);
    cudaError_t e = cudaSuccess;
    const uint32_t nparts = SWEEP_PARTS;
    cudaMemsetAsync(b.partial, 0, (size_t)nparts * 8, s);
    int h_state[2] = {0, 0};
    float *xa = b.x0, *xb = b.x1, *ca = b.c0, *cb = b.c1;
    int launched = 0;
    while (launched < max_iter) {
        const int chunk = std::min(8, max_iter - launched);
        for (int i = 0; i < chunk; ++i) {
            PullArgs a = proto;
            a.gather = contrib_pr ? ca : (weighted ? xa : ca);
            a.xold = xa;
            a.xnew = xb;
            a.contrib = contrib_pr ? cb : nullptr;
            a.partial = b.partial;
            a.state = b.state;
            if (!contrib_pr && !weighted) a.gather = ca;
            ProfScope ps(PROF_PULL, s);
            dispatch_tpv(g->cfg.threads_per_vertex, [&](auto t) {
                constexpr int T = decltype(t)::value;
                if (weighted)
                    GV_LAUNCH((k_pull_fused<T, true>), SWEEP_GRID, AN_THREADS, 0, s, d, a, it, ipart, SWEEP_GRID + FIN_GRID);
                else
                    GV_LAUNCH((k_pull_fused<T, false>), SWEEP_GRID, AN_THREADS, 0, s, d, a, it, ipart, SWEEP_GRID + FIN_GRID);
            });
            if (it.nitems)
                GV_LAUNCH(k_pull_items_fin, FIN_GRID, AN_THREADS, 0, s, d, a, it, (const float *)ipart, SWEEP_GRID);
            GV_LAUNCH(k_iter_done, 1, 256, 0, s, b.partial, nparts, eps, b.state, b.res);
            std::swap(xa, xb);
            std::swap(ca, cb);
        }
        launched += chunk;
        e = cudaMemcpyAsync(h_state, b.state, 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e, "sweeps");
        if (h_state[0]) break;
    }
    (void)weighted_rscale;
    *sweeps_out = h_state[1];
    // sweep i (1-based) wrote x1 when i is odd
    *result = (h_state[1] & 1) ? b.x1 : b.x0;
    return GV_OK;
}

gv_status copy_out_f32(const float *src, float *dst, uint32_t n, int mem, cudaStream_t s) {
    cudaError_t e = cudaMemcpyAsync(dst, src, (size_t)n * 4,
                                    mem == GV_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return cuda_status(e, "copy out");
}

gv_status transpose_pagerank(gv_graph *g, float alpha, float tol, int32_t max_iter, bool unit, const float *x_init,
                             int init_mem, uint32_t source, float *x_out, int32_t *sweeps, int mem, cudaStream_t s);

gv_status pagerank_impl(gv_graph *g, float alpha, float eps, int max_iter, const float *x_init, int init_mem,
                        uint32_t source, float *x_out, int32_t *sweeps, int mem, cudaStream_t s) {
    const uint32_t n = g->d.n;
    if (g->cfg.directed) {  // pull over the in-edges: the sorted transpose, unit weights
        int32_t sw = 0;
        gv_status st = transpose_pagerank(g, alpha, eps, max_iter, true, x_init, init_mem, source, x_out, &sw, mem, s);
        g->last_sweeps = sw;
        if (sweeps) *sweeps = sw;
        return st;
    }
    if (plan_pagerank_enabled(g)) {  // the degree-ordered sweep plan (prplan.cu)
        bool planned = false;
        gv_status st = plan_pagerank(g, alpha, eps, max_iter, x_init, init_mem, source, x_out, sweeps, mem, s,
                                     &planned);
        if (st != GV_OK || planned) return st;
    }
    const uint32_t parts = SWEEP_PARTS;
    void *buf = analytics_scratch(g, iter_bytes(n, parts));
    if (!buf) return GV_ERR_NOMEM;
    IterBufs b = carve_iter(buf, n, parts);
    DevGraph d = g->d;
    if (x_init) {
        cudaError_t e = cudaMemcpyAsync(b.x0, x_init, (size_t)n * 4,
                                        init_mem == GV_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return cuda_status(e, "pagerank init");
    } else if (source == GV_NIL) {
        GV_LAUNCH(k_fill_f32, grid_for(n, 256), 256, 0, s, b.x0, n, 1.0f / (float)n, GV_NIL, 0.f);
    } else {
        GV_LAUNCH(k_fill_f32, grid_for(n, 256), 256, 0, s, b.x0, n, 0.f, source, 1.f);
    }
    GV_LAUNCH(k_contrib, grid_for(n, 256), 256, 0, s, d, (const float *)b.x0, (const float *)nullptr, b.c0);
    PullArgs a{};
    a.alpha = alpha;
    if (source == GV_NIL) {
        a.base_all = (1.0f - alpha) / (float)n;
        a.base_src = GV_NIL;
    } else {
        a.base_all = 0.f;
        a.base_src = source;
        a.base_src_val = 1.0f - alpha;
    }
    int sw = 0;
    float *res = nullptr;
    gv_status st = run_sweeps(g, s, b, a, false, nullptr, eps, max_iter, true, &sw, &res);
    if (st != GV_OK) return st;
    g->last_sweeps = sw;
    if (sweeps) *sweeps = sw;
    return copy_out_f32(res, x_out, n, mem, s);
}

// ------------------------------------------------------------------- TC
// Orientation: u -> v iff (deg u, u) < (deg v, v).  Max out-degree <= sqrt(2m).
__device__ __forceinline__ bool rank_less(uint32_t du, uint32_t u, uint32_t dv, uint32_t v) {
    return du < dv || (du == dv && u < v);
}

// Light vertices (fill <= LIGHT_FILL) count their oriented out-degree with
// a lane group; heavier vertices go through the chunked items.
template <int TPV>
__global__ void __launch_bounds__(AN_THREADS) k_tc_outdeg(DevGraph g, const uint32_t *__restrict__ deg,
                                                          uint32_t *__restrict__ dplus) {
    constexpr int GPC = AN_THREADS / TPV;
    __shared__ uint32_t tabs[GPC][BIG_BLOCKS];
    Group<TPV> G;
    uint32_t *tab = tabs[threadIdx.x / TPV];
    const uint32_t ngroups = gridDim.x * GPC;
    for (uint32_t u = blockIdx.x * GPC + threadIdx.x / TPV; u < g.n; u += ngroups) {
        const uint4 rec = g.vtx[u];
        const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB), du = rec.z;
        if (fill > LIGHT_FILL) continue;  // k_tc_items / k_tc_multi
        fill_block_table(g, rec.x, 0, nb, tab, G.gl, TPV);
        G.sync();
        uint32_t c = 0;
        for (uint32_t e = G.gl; e < fill; e += TPV) {
            const uint32_t v = g.pool[((size_t)tab[e >> g.logB] << g.logB) + (e & (g.B - 1))];
            if (v != GV_TOMB && rank_less(du, u, __ldg(deg + v), v)) ++c;
        }
        G.sync();
        c = G.sum(c);
        if (G.gl == 0) dplus[u] = c;
    }
}

// One warp per item of a heavy vertex.  WRITE = false counts the item's
// oriented entries into icnt; WRITE = true writes them at off[u] + ioff[item].
template <bool WRITE>
__global__ void __launch_bounds__(AN_THREADS) k_tc_items(DevGraph g, const uint32_t *__restrict__ deg, Items it,
                                                         uint32_t *__restrict__ icnt, const uint32_t *__restrict__ ioff,
                                                         const unsigned long long *__restrict__ off,
                                                         uint32_t *__restrict__ snap) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t nw = gridDim.x * (AN_THREADS / 32);
    for (uint32_t i = blockIdx.x * (AN_THREADS / 32) + (threadIdx.x >> 5); i < it.nitems; i += nw) {
        const uint32_t u = it.item_vertex[i];
        const uint32_t c = i - it.item_first[u];
        const uint4 rec = g.vtx[u];
        const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB), du = rec.z;
        const uint32_t kb0 = c << 5;
        const uint32_t my_blk = item_block(g, rec, kb0, nb);
        const uint32_t e0 = kb0 << g.logB;
        const uint32_t e1 = min(fill, (kb0 + 32) << g.logB);
        const uint32_t nq = (e1 - e0 + 3) >> 2;
        unsigned long long w = WRITE ? off[u] + ioff[i] : 0ull;
        const unsigned long long wend = WRITE ? off[u + 1] : 0ull;
        uint32_t total = 0;
        for (uint32_t q0 = 0; q0 < nq; q0 += 32) {
            const uint32_t q = q0 + lane;
            const uint32_t el = q << 2;
            const uint32_t pb = __shfl_sync(GV_FULL_MASK, my_blk, (el >> g.logB) & 31u);
            uint32_t ev[4] = {GV_TOMB, GV_TOMB, GV_TOMB, GV_TOMB};
            uint32_t k = 0;
            if (q < nq) {
                const uint4 qv = *reinterpret_cast<const uint4 *>(g.pool + ((size_t)pb << g.logB) + (el & (g.B - 1)));
                ev[0] = qv.x; ev[1] = qv.y; ev[2] = qv.z; ev[3] = qv.w;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (e0 + el + j >= e1 || ev[j] == GV_TOMB || !rank_less(du, u, __ldg(deg + ev[j]), ev[j]))
                        ev[j] = GV_TOMB;
                    else
                        ++k;
                }
            }
            if (WRITE) {
                uint32_t incl = k;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t t = __shfl_up_sync(GV_FULL_MASK, incl, o);
                    if (lane >= (uint32_t)o) incl += t;
                }
                unsigned long long p = w + (incl - k);
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (ev[j] != GV_TOMB) {
                        if (p < wend) snap[p] = ev[j];
                        ++p;
                    }
                w += __shfl_sync(GV_FULL_MASK, incl, 31);
            } else {
                total += k;
            }
        }
        if (!WRITE) {
            total = warp_sum(total);
            if (lane == 0) icnt[i] = total;
        }
    }
}

// Heavy vertices: dplus = sum of their items' counts; ioff = item prefix.
__global__ void k_tc_multi(Items it, const uint32_t *__restrict__ icnt, uint32_t *__restrict__ ioff,
                           uint32_t *__restrict__ dplus) {
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < it.nmulti; m += gridDim.x * blockDim.x) {
        const uint32_t v = it.multi[m];
        uint32_t run = 0;
        for (uint32_t i = it.item_first[v]; i < it.item_first[v + 1]; ++i) {
            ioff[i] = run;
            run += icnt[i];
        }
        dplus[v] = run;
    }
}

// Light vertices write their oriented lists in storage order.
template <int TPV>
__global__ void __launch_bounds__(AN_THREADS) k_tc_write(DevGraph g, const uint32_t *__restrict__ deg,
                                                         const unsigned long long *__restrict__ off,
                                                         uint32_t *__restrict__ snap) {
    constexpr int GPC = AN_THREADS / TPV;
    __shared__ uint32_t tabs[GPC][BIG_BLOCKS];
    Group<TPV> G;
    uint32_t *tab = tabs[threadIdx.x / TPV];
    const uint32_t ngroups = gridDim.x * GPC;
    for (uint32_t u = blockIdx.x * GPC + threadIdx.x / TPV; u < g.n; u += ngroups) {
        const uint4 rec = g.vtx[u];
        const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB), du = rec.z;
        if (fill > LIGHT_FILL) continue;  // k_tc_items<true>
        unsigned long long w = off[u];
        const unsigned long long wend = off[u + 1];
        fill_block_table(g, rec.x, 0, nb, tab, G.gl, TPV);
        G.sync();
        for (uint32_t c0 = 0; c0 < fill; c0 += TPV) {
            const uint32_t e = c0 + G.gl;
            uint32_t v = GV_TOMB;
            if (e < fill) v = g.pool[((size_t)tab[e >> g.logB] << g.logB) + (e & (g.B - 1))];
            const uint32_t keep = (v != GV_TOMB && rank_less(du, u, __ldg(deg + v), v)) ? 1u : 0u;
            uint32_t tot;
            const uint32_t pre = G.excl_scan(keep, tot);
            if (keep && w + pre < wend) snap[w + pre] = v;
            w += tot;
        }
        G.sync();
    }
}

// Sorts tiny lists in place (one thread) and routes the rest to the sorts
// (cnts[0] mid lists, cnts[1] big lists, cnts[2] longest big list).  Lists
// of core vertices (core_of != GV_NIL) are read by no merge and stay as they
// are.
__global__ void k_tc_classify(const unsigned long long *__restrict__ off, uint32_t n, uint32_t *__restrict__ snap,
                              uint32_t *__restrict__ mid_list, uint32_t *__restrict__ big_list,
                              unsigned long long *cnts, const uint32_t *__restrict__ core_of) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
        if (core_of && core_of[u] != GV_NIL) continue;
        const uint32_t len = (uint32_t)(off[u + 1] - off[u]);
        if (len > 1024) {
            big_list[atomicAdd(&cnts[1], 1ull)] = u;
            atomicMax(&cnts[2], (unsigned long long)len);
        }
        else if (len > 16) mid_list[atomicAdd(&cnts[0], 1ull)] = u;
        else if (len > 1) {
            uint32_t *a = snap + off[u];
            for (uint32_t i = 1; i < len; ++i) {
                const uint32_t x = a[i];
                uint32_t j = i;
                while (j > 0 && a[j - 1] > x) { a[j] = a[j - 1]; --j; }
                a[j] = x;
            }
        }
    }
}

// Bitonic sort of a[0, len) using smem buffer s of size P (power of two >= len).
__device__ void smem_bitonic(uint32_t *a, uint32_t len, uint32_t *s, uint32_t P, uint32_t t, uint32_t nt,
                             bool warp_only) {
    for (uint32_t i = t; i < P; i += nt) s[i] = i < len ? a[i] : 0xFFFFFFFFu;
    if (warp_only) __syncwarp(); else __syncthreads();
    for (uint32_t k = 2; k <= P; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = t; i < P; i += nt) {
                const uint32_t ixj = i ^ j;
                if (ixj > i) {
                    const bool up = (i & k) == 0;
                    const uint32_t x = s[i], y = s[ixj];
                    if ((x > y) == up) { s[i] = y; s[ixj] = x; }
                }
            }
            if (warp_only) __syncwarp(); else __syncthreads();
        }
    }
    for (uint32_t i = t; i < len; i += nt) a[i] = s[i];
    if (warp_only) __syncwarp(); else __syncthreads();
}

__global__ void __launch_bounds__(AN_THREADS) k_tc_sort_mid(const unsigned long long *__restrict__ off,
                                                            uint32_t *__restrict__ snap,
                                                            const uint32_t *__restrict__ list,
                                                            const unsigned long long *cnt) {
    __shared__ uint32_t buf[AN_THREADS / 32][1024];
    const uint32_t nl = (uint32_t)cnt[0];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t nw = gridDim.x * (AN_THREADS / 32);
    for (uint32_t i = blockIdx.x * (AN_THREADS / 32) + warp; i < nl; i += nw) {
        const uint32_t u = list[i];
        const uint32_t len = (uint32_t)(off[u + 1] - off[u]);
        uint32_t P = 32;
        while (P < len) P <<= 1;
        smem_bitonic(snap + off[u], len, buf[warp], P, lane, 32, true);
    }
}

__global__ void __launch_bounds__(1024) k_tc_sort_big(const unsigned long long *__restrict__ off,
                                                      uint32_t *__restrict__ snap, const uint32_t *__restrict__ list,
                                                      const unsigned long long *cnt, uint32_t cap) {
    extern __shared__ uint32_t sbuf[];
    const uint32_t nl = (uint32_t)cnt[1];
    for (uint32_t i = blockIdx.x; i < nl; i += gridDim.x) {
        const uint32_t u = list[i];
        const uint32_t len = (uint32_t)(off[u + 1] - off[u]);
        uint32_t P = 1024;
        while (P < len) P <<= 1;
        if (P > cap) continue;  // cannot happen: cap is sized from the longest list
        smem_bitonic(snap + off[u], len, sbuf, P, threadIdx.x, blockDim.x, false);
    }
}

// Co-rank on diagonal d of merging A (ties first) and B.
__device__ __forceinline__ uint32_t corank(const uint32_t *A, uint32_t la, const uint32_t *B, uint32_t lb, uint32_t d) {
    uint32_t lo = d > lb ? d - lb : 0, hi = d < la ? d : la;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (A[mid] <= B[d - mid - 1]) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Group per oriented edge (u -> v): merge-path intersection of N+(u), N+(v).
// MODE TC_INCIDENT: credit all three vertices; TC_OWNER: credit the smallest
// id (the reference's owner, tc_kernel.cu:25-30); TC_TOTAL: only the sum is
// wanted, every triangle is credited to u (no per-vertex meaning).
template <int TPV, int MODE>
__global__ void __launch_bounds__(AN_THREADS) k_tc_count(const unsigned long long *__restrict__ off,
                                                         const uint32_t *__restrict__ snap,
                                                         const uint32_t *__restrict__ esrc, uint64_t m_plus,
                                                         unsigned long long *__restrict__ tcount,
                                                         unsigned long long *__restrict__ work,
                                                         const uint32_t *__restrict__ elist,
                                                         const uint32_t *__restrict__ ecount) {
    constexpr int GPC = AN_THREADS / TPV;
    constexpr uint32_t HT = 2048;  // per-CTA credit table: hubs collect many credits
    __shared__ unsigned long long wred[AN_THREADS / 32];
    __shared__ uint32_t ht_key[HT];
    __shared__ unsigned long long ht_val[HT];
    for (uint32_t i = threadIdx.x; i < HT; i += blockDim.x) {
        ht_key[i] = GV_NIL;
        ht_val[i] = 0;
    }
    __syncthreads();
    auto add = [&](uint32_t key, unsigned long long amount) {
        uint32_t h = (key * 2654435761u) & (HT - 1);
        for (int probe = 0; probe < 8; ++probe) {
            uint32_t k = ht_key[h];
            if (k == GV_NIL) k = atomicCAS(&ht_key[h], GV_NIL, key);
            if (k == GV_NIL || k == key) {
                atomicAdd(&ht_val[h], amount);
                return;
            }
            h = (h + 1) & (HT - 1);
        }
        atomicAdd(&tcount[key], amount);
    };
    Group<TPV> G;
    const uint64_t ngroups = (uint64_t)gridDim.x * GPC;
    unsigned long long my_work = 0;  // list entries this group touched
    // every oriented edge, or only those listed in elist[0, *ecount) (the
    // edges the core probes leave)
    const uint64_t nedges = elist ? (uint64_t)*ecount : m_plus;
    for (uint64_t i = (uint64_t)blockIdx.x * GPC + threadIdx.x / TPV; i < nedges; i += ngroups) {
        const uint64_t ei = elist ? (uint64_t)elist[i] : i;
        const uint32_t u = esrc[ei], v = snap[ei];
        const uint32_t *A = snap + off[u];
        const uint32_t la = (uint32_t)(off[u + 1] - off[u]);
        const uint32_t *Bv = snap + off[v];
        const uint32_t lb = (uint32_t)(off[v + 1] - off[v]);
        const uint32_t small = min(la, lb), large = max(la, lb);
        if (small == 0) continue;  // group-uniform
        uint32_t cu = 0, cv = 0;
        const uint32_t uv_min = min(u, v);
        auto credit = [&](uint32_t w) {
            if (MODE == TC_TOTAL) {
                ++cu;
            } else if (MODE == TC_INCIDENT) {
                ++cu; ++cv;
                add(w, 1ull);
            } else if (w < uv_min) {
                add(w, 1ull);
            } else if (u < v) {
                ++cu;
            } else {
                ++cv;
            }
        };
        const uint32_t lg = 32 - __clz(large);
        uint32_t touched;
        if ((uint64_t)small * (lg + 1) < (uint64_t)la + lb) {
            // skewed pair: binary-search each entry of the short list in the long one
            const bool a_small = la <= lb;
            const uint32_t *S = a_small ? A : Bv, *L = a_small ? Bv : A;
            for (uint32_t i = G.gl; i < small; i += TPV) {
                const uint32_t w = S[i];
                const uint32_t pos = lower_bound_u32(L, large, w);
                if (pos < large && L[pos] == w) credit(w);
            }
            touched = small * (lg + 1);
        } else {
            // balanced pair: merge path, one diagonal range per lane
            const uint32_t tot = la + lb;
            const uint32_t per = (tot + TPV - 1) / TPV;
            const uint32_t d0 = min(tot, G.gl * per), d1 = min(tot, d0 + per);
            uint32_t i = corank(A, la, Bv, lb, d0), j = d0 - i;
            auto ld = [](const uint32_t *X, uint32_t x, uint32_t len) {
                return x < len ? __ldg(X + x) : 0xFFFFFFFFu;
            };
            if (MODE == TC_TOTAL) {
                // the next four entries of each list sit in registers and the
                // load that refills a window is needed four steps later, so
                // steps do not wait on each other's loads (1.5x faster on
                // R-MAT scale 22; with per-vertex credits the branchy step
                // loses to the branch-free one below)
                uint32_t a0 = ld(A, i, la), a1 = ld(A, i + 1, la), a2 = ld(A, i + 2, la), a3 = ld(A, i + 3, la);
                uint32_t b0 = ld(Bv, j, lb), b1 = ld(Bv, j + 1, lb), b2 = ld(Bv, j + 2, lb), b3 = ld(Bv, j + 3, lb);
                for (uint32_t d = d0; d < d1; ++d) {
                    cu += (a0 == b0 && a0 != 0xFFFFFFFFu) ? 1u : 0u;
                    if (a0 <= b0) {  // ties consume A first
                        a0 = a1;
                        a1 = a2;
                        a2 = a3;
                        a3 = ld(A, i + 4, la);
                        ++i;
                    } else {
                        b0 = b1;
                        b1 = b2;
                        b2 = b3;
                        b3 = ld(Bv, j + 4, lb);
                        ++j;
                    }
                }
            } else {
                // branch-free merge step: lanes stay converged, only matches diverge
                uint32_t a = ld(A, i, la), bb = ld(Bv, j, lb);
                for (uint32_t d = d0; d < d1; ++d) {
                    const uint32_t ta = (a <= bb) ? 1u : 0u;  // ties consume A first
                    if (a == bb && a != 0xFFFFFFFFu) credit(a);
                    i += ta;
                    j += 1u - ta;
                    a = ld(A, i, la);
                    bb = ld(Bv, j, lb);
                }
            }
            touched = tot;
        }
        cu = G.sum(cu);
        cv = G.sum(cv);
        if (G.gl == 0) {
            if (cu) add(u, cu);
            if (cv) add(v, cv);
            my_work += touched;
        }
    }
    my_work = warp_sum(my_work);
    if ((threadIdx.x & 31) == 0) wred[threadIdx.x >> 5] = my_work;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int i = 0; i < AN_THREADS / 32; ++i) t += wred[i];
        if (t) atomicAdd(work, t);
    }
    for (uint32_t i = threadIdx.x; i < HT; i += blockDim.x)
        if (ht_key[i] != GV_NIL && ht_val[i]) atomicAdd(&tcount[ht_key[i]], ht_val[i]);
}

// ------------------------------------------------ dense-core bit probes
// Total-only counts split the oriented edges u -> v by whether v lies in the
// dense core K = {v : deg v > D}, D the smallest degree that leaves at most
// core_max vertices above it.  K is an upper set of the orientation order, so
// N+(v) lies inside K for every v in K and is kept as a bitmap row over core
// indices.  An edge into the core counts |N+(u) & N+(v)| by testing the core
// entries of N+(u) against v's row; a CTA stages one row in shared memory and
// streams the core lists of a chunk of v's in-neighbours, one bit test per
// entry.  On R-MAT graphs the core edges carry most of the merge work (a few
// thousand hub-to-hub lists of several hundred entries), and a bit test costs
// one shared-memory load where a merge step waits on the previous one; the
// edges outside the core keep the merge path.
constexpr uint32_t TCC_BINS = 65536;   // degree histogram; the last bin holds every degree above
constexpr uint32_t TCC_CHUNK = 256;    // in-neighbours of one core vertex per work item
constexpr uint32_t TCC_THREADS = 256;
constexpr uint32_t TCC_DEFAULT = 65504;  // default core size bound
constexpr uint32_t TCC_MAX = 65504;      // core indices stay below TCC_DEAD
constexpr uint16_t TCC_DEAD = 0xFFFF;    // list padding: a bit no row sets
constexpr uint32_t TCC_SROW = 2048;      // staged row words (holds TCC_DEAD's word)
constexpr int TCC_UNROLL = 4;            // 16-byte loads in flight per lane

struct TcCore {
    uint32_t *hist;                 // [TCC_BINS]
    uint32_t *cidx;                 // [n] core index or GV_NIL
    uint32_t *ccnt;                 // [n] core entries of N+(u); then write cursors
    unsigned long long *coff;       // [n + 1]
    uint32_t *icnt;                 // [cmax + 1] in-neighbours per core vertex; then cursors
    unsigned long long *ioff;       // [cmax + 1]
    uint32_t *itcnt;                // [cmax + 1] work items per core vertex
    uint32_t *itoff;                // [cmax + 1]
    uint32_t *itc;                  // [items] core vertex of each work item
    uint32_t *rows;                 // [cmax][wmax] bitmap rows
    uint16_t *clist;                // core entries of every N+(u) as core indices, each list padded
                                    // with TCC_DEAD to a multiple of 8 (16-byte aligned starts)
    uint32_t *inl;                  // [m+] in-neighbours of every core vertex
    uint32_t *ctl;                  // [0] D (GV_NIL: no core), [1] core size, [2] rest edges
    uint32_t *rest;                 // [m+] oriented edges outside the core, for the merge
    uint32_t cmax, wmax;
};

// Degree histogram, lanes with the same bin merged before the atomic.
__global__ void k_tcc_hist(const uint32_t *__restrict__ deg, uint32_t n, uint32_t *__restrict__ hist) {
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t v = base + threadIdx.x;
        const uint32_t bin = v < n ? min(deg[v], TCC_BINS - 1) : GV_NIL;
        const uint32_t peers = __match_any_sync(GV_FULL_MASK, bin);
        if (bin != GV_NIL && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&hist[bin], __popc(peers));
    }
}

// One CTA of 1024 threads: D = the smallest d <= TCC_BINS - 2 with
// #{v : deg v > d} <= cmax (ctl[0]; GV_NIL when there is none or nothing
// lies above it).  Thread t owns bins [PER r, PER (r + 1)), r = 1023 - t, so
// the exclusive scan over threads counts the vertices in the bins above.
__global__ void __launch_bounds__(1024) k_tcc_pick(const uint32_t *__restrict__ hist, uint32_t cmax,
                                                   uint32_t *__restrict__ ctl) {
    constexpr uint32_t PER = TCC_BINS / 1024;
    __shared__ unsigned long long wtot[33];
    __shared__ unsigned long long best;  // (d << 32) | #{deg > d}: the smallest valid d wins
    const uint32_t t = threadIdx.x, r = 1023 - t;
    if (t == 0) best = ~0ull;
    unsigned long long local = 0;
    for (uint32_t i = 0; i < PER; ++i) local += hist[PER * r + i];
    unsigned long long tot;
    unsigned long long s = cta_excl_scan<unsigned long long, 1024>(local, wtot, tot);  // #{deg > last bin of r}
    unsigned long long mine = ~0ull;
    for (int i = (int)PER - 1; i >= 0; --i) {
        const uint32_t d = PER * r + (uint32_t)i;
        if (d <= TCC_BINS - 2 && s <= cmax) mine = ((unsigned long long)d << 32) | s;
        s += hist[d];
    }
    if (mine != ~0ull) atomicMin(&best, mine);
    __syncthreads();
    if (t == 0) {
        const bool ok = best != ~0ull && (uint32_t)best != 0;
        ctl[0] = ok ? (uint32_t)(best >> 32) : GV_NIL;
        ctl[1] = 0;
        ctl[2] = 0;
    }
}

// Core indices (warp-aggregated; the order does not change any count).
__global__ void k_tcc_index(const uint32_t *__restrict__ deg, uint32_t n, uint32_t *__restrict__ ctl,
                            uint32_t *__restrict__ cidx) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t D = ctl[0];
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t v = base + threadIdx.x;
        const bool in = v < n && D != GV_NIL && deg[v] > D;
        const uint32_t bal = __ballot_sync(GV_FULL_MASK, in);
        uint32_t b0 = 0;
        if (lane == 0 && bal) b0 = atomicAdd(&ctl[1], __popc(bal));
        b0 = __shfl_sync(GV_FULL_MASK, b0, 0);
        if (v < n) cidx[v] = in ? b0 + __popc(bal & ((1u << lane) - 1u)) : GV_NIL;
    }
}

// Per oriented edge u -> w with w in the core: one more core entry of u and
// one more in-neighbour of w; every other edge goes to the merge list.
__global__ void k_tcc_count(const uint32_t *__restrict__ snap, const uint32_t *__restrict__ esrc, uint64_t m_plus,
                            const uint32_t *__restrict__ cidx, uint32_t *__restrict__ ccnt,
                            uint32_t *__restrict__ icnt, uint32_t *__restrict__ rest, uint32_t *__restrict__ nrest) {
    const uint32_t lane = threadIdx.x & 31u;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < m_plus; base += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t e = base + threadIdx.x;
        uint32_t c = GV_NIL, u = GV_NIL;
        if (e < m_plus) {
            c = cidx[snap[e]];
            if (c != GV_NIL) u = esrc[e];
        }
        const uint32_t br = __ballot_sync(GV_FULL_MASK, e < m_plus && c == GV_NIL);
        uint32_t r0 = 0;
        if (lane == 0 && br) r0 = atomicAdd(nrest, __popc(br));
        r0 = __shfl_sync(GV_FULL_MASK, r0, 0);
        if (e < m_plus && c == GV_NIL) rest[r0 + __popc(br & ((1u << lane) - 1u))] = (uint32_t)e;
        const uint32_t pc = __match_any_sync(GV_FULL_MASK, c);
        if (c != GV_NIL && lane == (uint32_t)(__ffs(pc) - 1)) atomicAdd(&icnt[c], __popc(pc));
        const uint32_t pu = __match_any_sync(GV_FULL_MASK, u);
        if (u != GV_NIL && lane == (uint32_t)(__ffs(pu) - 1)) atomicAdd(&ccnt[u], __popc(pu));
    }
}

// Fills the core lists, the in-neighbour lists and the bitmap rows.
__global__ void k_tcc_fill(const uint32_t *__restrict__ snap, const uint32_t *__restrict__ esrc, uint64_t m_plus,
                           TcCore k) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t below = (1u << lane) - 1u;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < m_plus; base += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t e = base + threadIdx.x;
        uint32_t c = GV_NIL, u = GV_NIL;
        if (e < m_plus) {
            c = k.cidx[snap[e]];
            if (c != GV_NIL) u = esrc[e];
        }
        const uint32_t pc = __match_any_sync(GV_FULL_MASK, c);
        const uint32_t pu = __match_any_sync(GV_FULL_MASK, u);
        const uint32_t lc = (uint32_t)(__ffs(pc) - 1), lu = (uint32_t)(__ffs(pu) - 1);
        uint32_t bc = 0, bu = 0;
        if (c != GV_NIL && lane == lc) bc = atomicAdd(&k.icnt[c], __popc(pc));
        if (u != GV_NIL && lane == lu) bu = atomicAdd(&k.ccnt[u], __popc(pu));
        bc = __shfl_sync(GV_FULL_MASK, bc, lc);
        bu = __shfl_sync(GV_FULL_MASK, bu, lu);
        if (c == GV_NIL) continue;
        k.inl[k.ioff[c] + bc + __popc(pc & below)] = u;
        k.clist[k.coff[u] + bu + __popc(pu & below)] = (uint16_t)c;
        const uint32_t cu = k.cidx[u];
        if (cu != GV_NIL) atomicOr(&k.rows[(size_t)cu * k.wmax + (c >> 5)], 1u << (c & 31));
    }
}

// Core list lengths rounded up to a multiple of 8 entries.
__global__ void k_tcc_pad(uint32_t *__restrict__ ccnt, uint32_t n) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x)
        ccnt[u] = (ccnt[u] + 7u) & ~7u;
}

__global__ void k_tcc_items(const unsigned long long *__restrict__ ioff, uint32_t cmax, uint32_t *__restrict__ itcnt) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < cmax; c += gridDim.x * blockDim.x)
        itcnt[c] = (uint32_t)((ioff[c + 1] - ioff[c] + TCC_CHUNK - 1) / TCC_CHUNK);
}

// itc[i] = the core vertex of work item i (a warp per core vertex).
__global__ void k_tcc_item_owner(const uint32_t *__restrict__ itoff, uint32_t cmax, uint32_t *__restrict__ itc) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < cmax; c += nw)
        for (uint32_t i = itoff[c] + lane; i < itoff[c + 1]; i += 32) itc[i] = c;
}

// Reorders each core list so the probe's shared-memory loads meet distinct
// banks.  The probe's lanes read consecutive 8-entry rows of a list, and the
// t-th load of every lane reads column t; so the entries are put in
// round-robin order over their banks ((x >> 5) mod 32: first entry of each
// bank, then second, ...) and that sequence fills the list column by column.
// Consecutive rows of a column then hold entries of consecutive banks.
// Lists of one row, or longer than TCC_COLOR_MAX, keep their order (the
// counts never depend on it).
constexpr uint32_t TCC_COLOR_MAX = 2048;
constexpr uint32_t TCC_COLOR_J = 128;  // deepest bank rank handled; deeper lists keep their order
__global__ void __launch_bounds__(256) k_tcc_color(TcCore k, uint32_t n) {
    extern __shared__ uint16_t cbuf[];  // [8 warps][TCC_COLOR_MAX]
    __shared__ uint32_t hist[8][32], cur[8][32], tabM[8][TCC_COLOR_J], tabS[8][TCC_COLOR_J];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint16_t *out = cbuf + warp * TCC_COLOR_MAX;
    // the warp looks at 32 vertices at a time and reorders those with more than one row
    for (uint32_t u0 = (blockIdx.x * 8 + warp) * 32; u0 < n; u0 += gridDim.x * 8 * 32) {
        const uint32_t um = u0 + lane;
        uint32_t Lm = 0;
        unsigned long long am = 0;
        if (um < n) {
            am = k.coff[um];
            Lm = (uint32_t)(k.coff[um + 1] - am);
        }
        uint32_t todo = __ballot_sync(GV_FULL_MASK, Lm > 8 && Lm <= TCC_COLOR_MAX);
        while (todo) {
            const uint32_t t = __ffs(todo) - 1;
            todo &= todo - 1;
            const uint32_t L = __shfl_sync(GV_FULL_MASK, Lm, t);  // a multiple of 8
            const unsigned long long a = __shfl_sync(GV_FULL_MASK, am, t);
            uint16_t *cl = k.clist + a;
            hist[warp][lane] = 0;
            cur[warp][lane] = 0;
            __syncwarp();
            for (uint32_t i = lane; i < L; i += 32) atomicAdd(&hist[warp][(cl[i] >> 5) & 31u], 1u);
            __syncwarp();
            // lane = bank: M_j = banks with more than j entries, S_j = entries of ranks below j
            const uint32_t c = hist[warp][lane];
            uint32_t jmax = c;
#pragma unroll
            for (int o = 16; o; o >>= 1) jmax = max(jmax, __shfl_xor_sync(GV_FULL_MASK, jmax, o));
            if (jmax > TCC_COLOR_J) continue;  // warp-uniform
            uint32_t S = 0;
            for (uint32_t j = 0; j < jmax; ++j) {
                const uint32_t M = __ballot_sync(GV_FULL_MASK, c > j);
                if (lane == 0) {
                    tabM[warp][j] = M;
                    tabS[warp][j] = S;
                }
                S += __popc(M);
            }
            __syncwarp();
            const uint32_t R = L >> 3;
            for (uint32_t i = lane; i < L; i += 32) {
                const uint16_t x = cl[i];
                const uint32_t b = (x >> 5) & 31u;
                const uint32_t j = atomicAdd(&cur[warp][b], 1u);  // rank within its bank
                const uint32_t o = tabS[warp][j] + __popc(tabM[warp][j] & ((1u << b) - 1u));
                out[(o % R) * 8 + o / R] = x;
            }
            __syncwarp();
            for (uint32_t i = lane; i < L; i += 32) cl[i] = out[i];
            __syncwarp();
        }
    }
}

// Bit tests of eight core entries (one 16-byte load) against the staged row.
__device__ __forceinline__ uint32_t tcc_probe8(const uint32_t *srow, uint4 q) {
    uint32_t h = 0;
    const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const uint32_t lo = w[i] & 0xFFFFu, hi = w[i] >> 16;
        h += (srow[lo >> 5] >> (lo & 31)) & 1u;
        h += (srow[hi >> 5] >> (hi & 31)) & 1u;
    }
    return h;
}

// Work item = up to TCC_CHUNK in-neighbours u of one core vertex v: the CTA
// stages v's row, each warp fetches the list heads of its 32 u's at once (one
// per lane) and walks their lists as one run of 16-byte chunks (eight
// entries each), several loads per lane in flight.  Every triangle u < v < w
// (orientation order) with v in the core is counted here once.
static_assert(TCC_CHUNK == 32 * (TCC_THREADS / 32), "a warp takes one in-neighbour per lane");
__global__ void __launch_bounds__(TCC_THREADS) k_tcc_probe(TcCore k, unsigned long long *__restrict__ total,
                                                           unsigned long long *__restrict__ work) {
    __shared__ uint32_t srow[TCC_SROW];
    __shared__ unsigned long long wred[TCC_THREADS / 32][2];
    constexpr uint32_t NWARP = TCC_THREADS / 32;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t nitems = k.itoff[k.cmax];
    const uint32_t W = (k.ctl[1] + 31) >> 5;  // < TCC_SROW: the padding bit's word stays 0
    for (uint32_t i = W + threadIdx.x; i < TCC_SROW; i += TCC_THREADS) srow[i] = 0;
    unsigned long long cnt = 0, probes = 0;
    for (uint32_t item = blockIdx.x; item < nitems; item += gridDim.x) {
        const uint32_t c = k.itc[item];
        const unsigned long long j0 = k.ioff[c] + (unsigned long long)(item - k.itoff[c]) * TCC_CHUNK;
        const unsigned long long j1 = min(k.ioff[c + 1], j0 + TCC_CHUNK);
        // list heads of this warp's in-neighbours j0 + warp + NWARP t, t = lane
        const unsigned long long jj = j0 + warp + (unsigned long long)NWARP * lane;
        unsigned long long head = 0;
        uint32_t len = 0;
        if (jj < j1) {
            const uint32_t u = k.inl[jj];
            head = k.coff[u];
            len = (uint32_t)(k.coff[u + 1] - head);
        }
        __syncthreads();
        const uint32_t *row = k.rows + (size_t)c * k.wmax;
        for (uint32_t i = threadIdx.x; i < W; i += TCC_THREADS) srow[i] = row[i];
        __syncthreads();
        // the warp's 32 lists as one run of 16-byte chunks: chunk q belongs to
        // the lane t with pre_t <= q < pre_t + len_t / 8, so TCC_UNROLL loads
        // per lane stay in flight across list boundaries
        const uint32_t nq = len >> 3;
        uint32_t incl = nq;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(GV_FULL_MASK, incl, o);
            if (lane >= (uint32_t)o) incl += y;
        }
        const uint32_t pre = incl - nq, Q = __shfl_sync(GV_FULL_MASK, incl, 31);
        // chunk q of the run is chunk base_t + q of the list array (mod 2^32:
        // the list array holds fewer than 2^32 chunks)
        const uint32_t base = (uint32_t)(head >> 3) - pre;
        const uint4 *clist4 = reinterpret_cast<const uint4 *>(k.clist);
        uint32_t hits = 0;
        for (uint32_t q0 = 0; q0 < Q; q0 += 32 * TCC_UNROLL) {
            uint4 v[TCC_UNROLL];
#pragma unroll
            for (int r = 0; r < TCC_UNROLL; ++r) {
                const uint32_t q = q0 + 32u * r + lane;
                uint32_t t = 0;  // owner lane: the last with pre_t <= q
#pragma unroll
                for (uint32_t step = 16; step; step >>= 1) {
                    const uint32_t pc = __shfl_sync(GV_FULL_MASK, pre, t + step);
                    if (pc <= q) t += step;
                }
                const uint32_t bt = __shfl_sync(GV_FULL_MASK, base, t);
                v[r] = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);  // eight TCC_DEAD entries
                if (q < Q) v[r] = __ldg(clist4 + (bt + q));
            }
#pragma unroll
            for (int r = 0; r < TCC_UNROLL; ++r) hits += tcc_probe8(srow, v[r]);
        }
        const uint32_t seen = Q * 8;
        cnt += hits;
        probes += seen;  // the same in every lane of the warp
    }
    cnt = warp_sum(cnt);
    if (lane == 0) {
        wred[warp][0] = cnt;
        wred[warp][1] = probes;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0, p = 0;
        for (uint32_t i = 0; i < NWARP; ++i) {
            t += wred[i][0];
            p += wred[i][1];
        }
        if (t) atomicAdd(total, t);
        if (p) atomicAdd(work, p);
    }
}

// ------------------------------------------------ hash-probe intersection
// u-centric: N+(u) goes into a shared-memory hash set; every v in N+(u)
// streams N+(v) with coalesced loads and probes the set, so each entry costs
// one independent probe instead of a dependent merge step.  Pairs where
// N+(v) is much longer than N+(u) binary-search N+(u)'s entries in N+(v).
constexpr uint32_t TC_WARP_TAB = 512;  // per-warp set: N+(u) up to 256 entries
constexpr uint32_t TC_CREDIT_HT = 2048;

struct TcCredit {
    uint32_t *key;
    unsigned long long *val;
    unsigned long long *global;
    __device__ __forceinline__ void add(uint32_t k, unsigned long long amount) {
        uint32_t h = (k * 2654435761u) & (TC_CREDIT_HT - 1);
        for (int probe = 0; probe < 8; ++probe) {
            uint32_t cur = key[h];
            if (cur == GV_NIL) cur = atomicCAS(&key[h], GV_NIL, k);
            if (cur == GV_NIL || cur == k) {
                atomicAdd(&val[h], amount);
                return;
            }
            h = (h + 1) & (TC_CREDIT_HT - 1);
        }
        atomicAdd(&global[k], amount);
    }
    __device__ __forceinline__ void flush() {
        for (uint32_t i = threadIdx.x; i < TC_CREDIT_HT; i += blockDim.x)
            if (key[i] != GV_NIL && val[i]) atomicAdd(&global[key[i]], val[i]);
    }
};

// Multiplicative hash taking the high bits of the product (the low bits of
// x * odd depend only on the low bits of x and cluster sorted id lists).
__device__ __forceinline__ uint32_t tc_hash(uint32_t x, uint32_t mask) {
    return (uint32_t)(((unsigned long long)(x * 2654435761u) * (mask + 1ull)) >> 32);
}

// Callers size the table to at least twice the entries, so a free slot is
// always found; the probe count is bounded by the table size regardless.
__device__ __forceinline__ void set_insert(uint32_t *tab, uint32_t mask, uint32_t x) {
    uint32_t h = tc_hash(x, mask);
    for (uint32_t p = 0; p <= mask; ++p) {
        const uint32_t old = atomicCAS(&tab[h], GV_NIL, x);
        if (old == GV_NIL || old == x) return;
        h = (h + 1) & mask;
    }
}

// Membership in a hash set (mask != 0) or in a sorted array of `mask_or_len`
// entries (sorted == true).
__device__ __forceinline__ bool set_has(const uint32_t *tab, uint32_t mask, uint32_t x, bool sorted) {
    if (sorted) {
        const uint32_t pos = lower_bound_u32(tab, mask, x);
        return pos < mask && tab[pos] == x;
    }
    uint32_t h = tc_hash(x, mask);
    for (uint32_t p = 0; p <= mask; ++p) {
        const uint32_t k = tab[h];
        if (k == x) return true;
        if (k == GV_NIL) return false;
        h = (h + 1) & mask;
    }
    return false;
}

// ------------------------------------ packed hash-probe intersection
// (GV_TC_PACKED=1; on R-MAT scale 22 it reads 26% fewer list entries than the
// merge path but takes 1.8x longer: each probe is a random shared-memory
// access with a few slots of linear probing, where a merge step reads the
// next cached entry)
// u-centric: N+(u) goes into a hash set in shared memory; the lists N+(v),
// v in N+(u), are streamed as one concatenated run, 32 entries per warp step
// (one entry per lane, several short lists per step), each entry one probe
// of the set.  Work: sum_v d-(v) d+(v) probes + sum_u d+(u) inserts, against
// sum over oriented edges of d+(u) + d+(v) merge steps for the merge path
// (about 1.6x more on R-MAT), and the lists need no sorting.  Lane j of a
// step finds its list from the start offsets of the next 32 lists: one OR
// reduction of start bits and a popcount.
constexpr uint32_t TCP_LIGHT = 128;            // d+(u) handled by one warp
constexpr uint32_t TCP_WSET = 2 * TCP_LIGHT;   // per-warp set slots
constexpr int TCP_THREADS = 512;
constexpr int TCP_WARPS = TCP_THREADS / 32;
constexpr uint32_t TCP_CHUNK = 2048;           // lists per CTA step (heavy u)
constexpr uint32_t TCP_SSET = 8192;            // shared set slots of the heavy kernel

struct TcpWarp {
    uint32_t set[TCP_WSET];
    uint32_t vl[TCP_LIGHT];
    unsigned long long base[TCP_LIGHT];
    uint32_t pref[TCP_LIGHT + 1];
};

template <int MODE>
__device__ __forceinline__ void tcp_credit(TcCredit &cr, uint32_t u, uint32_t v, uint32_t w, uint32_t &cu) {
    if (MODE == TC_TOTAL) {
        ++cu;
    } else if (MODE == TC_INCIDENT) {
        ++cu;
        cr.add(v, 1ull);
        cr.add(w, 1ull);
    } else {
        const uint32_t m = min(u, min(v, w));
        if (m == u) ++cu;
        else cr.add(m, 1ull);
    }
}

// One step of 32 positions [p0, p0 + 32) of the concatenated lists of N+(v):
// list j covers positions [pref[j], pref[j + 1]), entry p of it sits at
// snap[base[j] + p].  j0 = the list holding p0.  Returns the list holding
// p0 + 32.
template <int MODE>
__device__ __forceinline__ uint32_t tcp_step(const uint32_t *__restrict__ snap, const uint32_t *set, uint32_t mask,
                                             const uint32_t *vl, const unsigned long long *base, const uint32_t *pref,
                                             uint32_t nv, uint32_t T, uint32_t p0, uint32_t j0, uint32_t u,
                                             TcCredit &cr, uint32_t &cu) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t S = (j0 + lane < nv) ? pref[j0 + lane] : 0xFFFFFFFFu;
    const uint32_t rel = S - p0;
    const uint32_t F = __reduce_or_sync(GV_FULL_MASK, rel < 32u ? (1u << rel) : 0u);
    const uint32_t G = F & ~1u;  // lists starting after p0 inside the step
    const uint32_t lm = lane == 31 ? 0xFFFFFFFFu : ((2u << lane) - 1u);
    const uint32_t j = j0 + __popc(G & lm);
    const uint32_t p = p0 + lane;
    if (p < T) {
        const uint32_t w = __ldg(snap + (base[j] + p));
        if (set_has(set, mask, w, false)) tcp_credit<MODE>(cr, u, vl[j], w, cu);
    }
    const uint32_t jl = j0 + __popc(G);
    return (jl + 1 <= nv && pref[jl + 1] <= p0 + 32) ? jl + 1 : jl;
}

// Compacts the lists v = A[i] (i in [i0, i0 + 32)) with d+(v) > 0 into
// vl / base / pref at nv, running total T (one warp); inserts v into `set`
// when it is given.
__device__ __forceinline__ void tcp_gather32(const unsigned long long *__restrict__ off, const uint32_t *A, uint32_t la,
                                             uint32_t i0, uint32_t *vl, unsigned long long *base, uint32_t *pref,
                                             uint32_t &nv, uint32_t &T, uint32_t *set, uint32_t mask) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t i = i0 + lane;
    uint32_t v = GV_NIL, dv = 0;
    unsigned long long ov = 0;
    if (i < la) {
        v = A[i];
        if (set) set_insert(set, mask, v);
        ov = off[v];
        dv = (uint32_t)(off[v + 1] - ov);
    }
    const bool keep = dv > 0;
    const uint32_t bal = __ballot_sync(GV_FULL_MASK, keep);
    uint32_t incl = dv;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(GV_FULL_MASK, incl, o);
        if (lane >= (uint32_t)o) incl += t;
    }
    const uint32_t tot = __shfl_sync(GV_FULL_MASK, incl, 31);
    if (keep) {
        const uint32_t pos = nv + __popc(bal & ((1u << lane) - 1u));
        const uint32_t start = T + incl - dv;
        vl[pos] = v;
        pref[pos] = start;
        base[pos] = ov - start;
    }
    nv += __popc(bal);
    T += tot;
}

template <int MODE>
__global__ void __launch_bounds__(TCP_THREADS) k_tcp_light(const unsigned long long *__restrict__ off,
                                                           const uint32_t *__restrict__ snap, uint32_t n,
                                                           unsigned long long *__restrict__ tcount,
                                                           unsigned long long *__restrict__ work) {
    extern __shared__ unsigned char tcp_dyn[];
    TcpWarp *ws = reinterpret_cast<TcpWarp *>(tcp_dyn);
    uint32_t *ck = reinterpret_cast<uint32_t *>(ws + TCP_WARPS);
    unsigned long long *cval = reinterpret_cast<unsigned long long *>(ck + TC_CREDIT_HT);
    __shared__ unsigned long long wred[TCP_WARPS];
    for (uint32_t i = threadIdx.x; i < TC_CREDIT_HT; i += blockDim.x) {
        ck[i] = GV_NIL;
        cval[i] = 0;
    }
    __syncthreads();
    TcCredit cr{ck, cval, tcount};
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    TcpWarp &W = ws[warp];
    unsigned long long my_work = 0;
    const uint32_t nw = gridDim.x * TCP_WARPS;
    for (uint32_t u = blockIdx.x * TCP_WARPS + warp; u < n; u += nw) {
        const unsigned long long ou = off[u];
        const uint32_t la = (uint32_t)(off[u + 1] - ou);
        if (la < 2 || la > TCP_LIGHT) continue;  // < 2: no triangle has u lowest; > TCP_LIGHT: k_tcp_heavy
        const uint32_t *A = snap + ou;
        uint32_t cap = 32;
        while (cap < 2 * la) cap <<= 1;
        const uint32_t mask = cap - 1;
        for (uint32_t i = lane; i < cap; i += 32) W.set[i] = GV_NIL;
        __syncwarp();
        uint32_t nv = 0, T = 0;
        for (uint32_t i0 = 0; i0 < la; i0 += 32) tcp_gather32(off, A, la, i0, W.vl, W.base, W.pref, nv, T, W.set, mask);
        if (lane == 0) W.pref[nv] = T;
        __syncwarp();
        uint32_t cu = 0, j0 = 0;
        for (uint32_t p0 = 0; p0 < T; p0 += 32)
            j0 = tcp_step<MODE>(snap, W.set, mask, W.vl, W.base, W.pref, nv, T, p0, j0, u, cr, cu);
        cu = warp_sum(cu);
        if (lane == 0) {
            if (cu) cr.add(u, cu);
            my_work += (unsigned long long)T + la;
        }
        __syncwarp();
    }
    if (lane == 0) wred[warp] = my_work;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int i = 0; i < TCP_WARPS; ++i) t += wred[i];
        if (t) atomicAdd(work, t);
    }
    cr.flush();
}

// Vertices with d+(u) > TCP_LIGHT into list; cnt[1] = the longest d+.
__global__ void k_tcp_heavy_list(const unsigned long long *__restrict__ off, uint32_t n, uint32_t *__restrict__ list,
                                 unsigned long long *cnt) {
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t u = base + threadIdx.x;
        uint32_t la = 0;
        if (u < n) la = (uint32_t)(off[u + 1] - off[u]);
        const bool heavy = la > TCP_LIGHT;
        const uint32_t bal = __ballot_sync(GV_FULL_MASK, heavy);
        unsigned long long at = 0;
        if (lane == 0 && bal) at = atomicAdd(cnt, (unsigned long long)__popc(bal));
        at = __shfl_sync(GV_FULL_MASK, at, 0);
        if (heavy) {
            list[at + __popc(bal & ((1u << lane) - 1u))] = u;
            atomicMax(cnt + 1, (unsigned long long)la);
        }
    }
}

// One CTA per heavy u: the set of N+(u) in shared memory (global, per CTA,
// above TCP_SSET / 2 entries); lists in chunks of TCP_CHUNK, warps over steps.
template <int MODE>
__global__ void __launch_bounds__(TCP_THREADS) k_tcp_heavy(const unsigned long long *__restrict__ off,
                                                           const uint32_t *__restrict__ snap,
                                                           unsigned long long *__restrict__ tcount,
                                                           const uint32_t *__restrict__ list,
                                                           const unsigned long long *cnt, uint32_t *__restrict__ gset,
                                                           uint32_t gcap, unsigned long long *__restrict__ work) {
    extern __shared__ unsigned char tcp_dyn[];
    uint32_t *sset = reinterpret_cast<uint32_t *>(tcp_dyn);
    uint32_t *vl = sset + TCP_SSET;
    unsigned long long *base = reinterpret_cast<unsigned long long *>(vl + TCP_CHUNK);
    uint32_t *pref = reinterpret_cast<uint32_t *>(base + TCP_CHUNK);
    uint32_t *ck = pref + TCP_CHUNK + 32;
    unsigned long long *cval = reinterpret_cast<unsigned long long *>(ck + TC_CREDIT_HT);
    __shared__ uint32_t s_nv, s_T;
    __shared__ uint32_t wsum[TCP_WARPS], wcnt[TCP_WARPS], cured[TCP_WARPS];
    __shared__ unsigned long long wred[TCP_WARPS];
    for (uint32_t i = threadIdx.x; i < TC_CREDIT_HT; i += blockDim.x) {
        ck[i] = GV_NIL;
        cval[i] = 0;
    }
    __syncthreads();
    TcCredit cr{ck, cval, tcount};
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t nh = (uint32_t)cnt[0];
    unsigned long long my_work = 0;
    for (uint32_t hi = blockIdx.x; hi < nh; hi += gridDim.x) {
        const uint32_t u = list[hi];
        const unsigned long long ou = off[u];
        const uint32_t la = (uint32_t)(off[u + 1] - ou);
        const uint32_t *A = snap + ou;
        uint32_t cap = 1024;
        while (cap < 2 * la) cap <<= 1;
        uint32_t *set = cap <= TCP_SSET ? sset : gset + (size_t)blockIdx.x * gcap;
        const uint32_t mask = cap - 1;
        for (uint32_t i = threadIdx.x; i < cap; i += blockDim.x) set[i] = GV_NIL;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < la; i += blockDim.x) set_insert(set, mask, A[i]);
        __syncthreads();
        uint32_t cu = 0;
        for (uint32_t c0 = 0; c0 < la; c0 += TCP_CHUNK) {
            const uint32_t cn = min(TCP_CHUNK, la - c0);
            // pass 1: lists kept and their entries per warp (warp w takes the
            // 32-list slices w, w + TCP_WARPS, ...); thread 0 turns them into
            // per-warp starting offsets
            uint32_t nv_w = 0, T_w = 0;
            for (uint32_t i0 = warp * 32; i0 < cn; i0 += TCP_THREADS) {
                const uint32_t i = i0 + lane;
                uint32_t dv = 0;
                if (i < cn) {
                    const uint32_t v = A[c0 + i];
                    dv = (uint32_t)(off[v + 1] - off[v]);
                }
                nv_w += __popc(__ballot_sync(GV_FULL_MASK, dv > 0));
                T_w += warp_sum(dv);
            }
            if (lane == 0) {
                wcnt[warp] = nv_w;
                wsum[warp] = T_w;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                uint32_t a = 0, t = 0;
                for (int w = 0; w < TCP_WARPS; ++w) {
                    const uint32_t x = wcnt[w], y = wsum[w];
                    wcnt[w] = a;
                    wsum[w] = t;
                    a += x;
                    t += y;
                }
                s_nv = a;
                s_T = t;
                pref[a] = t;
            }
            __syncthreads();
            // pass 2: place the same slices in the same order
            uint32_t nv = wcnt[warp], T = wsum[warp];
            for (uint32_t i0 = warp * 32; i0 < cn; i0 += TCP_THREADS)
                tcp_gather32(off, A + c0, cn, i0, vl, base, pref, nv, T, nullptr, 0);
            __syncthreads();
            const uint32_t NV = s_nv, TT = s_T;
            for (uint32_t p0 = warp * 32; p0 < TT; p0 += TCP_THREADS) {
                uint32_t j0 = 0;
                if (lane == 0) {  // last list starting at or before p0
                    uint32_t lo = 0, hi2 = NV;
                    while (hi2 - lo > 1) {
                        const uint32_t mid = (lo + hi2) >> 1;
                        if (pref[mid] <= p0) lo = mid;
                        else hi2 = mid;
                    }
                    j0 = lo;
                }
                j0 = __shfl_sync(GV_FULL_MASK, j0, 0);
                tcp_step<MODE>(snap, set, mask, vl, base, pref, NV, TT, p0, j0, u, cr, cu);
            }
            if (lane == 0 && warp == 0) my_work += TT;
            __syncthreads();
        }
        cu = warp_sum(cu);
        if (lane == 0) cured[warp] = cu;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t t = 0;
            for (int w = 0; w < TCP_WARPS; ++w) t += cured[w];
            if (t) cr.add(u, t);
            my_work += la;
        }
        __syncthreads();
    }
    my_work = warp_sum(my_work);
    if (lane == 0) wred[warp] = my_work;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int i = 0; i < TCP_WARPS; ++i) t += wred[i];
        if (t) atomicAdd(work, t);
    }
    cr.flush();
}

__global__ void k_tc_esrc(const unsigned long long *__restrict__ off, uint32_t n, uint32_t *__restrict__ esrc) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x)
        for (unsigned long long i = off[u]; i < off[u + 1]; ++i) esrc[i] = u;
}

__global__ void k_sum_u64(const unsigned long long *__restrict__ x, uint32_t n, unsigned long long *out) {
    unsigned long long t = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) t += x[v];
    t = warp_sum(t);
    if ((threadIdx.x & 31) == 0 && t) atomicAdd(out, t);
}

__global__ void k_gather_u64(const unsigned long long *__restrict__ x, const uint32_t *__restrict__ idx, uint64_t k,
                             unsigned long long *__restrict__ out) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < k; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = x[idx[i]];
}

struct TcBufs {
    uint32_t *dplus;
    unsigned long long *off;
    uint32_t *snap, *esrc, *mid, *big, *hubs;
    unsigned long long *cnts;  // [0] mid lists, [1] big lists, [2] hubs
    unsigned long long *tcount;
    unsigned long long *hcur;  // per-hub write cursors
};

// Core size bound of the total-only count: GV_TC_CORE=<vertices> (0: merge
// every edge), rounded down to a multiple of 32, at most TCC_MAX (core
// indices are 16-bit and leave TCC_DEAD free).
uint32_t tc_core_max() {
    const char *env = std::getenv("GV_TC_CORE");
    long v = env ? std::strtol(env, nullptr, 10) : (long)TCC_DEFAULT;
    v = std::max<long>(0, std::min<long>(v, (long)TCC_MAX));
    return (uint32_t)v & ~31u;
}

// GV_TC_COLOR=0 leaves the core lists in fill order (for comparison).
bool tc_color() {
    const char *env = std::getenv("GV_TC_COLOR");
    return !(env && env[0] == '0');
}

// Dense core of a total-only count, first half: carves the core buffers from
// auxiliary slot 10 and picks the core (k.cidx).  No host synchronisation.
gv_status tc_core_select(gv_graph *g, const TcBufs &b, uint64_t mplus, uint32_t cmax, TcCore &k, cudaStream_t s) {
    const uint32_t n = g->d.n;
    const uint32_t wmax = (cmax + 31) / 32;
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t o_hist = 0, o_ctl = o_hist + al((size_t)TCC_BINS * 4), o_cidx = o_ctl + 256;
    const size_t o_ccnt = o_cidx + al((size_t)n * 4), o_coff = o_ccnt + al((size_t)n * 4);
    const size_t o_icnt = o_coff + al(((size_t)n + 1) * 8), o_ioff = o_icnt + al(((size_t)cmax + 1) * 4);
    const size_t o_itcnt = o_ioff + al(((size_t)cmax + 1) * 8), o_itoff = o_itcnt + al(((size_t)cmax + 1) * 4);
    const size_t o_rows = o_itoff + al(((size_t)cmax + 1) * 4), o_clist = o_rows + al((size_t)cmax * wmax * 4);
    const size_t o_inl = o_clist + al(((size_t)mplus + 8 * (size_t)n) * 2), o_itc = o_inl + al((size_t)mplus * 4);
    const size_t max_items = (size_t)mplus / TCC_CHUNK + cmax + 1;  // sum of ceil(in-degree / chunk)
    const size_t o_rest = o_itc + al(max_items * 4), bytes = o_rest + al((size_t)mplus * 4);
    char *p = (char *)aux_scratch(g, 10, bytes);
    if (!p) return GV_ERR_NOMEM;
    k.hist = (uint32_t *)(p + o_hist);
    k.ctl = (uint32_t *)(p + o_ctl);
    k.cidx = (uint32_t *)(p + o_cidx);
    k.ccnt = (uint32_t *)(p + o_ccnt);
    k.coff = (unsigned long long *)(p + o_coff);
    k.icnt = (uint32_t *)(p + o_icnt);
    k.ioff = (unsigned long long *)(p + o_ioff);
    k.itcnt = (uint32_t *)(p + o_itcnt);
    k.itoff = (uint32_t *)(p + o_itoff);
    k.rows = (uint32_t *)(p + o_rows);
    k.clist = (uint16_t *)(p + o_clist);
    k.inl = (uint32_t *)(p + o_inl);
    k.itc = (uint32_t *)(p + o_itc);
    k.rest = (uint32_t *)(p + o_rest);
    k.cmax = cmax;
    k.wmax = wmax;
    const uint32_t *deg = b.hubs;  // live degrees, as the orientation used them
    {
        ProfScope ps(PROF_TC_CORE, s);
        cudaMemsetAsync(k.hist, 0, (size_t)TCC_BINS * 4, s);
        cudaMemsetAsync(k.ccnt, 0, (size_t)n * 4, s);
        cudaMemsetAsync(k.icnt, 0, ((size_t)cmax + 1) * 4, s);
        cudaMemsetAsync(k.rows, 0, (size_t)cmax * wmax * 4, s);
        GV_LAUNCH(k_tcc_hist, grid_for(n, 256), 256, 0, s, deg, n, k.hist);
        GV_LAUNCH(k_tcc_pick, 1, 1024, 0, s, (const uint32_t *)k.hist, cmax, k.ctl);
        GV_LAUNCH(k_tcc_index, grid_for(n, 256), 256, 0, s, deg, n, k.ctl, k.cidx);
    }
    return cuda_status(cudaGetLastError(), "tc core");
}

// Second half, once the lists outside the core are sorted: builds the rows,
// core lists, in-neighbour lists and the list of edges left to the merge
// (k.rest, count k.ctl[2]), then adds the core edges' triangles into
// tcount[0].  No host synchronisation.
gv_status tc_core_count(gv_graph *g, const TcBufs &b, uint64_t mplus, TcCore &k, unsigned long long *work,
                        cudaStream_t s) {
    const uint32_t n = g->d.n, cmax = k.cmax;
    {
        ProfScope ps(PROF_TC_CORE, s);
        const unsigned egrid = grid_for(mplus, 256, 148 * 16);
        GV_LAUNCH(k_tcc_count, egrid, 256, 0, s, (const uint32_t *)b.snap, (const uint32_t *)b.esrc, mplus,
                  (const uint32_t *)k.cidx, k.ccnt, k.icnt, k.rest, k.ctl + 2);
        GV_LAUNCH(k_tcc_pad, grid_for(n, 256), 256, 0, s, k.ccnt, n);
        scan_exclusive_u32_to_u64(k.ccnt, k.coff, n, k.coff + n, g->bs.scan_tmp, s);
        cudaMemsetAsync(k.clist, 0xFF, ((size_t)mplus + 8 * (size_t)n) * 2, s);  // padding = TCC_DEAD
        scan_exclusive_u32_to_u64(k.icnt, k.ioff, cmax, k.ioff + cmax, g->bs.scan_tmp, s);
        cudaMemsetAsync(k.ccnt, 0, (size_t)n * 4, s);
        cudaMemsetAsync(k.icnt, 0, ((size_t)cmax + 1) * 4, s);
        GV_LAUNCH(k_tcc_fill, egrid, 256, 0, s, (const uint32_t *)b.snap, (const uint32_t *)b.esrc, mplus, k);
        if (tc_color())
            GV_LAUNCH(k_tcc_color, grid_for(n, 8 * 32, 148 * 8), 256, (size_t)8 * TCC_COLOR_MAX * 2, s, k, n);
        GV_LAUNCH(k_tcc_items, grid_for(cmax, 256), 256, 0, s, (const unsigned long long *)k.ioff, cmax, k.itcnt);
        scan_exclusive_u32(k.itcnt, k.itoff, cmax, k.itoff + cmax, g->bs.scan_tmp, s);
        GV_LAUNCH(k_tcc_item_owner, grid_for(cmax, 8), 256, 0, s, (const uint32_t *)k.itoff, cmax, k.itc);
    }
    {
        ProfScope ps(PROF_TC_PROBE, s);
        // 32 CTAs per SM of shares (7.0 ms for the probes at R-MAT scale 22,
        // 7.7 with 8): the block scheduler evens out the rows' uneven work
        GV_LAUNCH(k_tcc_probe, 148 * 32, TCC_THREADS, 0, s, k, b.tcount, work + 1);
    }
    cudaMemcpyAsync(work + 2, k.ctl + 1, 4, cudaMemcpyDeviceToDevice, s);  // core size (low word)
    return cuda_status(cudaGetLastError(), "tc core");
}

// Builds the oriented sorted snapshot and counts.  tcount[n] receives the
// per-vertex counts (owner or incident).  Returns m_plus via *mplus.
gv_status tc_run(gv_graph *g, cudaStream_t s, int mode, unsigned long long **tcount_out) {
    if (g->cfg.directed) { set_error("triangle counting needs an undirected store"); return GV_ERR_STATE; }
    DevGraph d = g->d;
    const uint32_t n = d.n;
    uint64_t live = 0;
    {
        Ctl c;
        gv_status st = read_ctl(g, &c, s);
        if (st != GV_OK) return st;
        live = c.live_edges;
    }
    // An oriented snapshot holds at most one entry per live entry.
    const size_t head = ((size_t)n + 1) * 8 + (size_t)n * 8 * 2 + 64 + (size_t)n * 4 * 4;
    void *buf = analytics_scratch(g, head + 2 * (live + 1) * 4 + 256);
    if (!buf) return GV_ERR_NOMEM;
    TcBufs b;
    {
        char *p = (char *)buf;
        b.off = (unsigned long long *)p; p += ((size_t)n + 1) * 8;
        b.tcount = (unsigned long long *)p; p += (size_t)n * 8;
        b.hcur = (unsigned long long *)p; p += (size_t)n * 8;
        b.cnts = (unsigned long long *)p; p += 64;
        b.dplus = (uint32_t *)p; p += (size_t)n * 4;
        b.mid = (uint32_t *)p; p += (size_t)n * 4;
        b.big = (uint32_t *)p; p += (size_t)n * 4;
        b.hubs = (uint32_t *)p; p += (size_t)n * 4;
        b.snap = (uint32_t *)p; p += (live + 1) * 4;
        b.esrc = (uint32_t *)p;
    }
    const uint32_t tpv = g->cfg.threads_per_vertex;
    unsigned long long mplus = 0;
    {
        ProfScope ps(PROF_TC_SNAPSHOT, s);
        uint32_t *deg = b.hubs;  // live degree per vertex (4 B, stays in L2)
        launch_degrees(g, deg, s);
        cudaMemsetAsync(b.cnts, 0, 64, s);
        Items it{};
        float *ip = nullptr;
        gv_status st = build_items(g, s, b.cnts + 3, &it, &ip, false);
        if (st != GV_OK) return st;
        uint32_t *icnt = (uint32_t *)ip;
        uint32_t *ioff = nullptr;
        if (it.nitems) {
            ioff = (uint32_t *)aux_scratch(g, 3, (size_t)it.nitems * 4);
            if (!ioff) return GV_ERR_NOMEM;
        }
        dispatch_tpv(tpv, [&](auto t) {
            constexpr int T = decltype(t)::value;
            // per-vertex lists of uneven length: many CTA shares (the snapshot
            // 2.1 ms at R-MAT scale 22 against 2.4 capped at 148 * 8)
            GV_LAUNCH((k_tc_outdeg<T>), grid_for(n, AN_THREADS / T, 148 * 32), AN_THREADS, 0, s, d, (const uint32_t *)deg,
                      b.dplus);
        });
        if (it.nitems) {
            GV_LAUNCH(k_tc_items<false>, PULL_GRID, AN_THREADS, 0, s, d, (const uint32_t *)deg, it, icnt,
                      (const uint32_t *)nullptr, (const unsigned long long *)nullptr, (uint32_t *)nullptr);
            GV_LAUNCH(k_tc_multi, grid_for(it.nmulti, 256), 256, 0, s, it, (const uint32_t *)icnt, ioff, b.dplus);
        }
        scan_exclusive_u32_to_u64(b.dplus, b.off, n, b.off + n, g->bs.scan_tmp, s);
        cudaMemcpyAsync(&mplus, b.off + n, 8, cudaMemcpyDeviceToHost, s);
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e, "tc");
        if (mplus > live) { set_error("oriented snapshot larger than the store"); return GV_ERR_STATE; }
        cudaMemsetAsync(b.tcount, 0, (size_t)n * 8, s);
        dispatch_tpv(tpv, [&](auto t) {
            constexpr int T = decltype(t)::value;
            GV_LAUNCH((k_tc_write<T>), grid_for(n, AN_THREADS / T, 148 * 32), AN_THREADS, 0, s, d, (const uint32_t *)deg,
                      (const unsigned long long *)b.off, b.snap);
        });
        if (it.nitems)
            GV_LAUNCH(k_tc_items<true>, PULL_GRID, AN_THREADS, 0, s, d, (const uint32_t *)deg, it, icnt,
                      (const uint32_t *)ioff, (const unsigned long long *)b.off, b.snap);
    }
    // per-graph word (views own theirs), so concurrent counts on views do not share it
    unsigned long long *work = (unsigned long long *)g->bs.tile_cnt + 1;
    cudaMemsetAsync(work, 0, 24, s);  // merged entries, core probes, core vertices
    const char *packed_env = std::getenv("GV_TC_PACKED");
    if (packed_env && packed_env[0] == '1') {
        // packed hash probe: lists unsorted, u with d+ > TCP_LIGHT to one CTA each
        unsigned long long *hc = b.cnts + 4;  // [0] heavy count, [1] longest d+
        cudaMemsetAsync(hc, 0, 16, s);
        GV_LAUNCH(k_tcp_heavy_list, grid_for(n, 256), 256, 0, s, (const unsigned long long *)b.off, n, b.mid, hc);
        unsigned long long hh[2] = {0, 0};
        cudaError_t e = cudaMemcpyAsync(hh, hc, 16, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e, "tc plan");
        const size_t light_smem = sizeof(TcpWarp) * TCP_WARPS + (size_t)TC_CREDIT_HT * 12;
        const size_t heavy_smem = (size_t)TCP_SSET * 4 + (size_t)TCP_CHUNK * 12 + ((size_t)TCP_CHUNK + 32) * 4 +
                                  (size_t)TC_CREDIT_HT * 12;
        const unsigned heavy_grid = (unsigned)std::min<unsigned long long>(std::max<unsigned long long>(hh[0], 1), 148 * 2);
        uint32_t gcap = 0;
        uint32_t *gset = nullptr;
        if (2 * hh[1] > TCP_SSET) {  // sets above the shared table live in global memory, one per CTA
            gcap = 1024;
            while (gcap < 2 * hh[1]) gcap <<= 1;
            gset = (uint32_t *)aux_scratch(g, 7, (size_t)gcap * heavy_grid * 4);
            if (!gset) return GV_ERR_NOMEM;
        }
        const unsigned light_grid = 148 * 3;
        ProfScope ps(PROF_TC_COUNT, s);
        const unsigned long long *off_c = b.off;
        const uint32_t *snap_c = b.snap;
        auto launch = [&](auto mode_c) {
            constexpr int M = decltype(mode_c)::value;
            cudaFuncSetAttribute(k_tcp_light<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)light_smem);
            cudaFuncSetAttribute(k_tcp_heavy<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)heavy_smem);
            GV_LAUNCH(k_tcp_light<M>, light_grid, TCP_THREADS, light_smem, s, off_c, snap_c, n, b.tcount, work);
            if (hh[0])
                GV_LAUNCH(k_tcp_heavy<M>, heavy_grid, TCP_THREADS, heavy_smem, s, off_c, snap_c, b.tcount,
                          (const uint32_t *)b.mid, (const unsigned long long *)hc, gset, gcap, work);
        };
        if (mode == TC_INCIDENT) launch(std::integral_constant<int, TC_INCIDENT>{});
        else if (mode == TC_TOTAL) launch(std::integral_constant<int, TC_TOTAL>{});
        else launch(std::integral_constant<int, TC_OWNER>{});
        g->last_tc_oriented = mplus;
        *tcount_out = b.tcount;
        return cuda_status(cudaGetLastError(), "tc launch");
    }
    // merge path (default): sorted lists, merge-path intersection per oriented
    // edge; for total-only counts the edges into the dense core go to bit
    // probes first, and the core's own lists (read by no merge) stay unsorted
    GV_LAUNCH(k_tc_esrc, grid_for(n, 256), 256, 0, s, (const unsigned long long *)b.off, n, b.esrc);
    // the core is picked first: its lists are read by no merge and stay unsorted
    TcCore core{};
    const bool use_core = mode == TC_TOTAL && mplus && mplus < (1ull << 32) &&  // merge-list edge ids are 32-bit
                          std::min<uint32_t>(tc_core_max(), n) > 0;
    if (use_core) {
        gv_status st = tc_core_select(g, b, mplus, std::min<uint32_t>(tc_core_max(), n), core, s);
        if (st != GV_OK) return st;
    }
    const uint32_t *core_of = use_core ? core.cidx : nullptr;
    {
        ProfScope ps(PROF_TC_SORT, s);
        GV_LAUNCH(k_tc_classify, grid_for(n, 256), 256, 0, s, (const unsigned long long *)b.off, n, b.snap, b.mid,
                  b.big, b.cnts, core_of);
        GV_LAUNCH(k_tc_sort_mid, 148 * 32, AN_THREADS, 0, s, (const unsigned long long *)b.off, b.snap,  // 1.1 ms (1.3 with 148 * 4)
                  (const uint32_t *)b.mid, (const unsigned long long *)b.cnts);
        // the longest list bounds the CTA sort's shared memory
        unsigned long long h[3] = {0, 0, 0};
        cudaMemcpyAsync(h, b.cnts, 24, cudaMemcpyDeviceToHost, s);
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e, "tc");
        if (h[1]) {  // lists above 1024 entries: one CTA sort each
            uint32_t P = 1024;
            while (P < h[2]) P <<= 1;
            const size_t smem = (size_t)P * 4;
            if (smem > 227 * 1024) { set_error("oriented out-degree exceeds the shared-memory sort"); return GV_ERR_UNSUPPORTED; }
            cudaFuncSetAttribute(k_tc_sort_big, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            GV_LAUNCH(k_tc_sort_big, 148, 1024, smem, s, (const unsigned long long *)b.off, b.snap,
                      (const uint32_t *)b.big, (const unsigned long long *)b.cnts, P);
        }
    }
    const uint32_t *rest = nullptr, *nrest = nullptr;
    if (use_core) {
        gv_status st = tc_core_count(g, b, mplus, core, work, s);
        if (st != GV_OK) return st;
        rest = core.rest;
        nrest = core.ctl + 2;
    }
    {
        const unsigned cgrid = grid_for(mplus, AN_THREADS / 8, 148 * 64);  // 4.1 ms at scale 22 (4.4 capped at 148 * 16)
        ProfScope ps(PROF_TC_COUNT, s);
        const unsigned long long *off_c = b.off;
        if (mode == TC_INCIDENT)
            GV_LAUNCH((k_tc_count<8, TC_INCIDENT>), cgrid, AN_THREADS, 0, s, off_c, b.snap, b.esrc, mplus, b.tcount, work,
                      (const uint32_t *)nullptr, (const uint32_t *)nullptr);
        else if (mode == TC_TOTAL)
            // 16 lanes per edge: the lists left outside the core are short, and
            // 16 lanes split the co-rank search and the merge best (4.4 ms
            // against 5.1 with 8 and 4.9 with 32 at scale 22)
            GV_LAUNCH((k_tc_count<16, TC_TOTAL>), cgrid, AN_THREADS, 0, s, off_c, b.snap, b.esrc, mplus, b.tcount, work,
                      rest, nrest);
        else
            GV_LAUNCH((k_tc_count<8, TC_OWNER>), cgrid, AN_THREADS, 0, s, off_c, b.snap, b.esrc, mplus, b.tcount, work,
                      (const uint32_t *)nullptr, (const uint32_t *)nullptr);
    }
    g->last_tc_oriented = mplus;
    *tcount_out = b.tcount;
    return cuda_status(cudaGetLastError(), "tc launch");
}

// ------------------------------------------------------- weighted PageRank
__global__ void k_row_inv_deg(DevGraph g, float *__restrict__ rinv) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < g.n; u += gridDim.x * blockDim.x) {
        const uint32_t dl = g.vtx[u].z;
        rinv[u] = dl ? 1.0f / (float)dl : 0.f;
    }
}

__global__ void k_row_sums(DevGraph g, float *__restrict__ rinv) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < g.n; u += gridDim.x * blockDim.x) {
        const uint4 rec = g.vtx[u];
        const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB);
        double sacc = 0.0;
        for (uint32_t k = 0; k < nb; ++k) {
            const uint32_t b = k == 0 ? rec.x : cbt_block(g.left, g.right, rec.x, k);
            const uint32_t slots = min(g.B, fill - (k << g.logB));
            const size_t base = (size_t)b << g.logB;
            for (uint32_t i = 0; i < slots; ++i)
                if (g.pool[base + i] != GV_TOMB) sacc += (double)g.wpool[base + i];
        }
        rinv[u] = sacc > 0.0 ? (float)(1.0 / sacc) : 0.f;
    }
}

// Transposed snapshot: in-edges of every v with the raw weight.
// In-edge transpose for weighted PageRank: one key (v << bitsn | u) per
// stored entry (found from the exported offsets), the weight's bits carried
// as the value; a stable radix sort then groups in-edges by v, ordered by u,
// so the transpose (and every sum over it) is the same on every call.
__global__ void k_wpr_keys(const unsigned long long *__restrict__ off, const uint32_t *__restrict__ dst,
                           const float *__restrict__ w, uint32_t n, uint64_t E, uint32_t bitsn,
                           unsigned long long *__restrict__ keys, uint32_t *__restrict__ vals) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = n;  // last u with off[u] <= i
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (off[mid] <= i) lo = mid;
            else hi = mid;
        }
        keys[i] = ((unsigned long long)dst[i] << bitsn) | lo;
        vals[i] = __float_as_uint(w ? w[i] : 1.0f);
    }
}

// toff[v] = first sorted key of destination v (v = 0..n).
__global__ void k_wpr_toff(const unsigned long long *__restrict__ keys, uint64_t E, uint32_t n, uint32_t bitsn,
                           unsigned long long *__restrict__ toff) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v <= n; v += gridDim.x * blockDim.x) {
        const unsigned long long x = (unsigned long long)v << bitsn;
        uint64_t lo = 0, hi = E;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (keys[mid] < x) lo = mid + 1;
            else hi = mid;
        }
        toff[v] = lo;
    }
}

__global__ void k_wpr_unpack(const unsigned long long *__restrict__ keys, const uint32_t *__restrict__ vals, uint64_t E,
                             unsigned long long mask, uint32_t *__restrict__ tsrc, float *__restrict__ tw) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (uint64_t)gridDim.x * blockDim.x) {
        tsrc[i] = (uint32_t)(keys[i] & mask);
        tw[i] = __uint_as_float(vals[i]);
    }
}

// Vertices with more than WPR_HEAVY in-edges (one CTA each in the sweeps).
constexpr uint32_t WPR_HEAVY = 1024;
constexpr unsigned WPR_HEAVY_GRID = FIN_GRID;

__global__ void k_wpr_heavy_list(const unsigned long long *__restrict__ toff, uint32_t n, uint32_t *__restrict__ list,
                                 uint32_t *cnt) {
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t v = base + threadIdx.x;
        const bool heavy = v < n && toff[v + 1] - toff[v] > WPR_HEAVY;
        const uint32_t bal = __ballot_sync(GV_FULL_MASK, heavy);
        uint32_t at = 0;
        if (lane == 0 && bal) at = atomicAdd(cnt, (uint32_t)__popc(bal));
        at = __shfl_sync(GV_FULL_MASK, at, 0);
        if (heavy) list[at + __popc(bal & ((1u << lane) - 1u))] = v;
    }
}

// Heavy in-edge lists: the CTA's threads stride over the list, the block sum
// is taken in a fixed order; partial slot part_base + blockIdx.x.
__global__ void __launch_bounds__(AN_THREADS) k_wpr_fwd_heavy(const unsigned long long *__restrict__ toff,
                                                              const uint32_t *__restrict__ tsrc,
                                                              const float *__restrict__ tw,
                                                              const uint32_t *__restrict__ list, const uint32_t *cnt,
                                                              PullArgs a, uint32_t part_base) {
    __shared__ float red[AN_THREADS / 32];
    if (a.state[0]) return;
    const uint32_t nh = *cnt;
    double res = 0.0;
    for (uint32_t h = blockIdx.x; h < nh; h += gridDim.x) {
        const uint32_t v = list[h];
        float sum = 0.f;
        for (unsigned long long i = toff[v] + threadIdx.x; i < toff[v + 1]; i += AN_THREADS)
            sum += tw[i] * __ldg(a.gather + tsrc[i]);
        sum = warp_sum(sum);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
        __syncthreads();
        if (threadIdx.x == 0) {
            float t = 0.f;
            for (int i = 0; i < AN_THREADS / 32; ++i) t += red[i];
            pull_finish(a, v, t, 0, res);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) a.partial[part_base + blockIdx.x] = res;
}

// Group per v over its in-edges: x'[v] = base + alpha * sum w_uv * contrib[u]
template <int TPV>
__global__ void __launch_bounds__(AN_THREADS) k_wpr_fwd(uint32_t n, const unsigned long long *__restrict__ toff,
                                                        const uint32_t *__restrict__ tsrc, const float *__restrict__ tw,
                                                        PullArgs a) {
    __shared__ double red[AN_THREADS / 32];
    if (a.state[0]) return;
    constexpr int GPC = AN_THREADS / TPV;
    Group<TPV> G;
    double res = 0.0;
    const uint32_t ngroups = gridDim.x * GPC;
    for (uint32_t v = blockIdx.x * GPC + threadIdx.x / TPV; v < n; v += ngroups) {
        if (toff[v + 1] - toff[v] > WPR_HEAVY) continue;  // k_wpr_fwd_heavy
        float sum = 0.f;
        for (unsigned long long i = toff[v] + G.gl; i < toff[v + 1]; i += TPV) sum += tw[i] * __ldg(a.gather + tsrc[i]);
        sum = G.sum(sum);
        if (G.gl == 0) pull_finish(a, v, sum, 0, res);
    }
    res = warp_sum(res);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = res;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < AN_THREADS / 32; ++i) t += red[i];
        a.partial[blockIdx.x] = t;
    }
}

__global__ void k_mul(const float *__restrict__ x, const float *__restrict__ r, float *__restrict__ y, uint32_t n) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) y[v] = x[v] * r[v];
}

// Gradient per entry from the exported CSR (dst in export order): one thread
// per entry, its source found by binary search in the offsets, so hubs cost
// no more than any other vertex.
__global__ void k_wpr_grad_flat(const unsigned long long *__restrict__ off, const uint32_t *__restrict__ dst,
                                uint64_t E, uint32_t n, const float *__restrict__ x, const float *__restrict__ lam,
                                const float *__restrict__ c, const float *__restrict__ rinv, float alpha, int mode,
                                float *__restrict__ grad) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = n;  // last u with off[u] <= i
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (off[mid] <= i) lo = mid;
            else hi = mid;
        }
        const uint32_t u = lo;
        const float lv = lam[dst[i]];
        grad[i] = (mode == 1) ? alpha * x[u] * lv : x[u] * (alpha * lv + (c[u] - lam[u])) * rinv[u];
    }
}

// ------------------------------------------------------ batched PPR queries
// k <= 32 personalised PageRank queries share every adjacency read: lane j
// of a warp owns query j, values are vertex-major (x[v * k + j]), and one
// coalesced load of a neighbour's k contributions serves all queries.
struct PprBatch {
    uint32_t k;
    const uint32_t *sources;  // device, k
    float alpha;
    const float *gather;      // contributions (n * k)
    const float *xold;
    float *xnew, *cnew;
    double *partial;          // [grid][32]
    const int *state;
};

__device__ __forceinline__ void ppr_finish(const DevGraph &g, const PprBatch &a, uint32_t v, float acc, uint32_t lane,
                                           double &res) {
    if (lane >= a.k) return;
    const float base = (a.sources[lane] == v) ? (1.0f - a.alpha) : 0.f;
    const float xv = base + a.alpha * acc;
    const size_t at = (size_t)v * a.k + lane;
    a.xnew[at] = xv;
    const uint32_t d = g.vtx[v].z;
    a.cnew[at] = d ? xv / (float)d : 0.f;
    res += (double)fabsf(xv - a.xold[at]);
}

// Warp per vertex of the thread-per-vertex and lane-group tiers (it.tiny,
// then it.light), lane = query; CTA vb of vg, residual slot vb.
__device__ __forceinline__ void ppr_light_body(const DevGraph &g, const PprBatch &a, const Items &it, uint32_t vb,
                                               uint32_t vg) {
    __shared__ double red[AN_THREADS / 32][32];
    if (a.state[0]) return;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double res = 0.0;
    const uint32_t nw = vg * (AN_THREADS / 32), nv = it.ntiny + it.nlight;
    for (uint32_t i = vb * (AN_THREADS / 32) + warp; i < nv; i += nw) {
        const uint32_t v = i < it.ntiny ? it.tiny[i] : it.light[i - it.ntiny];
        const uint4 rec = g.vtx[v];
        const uint32_t fill = rec.y;
        const uint32_t nb = blocks_for(fill, g.logB);
        const uint32_t my_blk = item_block(g, rec, 0, nb);  // lane k holds block k (nb <= 8)
        float acc = 0.f;
        for (uint32_t e0 = 0; e0 < fill; e0 += 32) {
            const uint32_t e = e0 + lane;
            const uint32_t pb = __shfl_sync(GV_FULL_MASK, my_blk, (e >> g.logB) & 31u);
            const uint32_t u = (e < fill) ? g.pool[((size_t)pb << g.logB) + (e & (g.B - 1))] : GV_TOMB;
            const uint32_t cnt = min(32u, fill - e0);
#pragma unroll 8
            for (uint32_t j = 0; j < cnt; ++j) {
                const uint32_t w = __shfl_sync(GV_FULL_MASK, u, j);
                if (w != GV_TOMB && lane < a.k) acc += __ldg(a.gather + (size_t)w * a.k + lane);
            }
        }
        ppr_finish(g, a, v, acc, lane, res);
    }
    red[warp][lane] = res;
    __syncthreads();
    if (warp == 0) {
        double t = 0.0;
        for (int w = 0; w < AN_THREADS / 32; ++w) t += red[w][lane];
        a.partial[(size_t)vb * 32 + lane] = t;
    }
}

__device__ __forceinline__ void ppr_items_body(const DevGraph &g, const PprBatch &a, const Items &it,
                                               float *__restrict__ ipart, uint32_t vb, uint32_t vg) {
    if (a.state[0]) return;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t nw = vg * (AN_THREADS / 32);
    for (uint32_t i = vb * (AN_THREADS / 32) + (threadIdx.x >> 5); i < it.nitems; i += nw) {
        const uint32_t v = it.item_vertex[i];
        const uint32_t c = i - it.item_first[v];
        const uint4 rec = g.vtx[v];
        const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB);
        const uint32_t kb0 = c << 5;
        const uint32_t my_blk = item_block(g, rec, kb0, nb);
        const uint32_t e0 = kb0 << g.logB, e1 = min(fill, (kb0 + 32) << g.logB);
        float acc = 0.f;
        for (uint32_t q0 = e0; q0 < e1; q0 += 32) {
            const uint32_t el = q0 - e0 + lane;
            const uint32_t pb = __shfl_sync(GV_FULL_MASK, my_blk, (el >> g.logB) & 31u);
            const uint32_t u = (q0 + lane < e1) ? g.pool[((size_t)pb << g.logB) + (el & (g.B - 1))] : GV_TOMB;
            const uint32_t cnt = min(32u, e1 - q0);
#pragma unroll 8
            for (uint32_t j = 0; j < cnt; ++j) {
                const uint32_t w = __shfl_sync(GV_FULL_MASK, u, j);
                if (w != GV_TOMB && lane < a.k) acc += __ldg(a.gather + (size_t)w * a.k + lane);
            }
        }
        ipart[(size_t)i * 32 + lane] = acc;
    }
}

// One launch for both parts of a batched sweep: CTA i takes the warp-per-
// vertex part when i is even (residual slot i / 2), the hub items when odd.
__global__ void __launch_bounds__(AN_THREADS) k_ppr_fused(DevGraph g, PprBatch a, Items it, float *__restrict__ ipart) {
    const uint32_t vb = blockIdx.x >> 1, vg = gridDim.x >> 1;
    if ((blockIdx.x & 1u) == 0) ppr_light_body(g, a, it, vb, vg);
    else ppr_items_body(g, a, it, ipart, vb, vg);
}

__global__ void __launch_bounds__(AN_THREADS) k_ppr_items_fin(DevGraph g, PprBatch a, Items it,
                                                              const float *__restrict__ ipart, uint32_t part_base) {
    __shared__ double red[AN_THREADS / 32][32];
    if (a.state[0]) return;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double res = 0.0;
    const uint32_t nw = gridDim.x * (AN_THREADS / 32);
    for (uint32_t m = blockIdx.x * (AN_THREADS / 32) + warp; m < it.nmulti; m += nw) {
        const uint32_t v = it.multi[m];
        float acc = 0.f;
        for (uint32_t i = it.item_first[v]; i < it.item_first[v + 1]; ++i) acc += ipart[(size_t)i * 32 + lane];
        ppr_finish(g, a, v, acc, lane, res);
    }
    red[warp][lane] = res;
    __syncthreads();
    if (warp == 0) {
        double t = 0.0;
        for (int w = 0; w < AN_THREADS / 32; ++w) t += red[w][lane];
        a.partial[(size_t)(part_base + blockIdx.x) * 32 + lane] = t;
    }
}

// Per query: sum of its residual partials; converged when every query is.
__global__ void k_ppr_done(const double *__restrict__ partial, uint32_t nparts, uint32_t k, float eps, int *state) {
    __shared__ int all_ok;
    if (state[0]) return;
    if (threadIdx.x == 0) all_ok = 1;
    __syncthreads();
    if (threadIdx.x < k) {
        double t = 0.0;
        for (uint32_t p = 0; p < nparts; ++p) t += partial[(size_t)p * 32 + threadIdx.x];
        if (!(t < (double)eps)) atomicAnd(&all_ok, 0);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        state[1] += 1;
        if (all_ok) state[0] = 1;
    }
}

__global__ void k_ppr_init(DevGraph g, const uint32_t *__restrict__ sources, uint32_t k, float *__restrict__ x,
                           float *__restrict__ c) {
    const size_t total = (size_t)g.n * k;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t v = (uint32_t)(i / k), j = (uint32_t)(i % k);
        const float xv = (sources[j] == v) ? 1.f : 0.f;
        x[i] = xv;
        const uint32_t d = g.vtx[v].z;
        c[i] = d ? xv / (float)d : 0.f;
    }
}

gv_status ppr_batch_impl(gv_graph *g, const uint32_t *sources, uint32_t k, float alpha, float eps, int max_iter,
                         float *x_out, int32_t *sweeps, int mem, cudaStream_t s) {
    if (plan_pagerank_enabled(g)) {  // the degree-ordered sweep plan (prplan.cu)
        bool planned = false;
        gv_status st = GV_OK;
        if (k == 1) {  // one query: the single-vector sweeps
            uint32_t src = GV_NIL;
            if (mem != GV_MEM_DEVICE) src = sources[0];
            else {
                cudaError_t e = cudaMemcpyAsync(&src, sources, 4, cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                if (e != cudaSuccess) return cuda_status(e, "ppr batch source");
            }
            if (src < g->d.n)
                st = plan_pagerank(g, alpha, eps, max_iter, nullptr, GV_MEM_HOST, src, x_out, sweeps, mem, s, &planned);
        } else {
            st = plan_ppr_batch(g, sources, mem, k, alpha, eps, max_iter, x_out, sweeps, mem, s, &planned);
        }
        if (st != GV_OK || planned) return st;
    }
    DevGraph d = g->d;
    const uint32_t n = d.n;
    const size_t vec = (size_t)n * k * sizeof(float);
    const uint32_t nparts = PULL_GRID + FIN_GRID;
    const size_t bytes = 4 * vec + (size_t)nparts * 32 * 8 + 64 + 128 + 256 * 3;
    char *p = (char *)analytics_scratch(g, bytes);
    if (!p) return GV_ERR_NOMEM;
    float *x[2] = {(float *)p, (float *)(p + vec)};
    float *c[2] = {(float *)(p + 2 * vec), (float *)(p + 3 * vec)};
    double *partial = (double *)(p + 4 * vec);
    int *state = (int *)(p + 4 * vec + (size_t)nparts * 32 * 8);
    uint32_t *dsrc = (uint32_t *)(p + 4 * vec + (size_t)nparts * 32 * 8 + 64);
    unsigned long long *nmulti = (unsigned long long *)(dsrc + 32);
    cudaMemcpyAsync(dsrc, sources, k * 4, mem == GV_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s);
    Items it{};
    float *ip_unused = nullptr;
    gv_status st = build_items(g, s, nmulti, &it, &ip_unused);
    if (st != GV_OK) return st;
    float *ipart = nullptr;
    if (it.nitems) {
        ipart = (float *)aux_scratch(g, 3, (size_t)it.nitems * 32 * sizeof(float));
        if (!ipart) return GV_ERR_NOMEM;
    }
    cudaMemsetAsync(state, 0, 16, s);
    cudaMemsetAsync(partial, 0, (size_t)nparts * 32 * 8, s);
    GV_LAUNCH(k_ppr_init, grid_for((uint64_t)n * k, 256, 148 * 16), 256, 0, s, d, (const uint32_t *)dsrc, k, x[0], c[0]);
    int h_state[2] = {0, 0};
    int launched = 0, cur = 0;
    cudaError_t e = cudaSuccess;
    while (launched < max_iter) {
        const int chunk = std::min(8, max_iter - launched);
        for (int i = 0; i < chunk; ++i) {
            PprBatch a{k, dsrc, alpha, c[cur], x[cur], x[cur ^ 1], c[cur ^ 1], partial, state};
            ProfScope ps(PROF_PULL, s);
            GV_LAUNCH(k_ppr_fused, 2 * PULL_GRID, AN_THREADS, 0, s, d, a, it, ipart);
            if (it.nitems)
                GV_LAUNCH(k_ppr_items_fin, FIN_GRID, AN_THREADS, 0, s, d, a, it, (const float *)ipart, PULL_GRID);
            GV_LAUNCH(k_ppr_done, 1, 32, 0, s, (const double *)partial, nparts, k, eps, state);
            cur ^= 1;
        }
        launched += chunk;
        e = cudaMemcpyAsync(h_state, state, 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e, "ppr batch");
        if (h_state[0]) break;
    }
    if (sweeps) *sweeps = h_state[1];
    e = cudaMemcpyAsync(x_out, x[h_state[1] & 1], vec, mem == GV_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return cuda_status(e, "ppr batch");
}

}  // namespace
}  // namespace gv

using namespace gv;

extern "C" {

gv_status gv_ppr_batch(gv_graph *g, const uint32_t *sources, uint32_t k, float alpha, float epsilon, int32_t max_iter,
                       float *x_out, int32_t *sweeps, int mem, void *stream) {
    if (!g || !sources || !x_out || k == 0 || k > 32 || max_iter < 0) { set_error("bad argument"); return GV_ERR_INVALID; }
    if (g->cfg.directed) { set_error("batched PPR needs an undirected (symmetric) store"); return GV_ERR_STATE; }
    if (mem == GV_MEM_HOST)
        for (uint32_t j = 0; j < k; ++j)
            if (sources[j] >= g->d.n) { set_error("source out of range"); return GV_ERR_INVALID; }
    return ppr_batch_impl(g, sources, k, alpha, epsilon, max_iter, x_out, sweeps, mem, (cudaStream_t)stream);
}

gv_status gv_pagerank(gv_graph *g, float alpha, float epsilon, int32_t max_iter, float *x_out, int32_t *sweeps,
                      int mem, void *stream) {
    if (!g || !x_out || max_iter < 0) return GV_ERR_INVALID;
    return pagerank_impl(g, alpha, epsilon, max_iter, nullptr, 0, GV_NIL, x_out, sweeps, mem, (cudaStream_t)stream);
}

gv_status gv_pagerank_dynamic(gv_graph *g, float alpha, float epsilon, int32_t max_iter, float *x_inout,
                              int32_t *sweeps, int mem, void *stream) {
    if (!g || !x_inout || max_iter < 0) return GV_ERR_INVALID;
    return pagerank_impl(g, alpha, epsilon, max_iter, x_inout, mem, GV_NIL, x_inout, sweeps, mem, (cudaStream_t)stream);
}

gv_status gv_ppr(gv_graph *g, uint32_t source, float alpha, float epsilon, int32_t max_iter, float *x_out,
                 int32_t *sweeps, int mem, void *stream) {
    if (!g || !x_out || max_iter < 0 || source >= g->d.n) return GV_ERR_INVALID;
    return pagerank_impl(g, alpha, epsilon, max_iter, nullptr, 0, source, x_out, sweeps, mem, (cudaStream_t)stream);
}

gv_status gv_tc(gv_graph *g, uint64_t *per_vertex, uint64_t *total, int mem, void *stream) {
    if (!g || !total) return GV_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    unsigned long long *tc = nullptr;
    // the total alone needs no per-vertex credit
    gv_status st = tc_run(g, s, per_vertex ? TC_OWNER : TC_TOTAL, &tc);
    if (st != GV_OK) return st;
    const uint32_t n = g->d.n;
    unsigned long long *dtot = (unsigned long long *)g->bs.tile_cnt;  // 8 bytes of batch scratch
    cudaMemsetAsync(dtot, 0, 8, s);
    GV_LAUNCH(k_sum_u64, grid_for(n, 256), 256, 0, s, (const unsigned long long *)tc, n, dtot);
    unsigned long long h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, dtot, 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && per_vertex)
        e = cudaMemcpyAsync(per_vertex, tc, (size_t)n * 8,
                            mem == GV_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "tc");
    *total = h;
    return GV_OK;
}

gv_status gv_tc_subset(gv_graph *g, const uint32_t *subset, uint64_t ns, uint64_t *out, int mem, void *stream) {
    if (!g || (ns && (!subset || !out))) return GV_ERR_INVALID;
    if (ns == 0) return GV_OK;
    cudaStream_t s = (cudaStream_t)stream;
    if (mem == GV_MEM_HOST)
        for (uint64_t i = 0; i < ns; ++i)
            if (subset[i] >= g->d.n) { set_error("subset vertex out of range"); return GV_ERR_INVALID; }
    uint32_t *didx = nullptr;
    unsigned long long *dout = nullptr;
    if (mem == GV_MEM_DEVICE) {
        didx = const_cast<uint32_t *>(subset);
        dout = (unsigned long long *)out;
    } else {
        const size_t at = (ns * 4 + 255) & ~size_t(255);
        char *b = (char *)aux_scratch(g, 0, at + ns * 8);
        if (!b) return GV_ERR_NOMEM;
        didx = (uint32_t *)b;
        dout = (unsigned long long *)(b + at);
        cudaError_t e = cudaMemcpyAsync(didx, subset, ns * 4, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return cuda_status(e, "tc subset input");
    }
    // local counts (neighbour hash sets, tc_local.cu) unless the subset's
    // neighbourhoods cover more than a few passes over the store;
    // GV_TC_SUBSET=local / global picks one path (for comparing them)
    const char *mode = std::getenv("GV_TC_SUBSET");
    const bool force_global = mode && std::strcmp(mode, "global") == 0;
    const bool force_local = mode && std::strcmp(mode, "local") == 0;
    bool done = false;
    gv_status st = GV_OK;
    if (!force_global) st = tc_local_subset(g, didx, ns, dout, s, &done, force_local);
    if (st != GV_OK) return st;
    g->last_tc_local = done ? 1 : 0;
    if (!done) {
        unsigned long long *tc = nullptr;
        st = tc_run(g, s, TC_INCIDENT, &tc);
        if (st != GV_OK) return st;
        GV_LAUNCH(k_gather_u64, grid_for(ns, 256), 256, 0, s, (const unsigned long long *)tc, (const uint32_t *)didx, ns, dout);
    }
    cudaError_t e = cudaSuccess;
    if (mem != GV_MEM_DEVICE) e = cudaMemcpyAsync(out, dout, ns * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return cuda_status(e, "tc subset");
}

}  // extern "C"

namespace gv {
namespace {

// PageRank over the sorted in-edge transpose of the store: weighted (raw
// weights normalised per row) or, with `unit`, plain PageRank on a directed
// store (every out-entry of u weighs 1 / outdeg(u)).  x_init (warm start) or
// a personalisation source as pagerank_impl takes them.
gv_status transpose_pagerank(gv_graph *g, float alpha, float tol, int32_t max_iter, bool unit, const float *x_init,
                             int init_mem, uint32_t source, float *x_out, int32_t *sweeps, int mem, cudaStream_t s) {
    DevGraph d = g->d;
    const uint32_t n = d.n;
    uint64_t live = 0;
    {
        Ctl c;
        gv_status st = read_ctl(g, &c, s);
        if (st != GV_OK) return st;
        live = c.live_edges;
    }
    const uint32_t parts = SWEEP_PARTS;
    const size_t bytes = iter_bytes(n, parts) + (size_t)n * 4 * 3 + ((size_t)n + 1) * 8 + (live + 1) * 8 + 512;
    void *buf = analytics_scratch(g, bytes);
    if (!buf) return GV_ERR_NOMEM;
    IterBufs b = carve_iter(buf, n, parts);
    char *p = (char *)buf + iter_bytes(n, parts);
    float *rinv = (float *)p; p += (size_t)n * 4;
    uint32_t *indeg = (uint32_t *)p; p += (size_t)n * 4;
    uint32_t *cursor = (uint32_t *)p; p += (size_t)n * 4;
    p = (char *)(((uintptr_t)p + 255) & ~(uintptr_t)255);
    unsigned long long *toff = (unsigned long long *)p; p += ((size_t)n + 1) * 8;
    uint32_t *tsrc = (uint32_t *)p; p += (live + 1) * 4;
    float *tw = (float *)p;
    uint32_t *heavy = cursor;  // list of vertices above WPR_HEAVY in-edges (n words)
    if (unit) GV_LAUNCH(k_row_inv_deg, grid_for(n, 256), 256, 0, s, d, rinv);
    else GV_LAUNCH(k_row_sums, grid_for(n, 256), 256, 0, s, d, rinv);
    {
        ProfScope ps(PROF_WPR_BUILD, s);
        // export (storage order), keys (v, u) with weight bits, stable radix sort by (v, u)
        const uint64_t E = live;
        const uint64_t rc = radix_counts_elems(std::max<uint64_t>(E, 1));
        const size_t o_off = 0, o_dst = o_off + (((size_t)n + 1) * 8 + 255) / 256 * 256;
        const size_t o_w = o_dst + (E * 4 + 255) / 256 * 256, o_k = o_w + (E * 4 + 255) / 256 * 256;
        const size_t o_k2 = o_k + (E * 8 + 255) / 256 * 256, o_v = o_k2 + (E * 8 + 255) / 256 * 256;
        const size_t o_v2 = o_v + (E * 4 + 255) / 256 * 256, o_c = o_v2 + (E * 4 + 255) / 256 * 256;
        const size_t o_t = o_c + (rc * 4 + 255) / 256 * 256;
        const size_t sbytes = o_t + scan_scratch_bytes(std::max<uint64_t>(rc, (uint64_t)n + 1)) + 256;
        char *sb = (char *)aux_scratch(g, 5, sbytes);
        if (!sb) return GV_ERR_NOMEM;
        unsigned long long *eoff = (unsigned long long *)(sb + o_off);
        uint32_t *edst = (uint32_t *)(sb + o_dst);
        float *ew = (float *)(sb + o_w);
        unsigned long long *k1 = (unsigned long long *)(sb + o_k), *k2 = (unsigned long long *)(sb + o_k2);
        uint32_t *v1 = (uint32_t *)(sb + o_v), *v2 = (uint32_t *)(sb + o_v2), *cnts = (uint32_t *)(sb + o_c);
        void *stmp = sb + o_t;
        launch_degrees(g, indeg, s);
        scan_exclusive_u32_to_u64(indeg, eoff, n, eoff + n, stmp, s);
        gv_status est = run_export(g, eoff, edst, unit ? nullptr : ew, s);
        if (est != GV_OK) return est;
        if (E) {
            GV_LAUNCH(k_wpr_keys, grid_for(E, 256, 148 * 16), 256, 0, s, (const unsigned long long *)eoff,
                      (const uint32_t *)edst, unit ? (const float *)nullptr : (const float *)ew, n, E, g->bitsn, k1, v1);
            const int which = radix_sort_u64(k1, k2, v1, v2, E, 2 * (int)g->bitsn, cnts, stmp, s);
            const unsigned long long *ks = which ? k2 : k1;
            GV_LAUNCH(k_wpr_unpack, grid_for(E, 256, 148 * 16), 256, 0, s, ks, which ? v2 : v1, E,
                      (1ull << g->bitsn) - 1, tsrc, tw);
            GV_LAUNCH(k_wpr_toff, grid_for((uint64_t)n + 1, 256), 256, 0, s, ks, E, n, g->bitsn, toff);
        } else {
            cudaMemsetAsync(toff, 0, ((size_t)n + 1) * 8, s);
        }
    }
    // count of the heavy list: the third word of the residual slot (the
    // sweeps write only its first 8 bytes)
    uint32_t *hcnt = reinterpret_cast<uint32_t *>(b.res) + 2;
    cudaMemsetAsync(hcnt, 0, 4, s);
    GV_LAUNCH(k_wpr_heavy_list, grid_for(n, 256), 256, 0, s, (const unsigned long long *)toff, n, heavy, hcnt);
    if (x_init) {
        cudaError_t ei = cudaMemcpyAsync(b.x0, x_init, (size_t)n * 4,
                                         init_mem == GV_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s);
        if (ei != cudaSuccess) return cuda_status(ei, "pagerank init");
    } else if (source == GV_NIL) {
        GV_LAUNCH(k_fill_f32, grid_for(n, 256), 256, 0, s, b.x0, n, 1.0f / (float)n, GV_NIL, 0.f);
    } else {
        GV_LAUNCH(k_fill_f32, grid_for(n, 256), 256, 0, s, b.x0, n, 0.f, source, 1.f);
    }
    cudaMemsetAsync(b.state, 0, 16, s);
    const uint32_t nparts = PULL_GRID + WPR_HEAVY_GRID;
    float *xa = b.x0, *xb = b.x1;
    int h_state[2] = {0, 0};
    int launched = 0;
    PullArgs a{};
    a.alpha = alpha;
    if (source == GV_NIL) {
        a.base_all = (1.0f - alpha) / (float)n;
        a.base_src = GV_NIL;
    } else {
        a.base_all = 0.f;
        a.base_src = source;
        a.base_src_val = 1.0f - alpha;
    }
    a.partial = b.partial;
    a.state = b.state;
    while (launched < max_iter) {
        const int chunk = std::min(8, max_iter - launched);
        for (int i = 0; i < chunk; ++i) {
            GV_LAUNCH(k_mul, grid_for(n, 256), 256, 0, s, (const float *)xa, (const float *)rinv, b.c0, n);
            a.gather = b.c0;
            a.xold = xa;
            a.xnew = xb;
            {
                ProfScope ps(PROF_WPR_SWEEP, s);
                dispatch_tpv(g->cfg.threads_per_vertex, [&](auto t) {
                    constexpr int T = decltype(t)::value;
                    GV_LAUNCH((k_wpr_fwd<T>), PULL_GRID, AN_THREADS, 0, s, n, (const unsigned long long *)toff,
                              (const uint32_t *)tsrc, (const float *)tw, a);
                });
                GV_LAUNCH(k_wpr_fwd_heavy, WPR_HEAVY_GRID, AN_THREADS, 0, s, (const unsigned long long *)toff,
                          (const uint32_t *)tsrc, (const float *)tw, (const uint32_t *)heavy, (const uint32_t *)hcnt, a,
                          PULL_GRID);
            }
            GV_LAUNCH(k_iter_done, 1, 256, 0, s, b.partial, nparts, tol, b.state, b.res);
            std::swap(xa, xb);
        }
        launched += chunk;
        cudaError_t e = cudaMemcpyAsync(h_state, b.state, 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e, "wpr forward");
        if (h_state[0]) break;
    }
    if (sweeps) *sweeps = h_state[1];
    return copy_out_f32((h_state[1] & 1) ? b.x1 : b.x0, x_out, n, mem, s);
}

}  // namespace
}  // namespace gv

extern "C" {

gv_status gv_wpr_forward(gv_graph *g, float alpha, float tol, int32_t max_iter, float *x_out, int32_t *sweeps, int mem,
                         void *stream) {
    if (!g || !x_out || max_iter < 0) return GV_ERR_INVALID;
    if (!g->cfg.weighted) { set_error("weighted PageRank needs a weighted store"); return GV_ERR_STATE; }
    return transpose_pagerank(g, alpha, tol, max_iter, false, nullptr, 0, GV_NIL, x_out, sweeps, mem,
                              (cudaStream_t)stream);
}

gv_status gv_wpr_backward(gv_graph *g, float alpha, float tol, int32_t max_iter, const float *x, const float *c,
                          int32_t mode, float *grad, uint64_t cap, float *lambda_out, int32_t *sweeps, int mem,
                          void *stream) {
    if (!g || !x || !c || max_iter < 0 || (mode != 0 && mode != 1)) return GV_ERR_INVALID;
    if (!g->cfg.weighted) { set_error("weighted PageRank needs a weighted store"); return GV_ERR_STATE; }
    cudaStream_t s = (cudaStream_t)stream;
    DevGraph d = g->d;
    const uint32_t n = d.n;
    uint64_t live = 0;
    {
        Ctl cc;
        gv_status st = read_ctl(g, &cc, s);
        if (st != GV_OK) return st;
        live = cc.live_edges;
    }
    if (grad && cap < live) { set_error("gradient capacity below the number of entries"); return GV_ERR_CAPACITY; }
    const uint32_t parts = SWEEP_PARTS;
    const size_t bytes = iter_bytes(n, parts) + (size_t)n * 4 * 4 + ((size_t)n + 1) * 8 + (live + 1) * 4 + 512;
    void *buf = analytics_scratch(g, bytes);
    if (!buf) return GV_ERR_NOMEM;
    IterBufs b = carve_iter(buf, n, parts);
    char *p = (char *)buf + iter_bytes(n, parts);
    float *rinv = (float *)p; p += (size_t)n * 4;
    float *dx = (float *)p; p += (size_t)n * 4;
    float *dc = (float *)p; p += (size_t)n * 4;
    uint32_t *deg = (uint32_t *)p; p += (size_t)n * 4;
    p = (char *)(((uintptr_t)p + 255) & ~(uintptr_t)255);
    unsigned long long *off = (unsigned long long *)p; p += ((size_t)n + 1) * 8;
    float *dgrad = (float *)p;
    const cudaMemcpyKind kin = mem == GV_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    cudaMemcpyAsync(dx, x, (size_t)n * 4, kin, s);
    cudaMemcpyAsync(dc, c, (size_t)n * 4, kin, s);
    GV_LAUNCH(k_row_sums, grid_for(n, 256), 256, 0, s, d, rinv);
    cudaMemcpyAsync(b.x0, dc, (size_t)n * 4, cudaMemcpyDeviceToDevice, s);  // lambda0 = c
    PullArgs a{};
    a.alpha = alpha;
    a.base_all = 0.f;
    a.base_src = GV_NIL;
    a.cvec = dc;
    a.rscale = rinv;
    int sw = 0;
    float *lam = nullptr;
    gv_status st = run_sweeps(g, s, b, a, true, rinv, tol, max_iter, false, &sw, &lam);
    if (st != GV_OK) return st;
    if (sweeps) *sweeps = sw;
    if (lambda_out) {
        st = copy_out_f32(lam, lambda_out, n, mem, s);
        if (st != GV_OK) return st;
    }
    if (!grad) return GV_OK;
    launch_degrees(g, deg, s);
    scan_exclusive_u32_to_u64(deg, off, n, off + n, g->bs.scan_tmp, s);
    float *gout = mem == GV_MEM_DEVICE ? grad : dgrad;
    if (live) {
        uint32_t *edst = (uint32_t *)aux_scratch(g, 5, live * 4 + 256);
        if (!edst) return GV_ERR_NOMEM;
        ProfScope ps(PROF_WPR_GRAD, s);
        st = run_export(g, off, edst, nullptr, s);
        if (st != GV_OK) return st;
        GV_LAUNCH(k_wpr_grad_flat, grid_for(live, 256, 148 * 16), 256, 0, s, (const unsigned long long *)off,
                  (const uint32_t *)edst, live, n, (const float *)dx, (const float *)lam, (const float *)dc,
                  (const float *)rinv, alpha, mode, gout);
    }
    cudaError_t e = cudaSuccess;
    if (mem != GV_MEM_DEVICE) e = cudaMemcpyAsync(grad, dgrad, live * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return cuda_status(e, "wpr gradient");
}

}  // extern "C"
