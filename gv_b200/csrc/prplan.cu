// PageRank over a sweep plan: the undirected store compiled, once per call,
// into a degree-ordered padded CSR that the sweeps read instead of walking
// the edge-block trees.
//
// Why: a pull sweep is bound by its gathers of the neighbours'
// contributions, not by the adjacency stream.  On R-MAT graphs those gathers
// concentrate on a few vertices (at scale 22 the 16 K highest-degree
// vertices receive 40% of them, the top 256 K 85%), but vertex ids scatter
// the hot values over the whole contribution vector, so every 32-byte sector
// the L1 keeps holds one hot value and seven cold ones.  The plan renumbers
// the vertices by descending degree class (stable in id order inside a
// class), so the hot contributions are contiguous: the top 16 K fit in 64 KB
// and stay in L1, the top 256 K in 1 MB of L2.  A row is the vertex's used
// slots in block order, tombstones and the padding to whole 16-byte quads
// written as a sentinel neighbour whose contribution is 0, so every load is
// an aligned uint4 and no tombstone or fill test remains; slot e of block k
// lands at k*B + e, so the blocks of a hub are copied in parallel.
//
// The plan: perm (new row -> vertex), inv (vertex -> new row), off[n+1]
// (uint32 row starts), col (neighbour rows, padded), the degree-class tier
// boundaries and the hub items.  Sweeps keep x and the contributions in plan
// order; the result is permuted back at the end.  Tiers by degree (rows are
// contiguous per tier): hubs of at least HUB_DEG entries are cut into items
// of ITEM_ENTRIES for one warp each (partials combined in item order), rows
// of WARP_DEG or more take a warp, rows of GROUP_DEG or more 8 lanes, the
// rest one thread; isolated rows take their value once and are not swept.
// One launch runs the four tiers, CTAs interleaved in
// proportion to their work; a finish kernel combines the hub partials and a
// one-CTA kernel sums the per-CTA residuals in a fixed order (deterministic).
//
// Same iteration as the store sweep (x0 = 1/n or the caller's start, L1 step
// < epsilon or max_iter, contributions x/deg, no dangling redistribution:
// src/algorithm/pagerank/pagerank.cu:3-68, pr_kernel.cu:3-48).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include "store.cuh"
#include "group.cuh"
#include "prims.cuh"
#include "launch.hpp"
#include "prof.hpp"

namespace gv {
namespace {

constexpr int PL_THREADS = 256;
constexpr uint32_t NCLASS = 34;        // degree classes: 0 (isolated), 1 + floor(log2 deg)
constexpr uint32_t PL_TILE = 4096;     // vertices per counting-sort tile
constexpr uint32_t HUB_DEG = 2048;     // rows with at least this many entries are cut into items
constexpr uint32_t ITEM_ENTRIES = 2048;
constexpr uint32_t WARP_DEG = 64;
constexpr uint32_t GROUP_DEG = 8;
constexpr unsigned PL_PERIOD = 16;
constexpr unsigned PL_WAVES_MAX = 148 * 128 / PL_PERIOD;
constexpr unsigned PL_GRID = PL_PERIOD * PL_WAVES_MAX;  // residual slots (the most CTAs a sweep launches)
constexpr unsigned PL_FIN = 148;

__device__ __forceinline__ uint32_t deg_class(uint32_t d) { return d ? 32u - __clz(d) : 0u; }

// ---------------------------------------------------------------- plan build
// Counting sort of the vertices by descending class, stable in id order:
// tile counts (class-major), a scan, then one warp per tile places its
// vertices in order.
__global__ void k_pl_count(DevGraph g, uint32_t ntiles, uint32_t *__restrict__ cnt) {
    __shared__ uint32_t h[NCLASS];
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        for (uint32_t i = threadIdx.x; i < NCLASS; i += blockDim.x) h[i] = 0;
        __syncthreads();
        const uint32_t v0 = t * PL_TILE, v1 = min(g.n, v0 + PL_TILE);
        for (uint32_t v = v0 + threadIdx.x; v < v1; v += blockDim.x)
            atomicAdd(&h[NCLASS - 1 - deg_class(g.vtx[v].z)], 1u);
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < NCLASS; i += blockDim.x) cnt[(size_t)i * ntiles + t] = h[i];
        __syncthreads();
    }
}

__global__ void k_pl_place(DevGraph g, uint32_t ntiles, const uint32_t *__restrict__ start,
                           uint32_t *__restrict__ perm, uint32_t *__restrict__ inv) {
    __shared__ uint32_t base[PL_THREADS / 32][NCLASS];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t t = blockIdx.x * (PL_THREADS / 32) + warp;
    if (t >= ntiles) return;
    for (uint32_t i = lane; i < NCLASS; i += 32) base[warp][i] = start[(size_t)i * ntiles + t];
    __syncwarp();
    const uint32_t v0 = t * PL_TILE, v1 = min(g.n, v0 + PL_TILE);
    for (uint32_t r = v0; r < v1; r += 32) {
        const uint32_t v = r + lane;
        const bool ok = v < v1;
        const uint32_t c = ok ? NCLASS - 1 - deg_class(g.vtx[v].z) : NCLASS;  // NCLASS: no vertex
        const uint32_t peers = __match_any_sync(GV_FULL_MASK, c);
        const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
        const uint32_t leader = __ffs(peers) - 1;
        uint32_t pos = 0;
        if (ok) pos = base[warp][c] + rank;
        __syncwarp();
        if (ok && lane == leader) base[warp][c] += __popc(peers);
        __syncwarp();
        if (ok) {
            perm[pos] = v;
            inv[v] = pos;
        }
    }
}

// class starts (first row of each class) from the scanned counts
__global__ void k_pl_class_starts(const uint32_t *__restrict__ start, uint32_t ntiles, uint32_t *__restrict__ out) {
    const uint32_t i = threadIdx.x;
    if (i < NCLASS) out[i] = start[(size_t)i * ntiles];
}

// Padded row lengths in plan order: a row holds the vertex's used slots
// (tombstones included, as the sentinel) rounded up to whole quads, so slot e
// of block k lands at k*B + e of the row and blocks are copied independently.
// Also the inverse live degrees and, per row of two or more blocks, its
// number of 32-block copy items.
__global__ void k_pl_rowlen(DevGraph g, const uint32_t *__restrict__ perm, uint32_t *__restrict__ plen,
                            float *__restrict__ rdeg, uint32_t *__restrict__ fitems) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
        const uint4 rec = g.vtx[perm[i]];
        plen[i] = (rec.y + 3u) & ~3u;
        rdeg[i] = rec.z ? 1.0f / (float)rec.z : 0.f;
        const uint32_t nb = blocks_for(rec.y, g.logB);
        fitems[i] = nb > 1 ? (nb + 31u) >> 5 : 0u;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) rdeg[g.n] = 0.f;
}

__device__ __forceinline__ uint32_t pl_map(uint32_t e, uint32_t slot, uint32_t fill, const uint32_t *__restrict__ inv,
                                           uint32_t n) {
    return (slot < fill && e != GV_TOMB) ? inv[e] : n;
}

// Rows of at most one block: 8 lanes per row copy its quads, neighbours
// renumbered, tombstones and the padding as the sentinel n.
__global__ void k_pl_fill_small(DevGraph g, const uint32_t *__restrict__ perm, const uint32_t *__restrict__ inv,
                                const uint32_t *__restrict__ off, uint32_t *__restrict__ col) {
    Group<8> G;
    const uint32_t ng = gridDim.x * (blockDim.x / 8);
    for (uint32_t i = blockIdx.x * (blockDim.x / 8) + threadIdx.x / 8; i < g.n; i += ng) {
        const uint4 rec = g.vtx[perm[i]];
        if (rec.y > g.B) continue;  // the copy items take it
        const uint32_t o = off[i], nq = (off[i + 1] - o) >> 2;
        const uint4 *src = reinterpret_cast<const uint4 *>(g.pool + ((size_t)rec.x << g.logB));
        uint4 *dst = reinterpret_cast<uint4 *>(col + o);
        for (uint32_t q = G.gl; q < nq; q += 8) {
            const uint4 v = src[q];
            const uint32_t e = q << 2;
            dst[q] = make_uint4(pl_map(v.x, e, rec.y, inv, g.n), pl_map(v.y, e + 1, rec.y, inv, g.n),
                                pl_map(v.z, e + 2, rec.y, inv, g.n), pl_map(v.w, e + 3, rec.y, inv, g.n));
        }
    }
}

// Rows of two or more blocks: a warp per item of 32 blocks, the lanes walk
// the tree to one block each, then copy the blocks quad by quad.
__global__ void k_pl_fill_items(DevGraph g, const uint32_t *__restrict__ perm, const uint32_t *__restrict__ inv,
                                const uint32_t *__restrict__ off, const uint32_t *__restrict__ frow,
                                const uint32_t *__restrict__ ffirst, uint32_t nitems, uint32_t *__restrict__ col) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nw = gridDim.x * (blockDim.x >> 5);
    const uint32_t qpb = g.B >> 2;  // quads per block
    for (uint32_t it = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); it < nitems; it += nw) {
        const uint32_t r = frow[it];
        const uint4 rec = g.vtx[perm[r]];
        const uint32_t nb = blocks_for(rec.y, g.logB);
        const uint32_t kb0 = (it - ffirst[r]) << 5;
        const uint32_t k = kb0 + lane;
        const uint32_t myb = k < nb ? (k == 0 ? rec.x : cbt_block(g.left, g.right, rec.x, k)) : GV_NIL;
        const uint32_t o = off[r];
        const uint32_t nk = min(32u, nb - kb0);
        for (uint32_t j = 0; j < nk; ++j) {
            const uint32_t b = __shfl_sync(GV_FULL_MASK, myb, j);
            const uint32_t kk = kb0 + j;
            const uint32_t e0 = kk << g.logB;
            const uint32_t quads = (min(g.B, rec.y - e0) + 3u) >> 2;
            const uint4 *src = reinterpret_cast<const uint4 *>(g.pool + ((size_t)b << g.logB));
            uint4 *dst = reinterpret_cast<uint4 *>(col + o + e0);
            for (uint32_t q = lane; q < quads; q += 32) {
                const uint4 v = src[q];
                const uint32_t e = e0 + (q << 2);
                dst[q] = make_uint4(pl_map(v.x, e, rec.y, inv, g.n), pl_map(v.y, e + 1, rec.y, inv, g.n),
                                    pl_map(v.z, e + 2, rec.y, inv, g.n), pl_map(v.w, e + 3, rec.y, inv, g.n));
            }
        }
        (void)qpb;
    }
}

// hub items: per hub row its item count, then item -> row
__global__ void k_pl_item_count(const uint32_t *__restrict__ off, uint32_t nhub, uint32_t *__restrict__ icnt) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nhub; i += gridDim.x * blockDim.x)
        icnt[i] = (off[i + 1] - off[i] + ITEM_ENTRIES - 1) / ITEM_ENTRIES;
}

__global__ void k_pl_item_fill(const uint32_t *__restrict__ ifirst, uint32_t nhub, uint32_t *__restrict__ irow) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nhub; i += gridDim.x * blockDim.x)
        for (uint32_t k = ifirst[i]; k < ifirst[i + 1]; ++k) irow[k] = i;
}

// x0 in plan order (from the caller's start, or 1/n, or the source), its
// contributions; x_out in vertex order at the end
// Isolated rows [rz, n) take their final value (the base, plus the source
// term) in both iterate buffers here and are left out of the sweeps.
__global__ void k_pl_init(uint32_t n, const uint32_t *__restrict__ perm, const float *__restrict__ xin,
                          float fill, uint32_t src_row, float src_val, const float *__restrict__ rdeg,
                          uint32_t rz, float base, float src_base, float *__restrict__ x, float *__restrict__ c,
                          float *__restrict__ x_other, float *__restrict__ c_other) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) {
        if (i == n) {
            x[n] = 0.f;
            c[n] = 0.f;
            c_other[n] = 0.f;
            continue;
        }
        if (i >= rz) {
            const float v = base + (i == src_row ? src_base : 0.f);
            x[i] = v;
            x_other[i] = v;
            c[i] = 0.f;
            c_other[i] = 0.f;
            continue;
        }
        const float v = xin ? xin[perm[i]] : (i == src_row ? src_val : fill);
        x[i] = v;
        c[i] = v * rdeg[i];
    }
}

__global__ void k_pl_out(uint32_t n, const uint32_t *__restrict__ inv, const float *__restrict__ x,
                         float *__restrict__ out) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) out[v] = x[inv[v]];
}

// ------------------------------------------------------------------- sweeps
struct PlanSweep {
    const uint32_t *off, *col, *irow, *ifirst;
    const float *rdeg;
    const float *gather;  // contributions, plan order, [n] = 0
    const float *xold;
    float *xnew, *cnew;
    float *ipart;
    double *partial;
    const int *state;
    float alpha, base;
    uint32_t src_row;     // personalised source (plan order) or GV_NIL
    float src_val;
    uint32_t rH, rW, rG, rZ, n, nitems;  // tier row boundaries; rows [rZ, n) are isolated
    uint32_t split;       // CTAs per period: items | warp << 8 | group << 16 | thread << 24
};

__device__ __forceinline__ float gather4(const float *__restrict__ c, uint4 q) {
    return (__ldg(c + q.x) + __ldg(c + q.y)) + (__ldg(c + q.z) + __ldg(c + q.w));
}

__device__ __forceinline__ void pl_finish(const PlanSweep &a, uint32_t i, float sum, double &res) {
    float b = a.base + (i == a.src_row ? a.src_val : 0.f);
    const float xv = b + a.alpha * sum;
    a.xnew[i] = xv;
    a.cnew[i] = xv * a.rdeg[i];
    res += (double)fabsf(xv - a.xold[i]);
}

// hub items: a warp per item of ITEM_ENTRIES entries, four quads per lane in flight
__device__ __forceinline__ void pl_items(const PlanSweep &a, uint32_t vb, uint32_t vg) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nw = vg * (PL_THREADS / 32);
    for (uint32_t it = vb * (PL_THREADS / 32) + (threadIdx.x >> 5); it < a.nitems; it += nw) {
        const uint32_t r = a.irow[it];
        const uint32_t k = it - a.ifirst[r];
        const uint32_t e0 = a.off[r] + k * ITEM_ENTRIES;
        const uint32_t e1 = min(a.off[r + 1], e0 + ITEM_ENTRIES);
        const uint4 *q = reinterpret_cast<const uint4 *>(a.col + e0);
        const uint32_t nq = (e1 - e0) >> 2;
        float sum = 0.f;
        for (uint32_t j = lane; j < nq; j += 128) {
            uint4 v0 = __ldcs(q + j), v1 = make_uint4(a.n, a.n, a.n, a.n), v2 = v1, v3 = v1;
            if (j + 32 < nq) v1 = __ldcs(q + j + 32);
            if (j + 64 < nq) v2 = __ldcs(q + j + 64);
            if (j + 96 < nq) v3 = __ldcs(q + j + 96);
            sum += (gather4(a.gather, v0) + gather4(a.gather, v1)) + (gather4(a.gather, v2) + gather4(a.gather, v3));
        }
        sum = warp_sum(sum);
        if (lane == 0) a.ipart[it] = sum;
    }
}

// rows of TPV lanes each over [r0, r1): quads strided by TPV, QF of them
// (4 QF gathers) in flight per lane
template <int TPV, int QF>
__device__ __forceinline__ void pl_rows(const PlanSweep &a, uint32_t r0, uint32_t r1, uint32_t vb, uint32_t vg,
                                        double &res) {
    Group<TPV> G;
    constexpr uint32_t GPC = PL_THREADS / TPV;
    const uint32_t ng = vg * GPC;
    for (uint32_t i = r0 + vb * GPC + threadIdx.x / TPV; i < r1; i += ng) {
        const uint32_t o = a.off[i];
        const uint32_t nq = (a.off[i + 1] - o) >> 2;
        const uint4 *q = reinterpret_cast<const uint4 *>(a.col + o);
        float sum = 0.f;
        for (uint32_t j = G.gl; j < nq; j += QF * TPV) {
            uint4 v[QF];
#pragma unroll
            for (int t = 0; t < QF; ++t)
                v[t] = (j + t * TPV < nq) ? __ldcs(q + j + t * TPV) : make_uint4(a.n, a.n, a.n, a.n);
            float part = 0.f;
#pragma unroll
            for (int t = 0; t < QF; ++t) part += gather4(a.gather, v[t]);
            sum += part;
        }
        if (TPV > 1) sum = G.sum(sum);
        if (G.gl == 0) pl_finish(a, i, sum, res);
    }
}

__global__ void __launch_bounds__(PL_THREADS) k_pl_sweep(PlanSweep a) {
    __shared__ double red[PL_THREADS / 32];
    if (a.state[0]) return;
    const uint32_t t0 = a.split & 0xFFu, t1 = (a.split >> 8) & 0xFFu, t2 = (a.split >> 16) & 0xFFu,
                   t3 = (a.split >> 24) & 0xFFu;
    const uint32_t r = blockIdx.x % PL_PERIOD, w = blockIdx.x / PL_PERIOD, waves = gridDim.x / PL_PERIOD;
    double res = 0.0;
    if (r < t0) pl_items(a, w * t0 + r, waves * t0);
    else if (r < t0 + t1) pl_rows<32, 4>(a, a.rH, a.rW, w * t1 + (r - t0), waves * t1, res);
    else if (r < t0 + t1 + t2) pl_rows<8, 2>(a, a.rW, a.rG, w * t2 + (r - t0 - t1), waves * t2, res);
    else pl_rows<1, 2>(a, a.rG, a.rZ, w * t3 + (r - t0 - t1 - t2), waves * t3, res);
    res = warp_sum(res);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = res;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < PL_THREADS / 32; ++i) s += red[i];
        a.partial[blockIdx.x] = s;
    }
}

// hub rows: their item partials in item order
__global__ void __launch_bounds__(PL_THREADS) k_pl_hub_fin(PlanSweep a, uint32_t part_base) {
    __shared__ double red[PL_THREADS / 32];
    if (a.state[0]) return;
    double res = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.rH; i += gridDim.x * blockDim.x) {
        float t = 0.f;
        for (uint32_t k = a.ifirst[i]; k < a.ifirst[i + 1]; ++k) t += a.ipart[k];
        pl_finish(a, i, t, res);
    }
    res = warp_sum(res);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = res;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < PL_THREADS / 32; ++i) s += red[i];
        a.partial[part_base + blockIdx.x] = s;
    }
}

// sums the per-CTA residuals in a fixed order; latches convergence
__global__ void k_pl_done(const double *__restrict__ partial, uint32_t nparts, float eps, int *state) {
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
        state[1] += 1;
        if (s < (double)eps) state[0] = 1;
    }
}

// CTAs per period for the four tiers in proportion to their work (entries
// plus a per-row cost of 16 entries); a tier with work gets at least one.
uint32_t plan_split(const double w[4]) {
    double tot = w[0] + w[1] + w[2] + w[3];
    uint32_t t[4] = {0, 0, 0, 0}, sum = 0;
    if (tot <= 0) return 1u | (1u << 8) | (1u << 16) | (13u << 24);
    for (int i = 0; i < 4; ++i) {
        t[i] = w[i] > 0 ? std::max<uint32_t>(1, (uint32_t)(PL_PERIOD * w[i] / tot + 0.5)) : 0;
        sum += t[i];
    }
    int big = 0;
    for (int i = 1; i < 4; ++i)
        if (t[i] > t[big]) big = i;
    while (sum > PL_PERIOD) { --t[big]; --sum; }
    while (sum < PL_PERIOD) { ++t[big]; ++sum; }
    return t[0] | (t[1] << 8) | (t[2] << 16) | (t[3] << 24);
}

template <typename T>
T *carve(char *&p, size_t count) {
    T *r = reinterpret_cast<T *>(p);
    p += ((count * sizeof(T)) + 255) & ~(size_t)255;
    return r;
}

}  // namespace

bool plan_pagerank_enabled(gv_graph *g) {
    if (g->cfg.directed || g->cfg.weighted) return false;
    const char *env = std::getenv("GV_PR_PLAN");
    return !(env && env[0] == '0');
}

gv_status plan_pagerank(gv_graph *g, float alpha, float eps, int max_iter, const float *x_init, int init_mem,
                        uint32_t source, float *x_out, int32_t *sweeps, int mem, cudaStream_t s,
                        bool *planned) {
    *planned = false;
    DevGraph d = g->d;
    const uint32_t n = d.n;
    Ctl cc;
    gv_status st = read_ctl(g, &cc, s);
    if (st != GV_OK) return st;
    // rows hold the used slots (at most the used blocks' slots) plus padding
    const uint64_t padded_max = (d.P - cc.free_top) * (uint64_t)d.B + 3ull * n;
    if (padded_max >= 0xFFFFFFF0ull || n == 0) return GV_OK;  // uint32 row starts: the store sweep serves it
    const uint32_t ntiles = (n + PL_TILE - 1) / PL_TILE;
    // scratch: plan arrays (aux slot 12), padded columns (13), copy items (14), hub items (15)
    const size_t plan_bytes = (size_t)5 * 256 + ((size_t)NCLASS * ntiles + 1) * 4 + (size_t)n * 4 * 2 +
                              ((size_t)n + 1) * 4 * 3 + ((size_t)n + 1) * 4 * 4 + (size_t)(NCLASS + 8) * 4 +
                              ((size_t)n + 1) * 8 + (size_t)PL_GRID * 8 + PL_FIN * 8 + 64 + 16 * 256 +
                              (size_t)n * 4;
    char *p = (char *)aux_scratch(g, 12, plan_bytes);
    if (!p) return GV_ERR_NOMEM;
    uint32_t *cnt = carve<uint32_t>(p, (size_t)NCLASS * ntiles + 1);
    uint32_t *perm = carve<uint32_t>(p, n);
    uint32_t *inv = carve<uint32_t>(p, n);
    uint32_t *off = carve<uint32_t>(p, (size_t)n + 1);
    uint32_t *ifirst = carve<uint32_t>(p, (size_t)n + 1);
    float *rdeg = carve<float>(p, (size_t)n + 1);
    float *x0 = carve<float>(p, (size_t)n + 1);
    float *x1 = carve<float>(p, (size_t)n + 1);
    float *c0 = carve<float>(p, (size_t)n + 1);
    float *c1 = carve<float>(p, (size_t)n + 1);
    uint32_t *cls = carve<uint32_t>(p, NCLASS + 8);
    double *partial = carve<double>(p, PL_GRID + PL_FIN);
    int *state = carve<int>(p, 16);
    float *xstage = carve<float>(p, n);  // a host start vector, vertex order
    // class order of the rows
    GV_LAUNCH(k_pl_count, std::min<uint32_t>(ntiles, 148 * 8), PL_THREADS, 0, s, d, ntiles, cnt);
    scan_exclusive_u32(cnt, cnt, (uint64_t)NCLASS * ntiles, cnt + (size_t)NCLASS * ntiles, g->bs.scan_tmp, s);
    GV_LAUNCH(k_pl_place, (ntiles + PL_THREADS / 32 - 1) / (PL_THREADS / 32), PL_THREADS, 0, s, d, ntiles,
              (const uint32_t *)cnt, perm, inv);
    GV_LAUNCH(k_pl_class_starts, 1, 64, 0, s, (const uint32_t *)cnt, ntiles, cls);
    // row lengths, starts, inverse degrees, copy items of the multi-block rows
    uint32_t *ffirst = ifirst;  // free until the hub items are built
    GV_LAUNCH(k_pl_rowlen, grid_for(n, 256), 256, 0, s, d, (const uint32_t *)perm, off, rdeg, ffirst);
    scan_exclusive_u32(off, off, n, off + n, g->bs.scan_tmp, s);
    scan_exclusive_u32(ffirst, ffirst, n, ffirst + n, g->bs.scan_tmp, s);
    uint32_t hcls[NCLASS], total = 0, nfill = 0;
    cudaMemcpyAsync(hcls, cls, NCLASS * 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&total, off + n, 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&nfill, ffirst + n, 4, cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "plan classes");
    // rows of class c hold degrees [2^(c-1), 2^c); classes run in descending order:
    // row boundaries of the tiers from the class starts
    auto first_row_below = [&](uint32_t deg) {  // first row whose degree is < deg (deg a power of two)
        const uint32_t c = 32u - (uint32_t)__builtin_clz(deg);  // class of deg itself
        return hcls[NCLASS - c];                                  // start of class c - 1
    };
    const uint32_t rH = first_row_below(HUB_DEG), rW = first_row_below(WARP_DEG), rG = first_row_below(GROUP_DEG);
    const uint32_t rZ = hcls[NCLASS - 1];  // first isolated row (class 0 comes last)
    // the padded, renumbered columns, straight from the store's blocks
    uint32_t *col = (uint32_t *)aux_scratch(g, 13, ((size_t)total + 4) * 4 + 256);
    uint32_t *frow = (uint32_t *)aux_scratch(g, 14, ((size_t)nfill + 1) * 4 + 256);
    if (!col || !frow) return GV_ERR_NOMEM;
    GV_LAUNCH(k_pl_fill_small, 148 * 16, PL_THREADS, 0, s, d, (const uint32_t *)perm, (const uint32_t *)inv,
              (const uint32_t *)off, col);
    if (nfill) {
        GV_LAUNCH(k_pl_item_fill, grid_for(n, 256), 256, 0, s, (const uint32_t *)ffirst, n, frow);
        GV_LAUNCH(k_pl_fill_items, 148 * 16, PL_THREADS, 0, s, d, (const uint32_t *)perm, (const uint32_t *)inv,
                  (const uint32_t *)off, (const uint32_t *)frow, (const uint32_t *)ffirst, nfill, col);
    }
    // hub items
    uint32_t nitems = 0;
    uint32_t *irow = nullptr;
    float *ipart = nullptr;
    if (rH) {
        GV_LAUNCH(k_pl_item_count, grid_for(rH, 256), 256, 0, s, (const uint32_t *)off, rH, ifirst);
        scan_exclusive_u32(ifirst, ifirst, rH, ifirst + rH, g->bs.scan_tmp, s);
        cudaMemcpyAsync(&nitems, ifirst + rH, 4, cudaMemcpyDeviceToHost, s);
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e, "plan items");
        char *q = (char *)aux_scratch(g, 15, (size_t)nitems * 8 + 512);
        if (!q) return GV_ERR_NOMEM;
        irow = carve<uint32_t>(q, nitems);
        ipart = carve<float>(q, nitems);
        GV_LAUNCH(k_pl_item_fill, grid_for(rH, 256), 256, 0, s, (const uint32_t *)ifirst, rH, irow);
    }
    // start vector
    uint32_t src_row = GV_NIL;
    if (source != GV_NIL) cudaMemcpyAsync(&src_row, inv + source, 4, cudaMemcpyDeviceToHost, s);
    uint32_t hoff[4] = {0, 0, 0, 0};
    const uint32_t rows[4] = {rH, rW, rG, rZ};
    for (int i = 0; i < 4; ++i) cudaMemcpyAsync(&hoff[i], off + rows[i], 4, cudaMemcpyDeviceToHost, s);
    const float *xin = nullptr;
    if (x_init) {
        if (init_mem == GV_MEM_DEVICE) xin = x_init;
        else {
            e = cudaMemcpyAsync(xstage, x_init, (size_t)n * 4, cudaMemcpyHostToDevice, s);
            if (e != cudaSuccess) return cuda_status(e, "pagerank init");
            xin = xstage;
        }
    }
    e = cudaStreamSynchronize(s);  // src_row, tier row starts
    if (e != cudaSuccess) return cuda_status(e, "plan source");
    const float fill = source == GV_NIL ? 1.0f / (float)n : 0.f;
    // x0 and its contributions in plan order; the isolated rows, which the
    // sweeps never reach, get their value in x1 too
    const float base = source == GV_NIL ? (1.0f - alpha) / (float)n : 0.f;
    GV_LAUNCH(k_pl_init, grid_for((uint64_t)n + 1, 256), 256, 0, s, n, (const uint32_t *)perm, xin, fill, src_row,
              1.f, (const float *)rdeg, rZ, base, source == GV_NIL ? 0.f : 1.0f - alpha, x0, c0, x1, c1);
    cudaMemsetAsync(state, 0, 16, s);
    cudaMemsetAsync(partial, 0, (PL_GRID + PL_FIN) * 8, s);
    // tier work (entries + 16 per row) from the row starts read back above
    const double w[4] = {(double)hoff[0], (double)(hoff[1] - hoff[0]) + 16.0 * (rW - rH),
                         (double)(hoff[2] - hoff[1]) + 16.0 * (rG - rW), (double)(hoff[3] - hoff[2]) + 16.0 * (rZ - rG)};
    // the sweep uses little shared memory: give the SM's on-chip memory to L1,
    // where the hot contributions live
    cudaFuncSetAttribute(k_pl_sweep, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
    cudaGetLastError();
    PlanSweep a{};
    a.off = off;
    a.col = col;
    a.irow = irow;
    a.ifirst = ifirst;
    a.rdeg = rdeg;
    a.partial = partial;
    a.state = state;
    a.ipart = ipart;
    a.alpha = alpha;
    a.base = base;
    a.src_row = src_row;
    a.src_val = source == GV_NIL ? 0.f : 1.0f - alpha;
    a.rH = rH;
    a.rW = rW;
    a.rG = rG;
    a.rZ = rZ;
    a.n = n;
    a.nitems = nitems;
    a.split = plan_split(w);
    // CTAs of the sweep: rounds of PL_PERIOD; GV_PL_WAVES overrides the number of rounds
    // eight waves of 8 resident CTAs per SM: at R-MAT scale 22 a sweep takes
    // 0.309 ms with eight, 0.314 with six, 0.325 with four, 0.359 with two and
    // 0.406 with one (smaller CTA shares even out the tiers' tails)
    unsigned waves = 148 * 64 / PL_PERIOD;
    if (const char *env = std::getenv("GV_PL_WAVES")) {
        const unsigned w = (unsigned)std::strtoul(env, nullptr, 10);
        if (w >= 1 && w <= PL_WAVES_MAX) waves = w;
    }
    const unsigned grid = waves * PL_PERIOD;
    float *xa = x0, *xb = x1, *ca = c0, *cb = c1;
    int h_state[2] = {0, 0};
    int launched = 0;
    while (launched < max_iter) {
        const int chunk = std::min(8, max_iter - launched);
        for (int i = 0; i < chunk; ++i) {
            a.gather = ca;
            a.xold = xa;
            a.xnew = xb;
            a.cnew = cb;
            {
                ProfScope ps(PROF_PULL, s);
                GV_LAUNCH(k_pl_sweep, grid, PL_THREADS, 0, s, a);
                if (rH) GV_LAUNCH(k_pl_hub_fin, PL_FIN, PL_THREADS, 0, s, a, grid);
            }
            GV_LAUNCH(k_pl_done, 1, 256, 0, s, (const double *)partial, grid + PL_FIN, eps, state);
            std::swap(xa, xb);
            std::swap(ca, cb);
        }
        launched += chunk;
        e = cudaMemcpyAsync(h_state, state, 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e, "plan sweeps");
        if (h_state[0]) break;
    }
    // sweep i (1-based) wrote x1 when i is odd
    const float *res = (h_state[1] & 1) ? x1 : x0;
    float *dst = mem == GV_MEM_DEVICE ? x_out : (h_state[1] & 1) ? x0 : x1;  // the other buffer is free
    GV_LAUNCH(k_pl_out, grid_for(n, 256), 256, 0, s, n, (const uint32_t *)inv, res, dst);
    if (mem != GV_MEM_DEVICE) e = cudaMemcpyAsync(x_out, dst, (size_t)n * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "plan out");
    g->last_sweeps = h_state[1];
    if (sweeps) *sweeps = h_state[1];
    *planned = true;
    return cuda_status(cudaGetLastError(), "plan pagerank");
}

}  // namespace gv
