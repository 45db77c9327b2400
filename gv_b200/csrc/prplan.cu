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
// (4 QF gathers) in flight per lane.  Rows of a group or a thread (TPV < 32)
// are short, so a row's dependent loads (bounds, quads, gathers, finish)
// would each wait in turn: the next row's bounds and first quads are loaded
// while this row's gathers are in flight.  Sums are formed in the same order
// either way.
template <int TPV, int QF>
__device__ __forceinline__ void pl_rows(const PlanSweep &a, uint32_t r0, uint32_t r1, uint32_t vb, uint32_t vg,
                                        double &res) {
    Group<TPV> G;
    constexpr uint32_t GPC = PL_THREADS / TPV;
    const uint32_t ng = vg * GPC;
    const uint4 sent = make_uint4(a.n, a.n, a.n, a.n);
    uint32_t i = r0 + vb * GPC + threadIdx.x / TPV;
    if constexpr (TPV == 32) {
        for (; i < r1; i += ng) {
            const uint32_t o = a.off[i];
            const uint32_t nq = (a.off[i + 1] - o) >> 2;
            const uint4 *q = reinterpret_cast<const uint4 *>(a.col + o);
            float sum = 0.f;
            for (uint32_t j = G.gl; j < nq; j += QF * TPV) {
                uint4 v[QF];
#pragma unroll
                for (int t = 0; t < QF; ++t) v[t] = (j + t * TPV < nq) ? __ldcs(q + j + t * TPV) : sent;
                float part = 0.f;
#pragma unroll
                for (int t = 0; t < QF; ++t) part += gather4(a.gather, v[t]);
                sum += part;
            }
            sum = G.sum(sum);
            if (G.gl == 0) pl_finish(a, i, sum, res);
        }
    } else {
        uint32_t o = 0, nq = 0;
        if (i < r1) {
            o = a.off[i];
            nq = (a.off[i + 1] - o) >> 2;
        }
        uint4 v[QF];
#pragma unroll
        for (int t = 0; t < QF; ++t)
            v[t] = (G.gl + t * TPV < nq) ? __ldcs(reinterpret_cast<const uint4 *>(a.col + o) + G.gl + t * TPV) : sent;
        while (i < r1) {
            const uint32_t in = i + ng;
            uint32_t on = 0, nqn = 0;
            if (in < r1) {
                on = a.off[in];
                nqn = (a.off[in + 1] - on) >> 2;
            }
            float sum = 0.f;
            {
                float part = 0.f;
#pragma unroll
                for (int t = 0; t < QF; ++t) part += gather4(a.gather, v[t]);
                sum += part;
            }
            const uint4 *q = reinterpret_cast<const uint4 *>(a.col + o);
            for (uint32_t j = G.gl + QF * TPV; j < nq; j += QF * TPV) {
                uint4 w[QF];
#pragma unroll
                for (int t = 0; t < QF; ++t) w[t] = (j + t * TPV < nq) ? __ldcs(q + j + t * TPV) : sent;
                float part = 0.f;
#pragma unroll
                for (int t = 0; t < QF; ++t) part += gather4(a.gather, w[t]);
                sum += part;
            }
            const uint4 *qn = reinterpret_cast<const uint4 *>(a.col + on);
#pragma unroll
            for (int t = 0; t < QF; ++t) v[t] = (G.gl + t * TPV < nqn) ? __ldcs(qn + G.gl + t * TPV) : sent;
            if (TPV > 1) sum = G.sum(sum);
            if (G.gl == 0) pl_finish(a, i, sum, res);
            i = in;
            o = on;
            nq = nqn;
        }
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

// ------------------------------------------------ batched PPR over the plan
// k personalised queries (2 <= k <= 32) share every adjacency read of a
// sweep.  Values are row-major in plan order with a power-of-two stride K >= k
// (x[row * K + q]), so the k contributions of one neighbour are one aligned
// load of at most 128 bytes.  A group of K lanes owns a row (lane q = query
// q); 32 / K groups share a warp.  Rows of WARP_DEG or more entries take the
// whole warp (groups interleave over the entries, then combine), hub rows are
// cut into the single sweep's items.  Entries are summed in row order inside a
// group and the groups combine in a fixed butterfly, so results repeat bit
// for bit.  Same iteration as the store's batched sweep (one lane per query,
// residual per query, every query under epsilon to stop).
struct PlanBatch {
    const uint32_t *off, *col, *irow, *ifirst;
    const float *rdeg;
    const float *gather;  // contributions [(n + 1) K], plan order
    const float *xold;
    float *xnew, *cnew;
    float *ipart;         // [nitems][K]
    double *partial;      // [CTA][32]
    const int *state;
    const uint32_t *srow; // [32]: query q's source row, GV_NIL past k
    float alpha, src_val;
    uint32_t k, rH, rW, rZ, n, nitems;
    uint32_t split;       // CTAs per period: items | warp rows << 8 (the rest: group rows)
};

// Entries [e0, e1) by the whole warp: group g takes the entries at g K + t of
// each run of 32 (U runs in flight); returns, in every lane, the sum for its
// query over all the entries.
template <int K>
__device__ __forceinline__ float plk_warp_segment(const PlanBatch &a, uint32_t e0, uint32_t e1) {
    constexpr int U = K >= 8 ? 1 : 8 / K;
    const uint32_t lane = threadIdx.x & 31u, q = lane % K, grp = lane / K;
    const bool live = q < a.k;
    float acc = 0.f;
    for (uint32_t b = e0; b < e1; b += 32 * U) {
        uint32_t c[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t e = b + 32 * u + lane;
            c[u] = e < e1 ? __ldcs(a.col + e) : a.n;
        }
        float v[U][K];
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int t = 0; t < K; ++t) {
                const uint32_t ct = __shfl_sync(GV_FULL_MASK, c[u], grp * K + t);
                v[u][t] = (ct < a.n && live) ? __ldg(a.gather + (size_t)ct * K + q) : 0.f;
            }
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int t = 0; t < K; ++t) acc += v[u][t];
    }
#pragma unroll
    for (int o = K; o < 32; o <<= 1) acc += __shfl_xor_sync(GV_FULL_MASK, acc, o);
    return acc;
}

template <int K>
__device__ __forceinline__ void plk_finish(const PlanBatch &a, uint32_t r, uint32_t q, uint32_t my_src, float acc,
                                           double &res) {
    const float b = my_src == r ? a.src_val : 0.f;
    const float xv = b + a.alpha * acc;
    const size_t at = (size_t)r * K + q;
    a.xnew[at] = xv;
    a.cnew[at] = xv * a.rdeg[r];
    res += (double)fabsf(xv - a.xold[at]);
}

template <int K>
__device__ __forceinline__ void plk_items(const PlanBatch &a, uint32_t vb, uint32_t vg) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nw = vg * (PL_THREADS / 32);
    for (uint32_t it = vb * (PL_THREADS / 32) + (threadIdx.x >> 5); it < a.nitems; it += nw) {
        const uint32_t r = a.irow[it];
        const uint32_t e0 = a.off[r] + (it - a.ifirst[r]) * ITEM_ENTRIES;
        const uint32_t e1 = min(a.off[r + 1], e0 + ITEM_ENTRIES);
        const float acc = plk_warp_segment<K>(a, e0, e1);
        if (lane < K) a.ipart[(size_t)it * K + lane] = acc;
    }
}

template <int K>
__device__ __forceinline__ void plk_warp_rows(const PlanBatch &a, uint32_t my_src, uint32_t vb, uint32_t vg,
                                              double &res) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nw = vg * (PL_THREADS / 32);
    for (uint32_t r = a.rH + vb * (PL_THREADS / 32) + (threadIdx.x >> 5); r < a.rW; r += nw) {
        const float acc = plk_warp_segment<K>(a, a.off[r], a.off[r + 1]);
        if (lane < a.k) plk_finish<K>(a, r, lane, my_src, acc, res);
    }
}

// Rows [rW, rZ): a group of K lanes per row, 32 / K rows per warp; lane q
// loads entry j + u K + q of its row, the group's lanes take turns as the
// neighbour.
template <int K>
__device__ __forceinline__ void plk_group_rows(const PlanBatch &a, uint32_t my_src, uint32_t vb, uint32_t vg,
                                               double &res) {
    constexpr int U = K >= 8 ? 1 : 8 / K;
    constexpr uint32_t G = 32 / K;
    const uint32_t lane = threadIdx.x & 31u, q = lane % K, grp = lane / K;
    const bool live = q < a.k;
    const uint32_t nw = vg * (PL_THREADS / 32);
    for (uint32_t rb = a.rW + (vb * (PL_THREADS / 32) + (threadIdx.x >> 5)) * G; rb < a.rZ; rb += nw * G) {
        const uint32_t r = rb + grp;
        const bool ok = r < a.rZ;
        const uint32_t o = ok ? a.off[r] : 0u, len = ok ? a.off[r + 1] - o : 0u;
        const uint32_t most = __reduce_max_sync(GV_FULL_MASK, len);
        float acc = 0.f;
        for (uint32_t j = 0; j < most; j += K * U) {
            uint32_t c[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint32_t e = j + u * K + q;
                c[u] = e < len ? __ldcs(a.col + o + e) : a.n;
            }
            float v[U][K];
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int t = 0; t < K; ++t) {
                    const uint32_t ct = __shfl_sync(GV_FULL_MASK, c[u], grp * K + t);
                    v[u][t] = (ct < a.n && live) ? __ldg(a.gather + (size_t)ct * K + q) : 0.f;
                }
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int t = 0; t < K; ++t) acc += v[u][t];
        }
        if (ok && live) plk_finish<K>(a, r, q, my_src, acc, res);
    }
}

// Per-query residual of a CTA into partial[slot][0, K): lanes of one query
// are combined across warps, then across the groups of a warp (fixed orders).
template <int K>
__device__ __forceinline__ void plk_residual(double res, double *__restrict__ partial, uint32_t slot) {
    __shared__ double red[PL_THREADS / 32][32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    red[warp][lane] = res;
    __syncthreads();
    if (warp == 0) {
        double t = 0.0;
        for (int w = 0; w < PL_THREADS / 32; ++w) t += red[w][lane];
#pragma unroll
        for (int o = K; o < 32; o <<= 1) t += __shfl_xor_sync(GV_FULL_MASK, t, o);
        if (lane < K) partial[(size_t)slot * 32 + lane] = t;
    }
}

template <int K>
__device__ __forceinline__ void plk_sweep_body(const PlanBatch &a) {
    if (a.state[0]) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t my_src = a.srow[lane % K];
    const uint32_t t0 = a.split & 0xFFu, t1 = (a.split >> 8) & 0xFFu, t2 = PL_PERIOD - t0 - t1;
    const uint32_t r = blockIdx.x % PL_PERIOD, w = blockIdx.x / PL_PERIOD, waves = gridDim.x / PL_PERIOD;
    double res = 0.0;
    if (r < t0) plk_items<K>(a, w * t0 + r, waves * t0);
    else if (r < t0 + t1) plk_warp_rows<K>(a, my_src, w * t1 + (r - t0), waves * t1, res);
    else plk_group_rows<K>(a, my_src, w * t2 + (r - t0 - t1), waves * t2, res);
    plk_residual<K>(res, a.partial, blockIdx.x);
}

// One sweep.  16 and 32 queries are compiled for six resident CTAs (40
// registers, a few spilled): at R-MAT scale 25 that took their sweeps from
// 17.4 to 14.9 ms and from 31.6 to 26.4 ms; fewer queries keep the
// compiler's choice (32-40 registers; capped at 40, 4 queries went from 4.9
// to 5.4 ms).
template <int K>
__global__ void __launch_bounds__(PL_THREADS) k_plk_sweep(PlanBatch a) {
    plk_sweep_body<K>(a);
}

template <int K>
__global__ void __launch_bounds__(PL_THREADS, 6) k_plk_sweep_wide(PlanBatch a) {
    plk_sweep_body<K>(a);
}

// hub rows: a thread per (row, query), the row's item partials in item order
template <int K>
__global__ void __launch_bounds__(PL_THREADS) k_plk_hub_fin(PlanBatch a, uint32_t part_base) {
    if (a.state[0]) return;
    const uint32_t q = threadIdx.x % K;  // the stride is a multiple of K
    const uint32_t my_src = a.srow[q];
    double res = 0.0;
    const uint32_t total = a.rH * K;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const uint32_t r = i / K;
        if (q >= a.k) continue;
        float t = 0.f;
        for (uint32_t it = a.ifirst[r]; it < a.ifirst[r + 1]; ++it) t += a.ipart[(size_t)it * K + q];
        plk_finish<K>(a, r, q, my_src, t, res);
    }
    plk_residual<K>(res, a.partial, part_base + blockIdx.x);
}

// per query (a warp each): its residual slots summed lane-strided, then
// across the lanes in a fixed order; converged when every query is
__global__ void k_plk_done(const double *__restrict__ partial, uint32_t nparts, uint32_t k, float eps, int *state) {
    __shared__ int all_ok;
    if (state[0]) return;
    if (threadIdx.x == 0) all_ok = 1;
    __syncthreads();
    const uint32_t q = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    if (q < k) {
        double t = 0.0;
        for (uint32_t p = lane; p < nparts; p += 32) t += partial[(size_t)p * 32 + q];
        t = warp_sum(t);
        if (lane == 0 && !(t < (double)eps)) atomicAnd(&all_ok, 0);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        state[1] += 1;
        if (all_ok) state[0] = 1;
    }
}

// source rows of the k queries; GV_NIL in the unused slots
__global__ void k_plk_sources(const uint32_t *__restrict__ sources, uint32_t k, uint32_t n,
                              const uint32_t *__restrict__ inv, uint32_t *__restrict__ srow) {
    const uint32_t q = threadIdx.x;
    if (q >= 32) return;
    const uint32_t v = q < k ? sources[q] : GV_NIL;
    srow[q] = v < n ? inv[v] : GV_NIL;  // a source out of range matches no row
}

// x0 = the source indicator per query and its contributions; isolated rows
// [rz, n) take their final value in both iterate buffers; row n (the
// sentinel) is zero.  Lanes past k are never read.
template <int K>
__global__ void k_plk_init(uint32_t n, const uint32_t *__restrict__ srow, const float *__restrict__ rdeg, uint32_t rz,
                           float src_base, float *__restrict__ x, float *__restrict__ c, float *__restrict__ x_other,
                           float *__restrict__ c_other) {
    const size_t total = ((size_t)n + 1) * K;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t r = (uint32_t)(i / K), q = (uint32_t)(i % K);
        const bool src = srow[q] == r;
        if (r == n) {
            x[i] = c[i] = x_other[i] = c_other[i] = 0.f;
        } else if (r >= rz) {
            const float v = src ? src_base : 0.f;
            x[i] = x_other[i] = v;
            c[i] = c_other[i] = 0.f;
        } else {  // both buffers: lanes past k are read (and never used) by the vector loads
            const float v = src ? 1.f : 0.f;
            x[i] = x_other[i] = v;
            c[i] = c_other[i] = v * rdeg[r];
        }
    }
}

// x_out[v][q] (stride k, vertex order) from the plan-order rows
template <int K>
__global__ void k_plk_out(uint32_t n, uint32_t k, const uint32_t *__restrict__ inv, const float *__restrict__ x,
                          float *__restrict__ out) {
    const size_t total = (size_t)n * k;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t v = (uint32_t)(i / k), q = (uint32_t)(i % k);
        out[i] = x[(size_t)inv[v] * K + q];
    }
}

}  // namespace

bool plan_pagerank_enabled(gv_graph *g) {
    if (g->cfg.directed || g->cfg.weighted) return false;
    const char *env = std::getenv("GV_PR_PLAN");
    return !(env && env[0] == '0');
}

namespace {

// The plan of the store's current adjacency (see the top of this file).
struct Plan {
    uint32_t *perm, *inv, *off, *ifirst, *col, *irow;
    float *rdeg;
    float *ipart;      // nitems x the caller's width
    char *extra;       // the caller's bytes at the end of the plan scratch
    uint32_t nitems, rH, rW, rG, rZ;
    uint32_t hoff[4];  // row starts of rows rH, rW, rG, rZ
};

// Builds the plan into auxiliary slots 12-15 (plan arrays and extra_bytes,
// padded columns, copy items, hub items with ipart_width floats each).
// *ok is false, with nothing built, when the padded rows would not fit
// uint32 row starts.
gv_status plan_build(gv_graph *g, size_t extra_bytes, uint32_t ipart_width, cudaStream_t s, Plan &P, bool *ok) {
    *ok = false;
    DevGraph d = g->d;
    const uint32_t n = d.n;
    Ctl cc;
    gv_status st = read_ctl(g, &cc, s);
    if (st != GV_OK) return st;
    // rows hold the used slots (at most the used blocks' slots) plus padding
    const uint64_t padded_max = (d.P - cc.free_top) * (uint64_t)d.B + 3ull * n;
    if (padded_max >= 0xFFFFFFF0ull || n == 0) return GV_OK;  // uint32 row starts: the store sweep serves it
    const uint32_t ntiles = (n + PL_TILE - 1) / PL_TILE;
    // seven arrays, each carved to a 256-byte boundary, then the caller's bytes
    const size_t plan_bytes = (size_t)8 * 256 + ((size_t)NCLASS * ntiles + 1) * 4 + (size_t)n * 4 * 2 +
                              ((size_t)n + 1) * 4 * 3 + (size_t)(NCLASS + 8) * 4 + extra_bytes;
    char *p = (char *)aux_scratch(g, 12, plan_bytes);
    if (!p) return GV_ERR_NOMEM;
    uint32_t *cnt = carve<uint32_t>(p, (size_t)NCLASS * ntiles + 1);
    P.perm = carve<uint32_t>(p, n);
    P.inv = carve<uint32_t>(p, n);
    P.off = carve<uint32_t>(p, (size_t)n + 1);
    P.ifirst = carve<uint32_t>(p, (size_t)n + 1);
    P.rdeg = carve<float>(p, (size_t)n + 1);
    uint32_t *cls = carve<uint32_t>(p, NCLASS + 8);
    P.extra = p;
    uint32_t *perm = P.perm, *inv = P.inv, *off = P.off, *ifirst = P.ifirst;
    // class order of the rows
    GV_LAUNCH(k_pl_count, std::min<uint32_t>(ntiles, 148 * 8), PL_THREADS, 0, s, d, ntiles, cnt);
    scan_exclusive_u32(cnt, cnt, (uint64_t)NCLASS * ntiles, cnt + (size_t)NCLASS * ntiles, g->bs.scan_tmp, s);
    GV_LAUNCH(k_pl_place, (ntiles + PL_THREADS / 32 - 1) / (PL_THREADS / 32), PL_THREADS, 0, s, d, ntiles,
              (const uint32_t *)cnt, perm, inv);
    GV_LAUNCH(k_pl_class_starts, 1, 64, 0, s, (const uint32_t *)cnt, ntiles, cls);
    // row lengths, starts, inverse degrees, copy items of the multi-block rows
    uint32_t *ffirst = ifirst;  // free until the hub items are built
    GV_LAUNCH(k_pl_rowlen, grid_for(n, 256), 256, 0, s, d, (const uint32_t *)perm, off, P.rdeg, ffirst);
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
    P.rH = first_row_below(HUB_DEG);
    P.rW = first_row_below(WARP_DEG);
    P.rG = first_row_below(GROUP_DEG);
    P.rZ = hcls[NCLASS - 1];  // first isolated row (class 0 comes last)
    // the padded, renumbered columns, straight from the store's blocks
    P.col = (uint32_t *)aux_scratch(g, 13, ((size_t)total + 4) * 4 + 256);
    uint32_t *frow = (uint32_t *)aux_scratch(g, 14, ((size_t)nfill + 1) * 4 + 256);
    if (!P.col || !frow) return GV_ERR_NOMEM;
    GV_LAUNCH(k_pl_fill_small, 148 * 16, PL_THREADS, 0, s, d, (const uint32_t *)perm, (const uint32_t *)inv,
              (const uint32_t *)off, P.col);
    if (nfill) {
        GV_LAUNCH(k_pl_item_fill, grid_for(n, 256), 256, 0, s, (const uint32_t *)ffirst, n, frow);
        GV_LAUNCH(k_pl_fill_items, 148 * 16, PL_THREADS, 0, s, d, (const uint32_t *)perm, (const uint32_t *)inv,
                  (const uint32_t *)off, (const uint32_t *)frow, (const uint32_t *)ffirst, nfill, P.col);
    }
    // hub items, and the entry offsets of the tier boundaries
    P.nitems = 0;
    P.irow = nullptr;
    P.ipart = nullptr;
    if (P.rH) {
        GV_LAUNCH(k_pl_item_count, grid_for(P.rH, 256), 256, 0, s, (const uint32_t *)off, P.rH, ifirst);
        scan_exclusive_u32(ifirst, ifirst, P.rH, ifirst + P.rH, g->bs.scan_tmp, s);
        cudaMemcpyAsync(&P.nitems, ifirst + P.rH, 4, cudaMemcpyDeviceToHost, s);
    }
    const uint32_t rows[4] = {P.rH, P.rW, P.rG, P.rZ};
    for (int i = 0; i < 4; ++i) cudaMemcpyAsync(&P.hoff[i], off + rows[i], 4, cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "plan items");
    if (P.rH) {
        char *q = (char *)aux_scratch(g, 15, (size_t)P.nitems * 4 * (1 + ipart_width) + 512);
        if (!q) return GV_ERR_NOMEM;
        P.irow = carve<uint32_t>(q, P.nitems);
        P.ipart = carve<float>(q, (size_t)P.nitems * ipart_width);
        GV_LAUNCH(k_pl_item_fill, grid_for(P.rH, 256), 256, 0, s, (const uint32_t *)ifirst, P.rH, P.irow);
    }
    *ok = true;
    return GV_OK;
}

}  // namespace

gv_status plan_pagerank(gv_graph *g, float alpha, float eps, int max_iter, const float *x_init, int init_mem,
                        uint32_t source, float *x_out, int32_t *sweeps, int mem, cudaStream_t s,
                        bool *planned) {
    *planned = false;
    const uint32_t n = g->d.n;
    // the single sweep's vectors and residual slots follow the plan arrays
    const size_t extra = ((size_t)n + 1) * 4 * 4 + 4 * 256 + (size_t)PL_GRID * 8 + PL_FIN * 8 + 256 + 64 + 256 +
                         (size_t)n * 4 + 256;
    Plan P{};
    bool ok = false;
    gv_status st = plan_build(g, extra, 1, s, P, &ok);
    if (st != GV_OK || !ok) return st;
    char *p = P.extra;
    float *x0 = carve<float>(p, (size_t)n + 1);
    float *x1 = carve<float>(p, (size_t)n + 1);
    float *c0 = carve<float>(p, (size_t)n + 1);
    float *c1 = carve<float>(p, (size_t)n + 1);
    double *partial = carve<double>(p, PL_GRID + PL_FIN);
    int *state = carve<int>(p, 16);
    float *xstage = carve<float>(p, n);  // a host start vector, vertex order
    const uint32_t *perm = P.perm, *inv = P.inv;
    const uint32_t rH = P.rH, rW = P.rW, rG = P.rG, rZ = P.rZ;
    cudaError_t e = cudaSuccess;
    // start vector
    uint32_t src_row = GV_NIL;
    if (source != GV_NIL) cudaMemcpyAsync(&src_row, inv + source, 4, cudaMemcpyDeviceToHost, s);
    const uint32_t *hoff = P.hoff;
    const float *xin = nullptr;
    if (x_init) {
        if (init_mem == GV_MEM_DEVICE) xin = x_init;
        else {
            e = cudaMemcpyAsync(xstage, x_init, (size_t)n * 4, cudaMemcpyHostToDevice, s);
            if (e != cudaSuccess) return cuda_status(e, "pagerank init");
            xin = xstage;
        }
    }
    e = cudaStreamSynchronize(s);  // src_row
    if (e != cudaSuccess) return cuda_status(e, "plan source");
    const float fill = source == GV_NIL ? 1.0f / (float)n : 0.f;
    // x0 and its contributions in plan order; the isolated rows, which the
    // sweeps never reach, get their value in x1 too
    const float base = source == GV_NIL ? (1.0f - alpha) / (float)n : 0.f;
    GV_LAUNCH(k_pl_init, grid_for((uint64_t)n + 1, 256), 256, 0, s, n, (const uint32_t *)perm, xin, fill, src_row,
              1.f, (const float *)P.rdeg, rZ, base, source == GV_NIL ? 0.f : 1.0f - alpha, x0, c0, x1, c1);
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
    a.off = P.off;
    a.col = P.col;
    a.irow = P.irow;
    a.ifirst = P.ifirst;
    a.rdeg = P.rdeg;
    a.partial = partial;
    a.state = state;
    a.ipart = P.ipart;
    a.alpha = alpha;
    a.base = base;
    a.src_row = src_row;
    a.src_val = source == GV_NIL ? 0.f : 1.0f - alpha;
    a.rH = rH;
    a.rW = rW;
    a.rG = rG;
    a.rZ = rZ;
    a.n = n;
    a.nitems = P.nitems;
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

namespace {

template <int K>
gv_status plan_ppr_batch_k(gv_graph *g, const Plan &P, const uint32_t *sources, int src_mem, uint32_t k, float alpha,
                           float eps, int max_iter, float *x_out, int32_t *sweeps, int mem, cudaStream_t s) {
    const uint32_t n = g->d.n;
    const size_t vec = ((size_t)n + 1) * K * sizeof(float);
    // many small CTA shares: the block scheduler evens out the tiers' tails
    const unsigned waves_default = 148 * 64 / PL_PERIOD;
    unsigned waves = waves_default;
    if (const char *env = std::getenv("GV_PLK_WAVES")) {
        const unsigned w = (unsigned)std::strtoul(env, nullptr, 10);
        if (w >= 1 && w <= PL_WAVES_MAX) waves = w;
    }
    const unsigned grid = waves * PL_PERIOD;
    const uint32_t nparts = grid + PL_FIN;
    // iterates and contributions (4 vectors of n + 1 rows), residual slots,
    // state, sources and their rows; a host result is staged in a free iterate
    const size_t bytes = 4 * vec + (size_t)nparts * 32 * 8 + 3 * 256;
    char *p = (char *)analytics_scratch(g, bytes + 4 * 256);
    if (!p) return GV_ERR_NOMEM;
    float *x0 = carve<float>(p, vec / 4), *x1 = carve<float>(p, vec / 4);
    float *c0 = carve<float>(p, vec / 4), *c1 = carve<float>(p, vec / 4);
    double *partial = carve<double>(p, (size_t)nparts * 32);
    int *state = carve<int>(p, 16);
    uint32_t *srow = carve<uint32_t>(p, 32);
    uint32_t *dsrc = carve<uint32_t>(p, 32);
    cudaError_t e = cudaMemcpyAsync(dsrc, sources, (size_t)k * 4,
                                    src_mem == GV_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_status(e, "plan ppr sources");
    GV_LAUNCH(k_plk_sources, 1, 32, 0, s, (const uint32_t *)dsrc, k, n, (const uint32_t *)P.inv, srow);
    GV_LAUNCH(k_plk_init<K>, grid_for(((uint64_t)n + 1) * K, 256, 148 * 16), 256, 0, s, n, (const uint32_t *)srow,
              (const float *)P.rdeg, P.rZ, 1.0f - alpha, x0, c0, x1, c1);
    cudaMemsetAsync(state, 0, 16, s);
    cudaMemsetAsync(partial, 0, (size_t)nparts * 32 * 8, s);
    // tier work: entries, plus 16 per row of a warp and 16 per group of rows
    constexpr uint32_t G = 32 / K;
    const double w[4] = {(double)P.hoff[0], (double)(P.hoff[1] - P.hoff[0]) + 16.0 * (P.rW - P.rH),
                         (double)(P.hoff[3] - P.hoff[1]) + 16.0 * ((P.rZ - P.rW + G - 1) / G), 0.0};
    // most of the SM's on-chip memory to L1, but room for the residual
    // tables (2 KB, plus 1 KB the system keeps per CTA) of 8 resident CTAs: a
    // zero carveout held the SM to two CTAs (25% of its warps)
    void (*sweep)(PlanBatch) = nullptr;
    if constexpr (K >= 16) sweep = k_plk_sweep_wide<K>;
    else sweep = k_plk_sweep<K>;
    cudaFuncSetAttribute(sweep, cudaFuncAttributePreferredSharedMemoryCarveout, 12);
    cudaGetLastError();
    PlanBatch a{};
    a.off = P.off;
    a.col = P.col;
    a.irow = P.irow;
    a.ifirst = P.ifirst;
    a.rdeg = P.rdeg;
    a.ipart = P.ipart;
    a.partial = partial;
    a.state = state;
    a.srow = srow;
    a.alpha = alpha;
    a.src_val = 1.0f - alpha;
    a.k = k;
    a.rH = P.rH;
    a.rW = P.rW;
    a.rZ = P.rZ;
    a.n = n;
    a.nitems = P.nitems;
    a.split = plan_split(w) & 0xFFFFu;  // items | warp rows; the group rows take the rest
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
                GV_LAUNCH(sweep, grid, PL_THREADS, 0, s, a);
                if (P.rH) GV_LAUNCH(k_plk_hub_fin<K>, PL_FIN, PL_THREADS, 0, s, a, grid);
            }
            GV_LAUNCH(k_plk_done, 1, 32 * k, 0, s, (const double *)partial, nparts, k, eps, state);
            std::swap(xa, xb);
            std::swap(ca, cb);
        }
        launched += chunk;
        e = cudaMemcpyAsync(h_state, state, 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e, "plan ppr sweeps");
        if (h_state[0]) break;
    }
    const float *res = (h_state[1] & 1) ? x1 : x0;
    float *dst = mem == GV_MEM_DEVICE ? x_out : (h_state[1] & 1) ? x0 : x1;  // n k floats fit an iterate
    GV_LAUNCH(k_plk_out<K>, grid_for((uint64_t)n * k, 256, 148 * 16), 256, 0, s, n, k, (const uint32_t *)P.inv, res,
              dst);
    if (mem != GV_MEM_DEVICE) e = cudaMemcpyAsync(x_out, dst, (size_t)n * k * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "plan ppr out");
    g->last_sweeps = h_state[1];
    if (sweeps) *sweeps = h_state[1];
    return cuda_status(cudaGetLastError(), "plan ppr batch");
}

}  // namespace

gv_status plan_ppr_batch(gv_graph *g, const uint32_t *sources, int src_mem, uint32_t k, float alpha, float eps,
                         int max_iter, float *x_out, int32_t *sweeps, int mem, cudaStream_t s, bool *planned) {
    *planned = false;
    // Per sweep at R-MAT scale 25 (1.05 G entries): 3.9 ms for 2 queries,
    // 9.6 for 8, 15.0 for 16 and 26.0 for 32, against 31-43 ms for the
    // store's batched sweep and 3.3 ms for one query's plan sweep.
    if (k < 2 || k > 32) return GV_OK;
    const uint32_t K = k <= 2 ? 2 : k <= 4 ? 4 : k <= 8 ? 8 : k <= 16 ? 16 : 32;
    Plan P{};
    bool ok = false;
    gv_status st = plan_build(g, 0, K, s, P, &ok);
    if (st != GV_OK || !ok) return st;
    *planned = true;
    switch (K) {
        case 2: return plan_ppr_batch_k<2>(g, P, sources, src_mem, k, alpha, eps, max_iter, x_out, sweeps, mem, s);
        case 4: return plan_ppr_batch_k<4>(g, P, sources, src_mem, k, alpha, eps, max_iter, x_out, sweeps, mem, s);
        case 8: return plan_ppr_batch_k<8>(g, P, sources, src_mem, k, alpha, eps, max_iter, x_out, sweeps, mem, s);
        case 16: return plan_ppr_batch_k<16>(g, P, sources, src_mem, k, alpha, eps, max_iter, x_out, sweeps, mem, s);
        default: return plan_ppr_batch_k<32>(g, P, sources, src_mem, k, alpha, eps, max_iter, x_out, sweeps, mem, s);
    }
}

}  // namespace gv
