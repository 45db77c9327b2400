// Batched updates: many update batches of uneven size applied as one window.
//
// Under set semantics the presence of a pair after a sequence of updates is
// decided by the last update that names it.  A window of batches is
// therefore expanded into keys in window order, stable-sorted once, reduced
// to the last operation per pair, and applied as one set-union insert of the
// net inserts plus one set-difference delete of the net deletes (the two
// sets are disjoint, so their order does not matter).  Every touched
// vertex's blocks are scanned once per window instead of once per batch and
// per operation type, and compaction runs once at the end.  The final graph
// equals applying the batches one by one; tests/test_batch_gpu.py checks it.
//
// The window is applied by one persistent launch (launch_window_apply in
// update.cu) when the free stack holds the window's worst case, else by the
// two-stage exact path (one insert and one delete pass).  With
// GV_BATCH_GRAPH the persistent path's device work is captured once per
// capacity (window entries rounded up to a power of two) and the captured
// graph is replayed for later windows: its sizes are read on the device.
//
// The reference applies one batch per host call with several host round
// trips each (src/dynamicStructure/graphvine.cu:222-451).
#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>
#include "../../include/gv_batch.h"
#include "store.cuh"
#include "group.cuh"
#include "prims.cuh"
#include "launch.hpp"
#include "prof.hpp"

namespace gv {
namespace {

constexpr int NET_THREADS = 256;
constexpr int NET_ITEMS = 8;
constexpr int NET_TILE = NET_THREADS * NET_ITEMS;

// Window expansion: op i is an insert when it lies in its batch's insert
// slice.  Keys as k_expand; the value carries the op type (1 = insert).
__global__ void k_window_expand(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst, uint64_t total,
                                const unsigned long long *__restrict__ bstart,
                                const unsigned long long *__restrict__ bsplit, uint32_t nb, int sym, uint32_t n,
                                uint32_t bitsn, unsigned long long *__restrict__ keys, uint32_t *__restrict__ vals,
                                uint8_t *__restrict__ affected, Ctl *ctl) {
    const unsigned long long sent = (bitsn >= 32) ? ~0ull : ((1ull << (2 * bitsn)) - 1ull);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = nb;  // last batch with bstart <= i
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (bstart[mid] <= i) lo = mid; else hi = mid;
        }
        const uint32_t type = (i < bsplit[lo]) ? 1u : 0u;
        const uint32_t s = src[i], d = dst[i];
        const bool bad = (s >= n) || (d >= n);
        if (bad) {
            atomicOr(&ctl->status, GV_DEV_ERR_RANGE);
            ctl->batch_abort = 1;
        }
        const bool drop = bad || (s == d);
        if (!drop) {
            affected[s] = 1;
            affected[d] = 1;
        }
        if (sym) {
            keys[2 * i] = drop ? sent : (((unsigned long long)s << bitsn) | d);
            keys[2 * i + 1] = drop ? sent : (((unsigned long long)d << bitsn) | s);
            vals[2 * i] = type;
            vals[2 * i + 1] = type;
        } else {
            keys[i] = drop ? sent : (((unsigned long long)s << bitsn) | d);
            vals[i] = type;
        }
    }
}

// keep = last of its run of equal keys, not the sentinel, and of type `want`
__device__ __forceinline__ bool net_keep(const unsigned long long *K, const uint32_t *V, uint64_t i, uint64_t N,
                                         unsigned long long sent, uint32_t want) {
    if (i >= N) return false;
    const unsigned long long k = K[i];
    if (k == sent) return false;
    if (i + 1 < N && K[i + 1] == k) return false;
    return V[i] == want;
}

__global__ void __launch_bounds__(NET_THREADS) k_net_count(const unsigned long long *__restrict__ K,
                                                           const uint32_t *__restrict__ V, uint64_t N,
                                                           unsigned long long sent, uint32_t want,
                                                           uint32_t *__restrict__ tile_cnt) {
    __shared__ uint32_t wt[33];
    const uint64_t base = (uint64_t)blockIdx.x * NET_TILE + (uint64_t)threadIdx.x * NET_ITEMS;
    uint32_t c = 0;
#pragma unroll
    for (int j = 0; j < NET_ITEMS; ++j) c += net_keep(K, V, base + j, N, sent, want) ? 1u : 0u;
    const uint32_t tot = cta_sum<uint32_t, NET_THREADS>(c, wt);
    if (threadIdx.x == 0) tile_cnt[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(NET_THREADS) k_net_write(const unsigned long long *__restrict__ K,
                                                           const uint32_t *__restrict__ V, uint64_t N,
                                                           unsigned long long sent, uint32_t want,
                                                           const uint32_t *__restrict__ tile_off,
                                                           unsigned long long *__restrict__ out) {
    __shared__ uint32_t wt[33];
    const uint64_t base = (uint64_t)blockIdx.x * NET_TILE + (uint64_t)threadIdx.x * NET_ITEMS;
    bool keep[NET_ITEMS];
    uint32_t c = 0;
#pragma unroll
    for (int j = 0; j < NET_ITEMS; ++j) {
        keep[j] = net_keep(K, V, base + j, N, sent, want);
        c += keep[j] ? 1u : 0u;
    }
    uint32_t tot;
    uint32_t p = cta_excl_scan<uint32_t, NET_THREADS>(c, wt, tot) + tile_off[blockIdx.x];
#pragma unroll
    for (int j = 0; j < NET_ITEMS; ++j)
        if (keep[j]) out[p++] = K[base + j];
}

// Fills out[count, N) with the sentinel so the compacted keys stay sorted.
__global__ void k_fill_sent(unsigned long long *__restrict__ out, const uint32_t *__restrict__ count, uint64_t N,
                            unsigned long long sent) {
    const uint64_t c = *count;
    for (uint64_t i = c + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = sent;
}

// Net effect over both operations: keep = last of its run of equal keys and
// not the sentinel; the kept keys (sorted, unique) and their operation go to
// out/otype.
__device__ __forceinline__ bool net_last(const unsigned long long *K, uint64_t i, uint64_t N, unsigned long long sent) {
    if (i >= N) return false;
    const unsigned long long k = K[i];
    if (k == sent) return false;
    return !(i + 1 < N && K[i + 1] == k);
}

__global__ void __launch_bounds__(NET_THREADS) k_net_all_count(const unsigned long long *__restrict__ K, uint64_t N,
                                                               unsigned long long sent,
                                                               uint32_t *__restrict__ tile_cnt) {
    __shared__ uint32_t wt[33];
    const uint64_t base = (uint64_t)blockIdx.x * NET_TILE + (uint64_t)threadIdx.x * NET_ITEMS;
    uint32_t c = 0;
#pragma unroll
    for (int j = 0; j < NET_ITEMS; ++j) c += net_last(K, base + j, N, sent) ? 1u : 0u;
    const uint32_t tot = cta_sum<uint32_t, NET_THREADS>(c, wt);
    if (threadIdx.x == 0) tile_cnt[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(NET_THREADS) k_net_all_write(const unsigned long long *__restrict__ K,
                                                               const uint32_t *__restrict__ V, uint64_t N,
                                                               unsigned long long sent,
                                                               const uint32_t *__restrict__ tile_off,
                                                               unsigned long long *__restrict__ out,
                                                               uint32_t *__restrict__ otype) {
    __shared__ uint32_t wt[33];
    const uint64_t base = (uint64_t)blockIdx.x * NET_TILE + (uint64_t)threadIdx.x * NET_ITEMS;
    bool keep[NET_ITEMS];
    uint32_t c = 0;
#pragma unroll
    for (int j = 0; j < NET_ITEMS; ++j) {
        keep[j] = net_last(K, base + j, N, sent);
        c += keep[j] ? 1u : 0u;
    }
    uint32_t tot;
    uint32_t p = cta_excl_scan<uint32_t, NET_THREADS>(c, wt, tot) + tile_off[blockIdx.x];
#pragma unroll
    for (int j = 0; j < NET_ITEMS; ++j)
        if (keep[j]) {
            out[p] = K[base + j];
            otype[p] = V[base + j];
            ++p;
        }
}

// Segments of the net keys (one per source vertex): heads counted per tile,
// then seg_vertex/seg_start, the destinations (bdst) and cleared found flags
// written; ctl->nseg and seg_start[nseg] set by the first thread.
__device__ __forceinline__ bool wseg_head(const unsigned long long *K, uint64_t i, uint32_t cnt, uint32_t bitsn) {
    if (i >= cnt) return false;
    return i == 0 || (K[i] >> bitsn) != (K[i - 1] >> bitsn);
}

__global__ void __launch_bounds__(NET_THREADS) k_wseg_count(const unsigned long long *__restrict__ K,
                                                            const uint32_t *__restrict__ count, uint32_t bitsn,
                                                            uint32_t *__restrict__ tile_cnt) {
    __shared__ uint32_t wt[33];
    const uint32_t cnt = *count;
    const uint64_t base = (uint64_t)blockIdx.x * NET_TILE + (uint64_t)threadIdx.x * NET_ITEMS;
    uint32_t c = 0;
#pragma unroll
    for (int j = 0; j < NET_ITEMS; ++j) c += wseg_head(K, base + j, cnt, bitsn) ? 1u : 0u;
    const uint32_t tot = cta_sum<uint32_t, NET_THREADS>(c, wt);
    if (threadIdx.x == 0) tile_cnt[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(NET_THREADS) k_wseg_write(const unsigned long long *__restrict__ K,
                                                            const uint32_t *__restrict__ count, uint32_t bitsn,
                                                            const uint32_t *__restrict__ tile_off,
                                                            const uint32_t *__restrict__ nseg_total,
                                                            uint32_t *__restrict__ bdst, uint8_t *__restrict__ found,
                                                            uint32_t *__restrict__ seg_vertex,
                                                            uint32_t *__restrict__ seg_start, Ctl *ctl) {
    __shared__ uint32_t wt[33];
    const uint32_t cnt = *count;
    const uint64_t base = (uint64_t)blockIdx.x * NET_TILE + (uint64_t)threadIdx.x * NET_ITEMS;
    const unsigned long long dmask = (1ull << bitsn) - 1ull;
    bool h[NET_ITEMS];
    uint32_t c = 0;
#pragma unroll
    for (int j = 0; j < NET_ITEMS; ++j) {
        h[j] = wseg_head(K, base + j, cnt, bitsn);
        c += h[j] ? 1u : 0u;
    }
    uint32_t tot;
    uint32_t p = cta_excl_scan<uint32_t, NET_THREADS>(c, wt, tot) + tile_off[blockIdx.x];
#pragma unroll
    for (int j = 0; j < NET_ITEMS; ++j) {
        const uint64_t i = base + j;
        if (i < cnt) {
            bdst[i] = (uint32_t)(K[i] & dmask);
            found[i] = 0;
        }
        if (h[j]) {
            seg_vertex[p] = (uint32_t)(K[i] >> bitsn);
            seg_start[p] = (uint32_t)i;
            ++p;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const uint32_t ns = *nseg_total;
        ctl->nseg = ns;
        seg_start[ns] = cnt;
    }
}

// Window header on the device: the graph of a window reads its sizes here,
// so one captured graph serves every window that fits its capacity.
struct WinHeader {
    unsigned long long total;  // pairs in the window
    unsigned int nb;           // batches
    unsigned int pad;
};

// Window expansion with sizes from the header; keys past the window's
// entries (up to the capacity E) become the sentinel.
__global__ void k_window_expand_dev(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
                                    const WinHeader *__restrict__ hdr, uint64_t E,
                                    const unsigned long long *__restrict__ bstart,
                                    const unsigned long long *__restrict__ bsplit, int sym, uint32_t n, uint32_t bitsn,
                                    unsigned long long *__restrict__ keys, uint32_t *__restrict__ vals,
                                    uint8_t *__restrict__ affected, Ctl *ctl) {
    const unsigned long long sent = (bitsn >= 32) ? ~0ull : ((1ull << (2 * bitsn)) - 1ull);
    const uint64_t total = hdr->total;
    const uint32_t nb = hdr->nb;
    const uint64_t per = sym ? 2 : 1;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i * per < E; i += (uint64_t)gridDim.x * blockDim.x) {
        if (i >= total) {
            keys[per * i] = sent;
            vals[per * i] = 0;
            if (sym) {
                keys[per * i + 1] = sent;
                vals[per * i + 1] = 0;
            }
            continue;
        }
        uint32_t lo = 0, hi = nb;  // last batch with bstart <= i
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (bstart[mid] <= i) lo = mid; else hi = mid;
        }
        const uint32_t type = (i < bsplit[lo]) ? 1u : 0u;
        const uint32_t s = src[i], d = dst[i];
        const bool bad = (s >= n) || (d >= n);
        if (bad) {
            atomicOr(&ctl->status, GV_DEV_ERR_RANGE);
            ctl->batch_abort = 1;
        }
        const bool drop = bad || (s == d);
        if (!drop) {
            affected[s] = 1;
            affected[d] = 1;
        }
        if (sym) {
            keys[2 * i] = drop ? sent : (((unsigned long long)s << bitsn) | d);
            keys[2 * i + 1] = drop ? sent : (((unsigned long long)d << bitsn) | s);
            vals[2 * i] = type;
            vals[2 * i + 1] = type;
        } else {
            keys[i] = drop ? sent : (((unsigned long long)s << bitsn) | d);
            vals[i] = type;
        }
    }
}

// ------------------------------------------------------- window queries
// k <= 32 personalised PageRank queries answered on the graph a window
// leaves, inside the window's graph: every size is read on the device, so
// the sweeps can be captured with the window and replayed.  A warp serves a
// vertex with lane j on query j (x and contributions vertex-major, x[v*k+j]);
// vertices of more than WQ_LIGHT_FILL entries are cut into items of 32
// blocks whose partials a finish kernel adds in item order (the split of
// gv_ppr_batch).  The item count is bounded by the pool: at most one item
// per 32 used blocks plus one per vertex of more than WQ_LIGHT_FILL entries,
// which sizes the buffers at capture time.
constexpr uint32_t WQ_LIGHT_FILL = 256;
constexpr int WQ_THREADS = 256;
constexpr unsigned WQ_GRID = 148 * 8;   // light CTAs; as many item CTAs, interleaved
constexpr unsigned WQ_FIN = 148;

struct WinQuery {
    uint32_t k;
    const uint32_t *sources;   // device, k
    float alpha;
    const float *gather;       // contributions, n * k
    const float *xold;
    float *xnew, *cnew;
    double *partial;           // [WQ_GRID + WQ_FIN][32]
    const int *state;          // [0] done, [1] sweeps
    const uint32_t *first;     // [n + 1] first item of each vertex; first[n] = items
    const uint32_t *ivert;     // item -> vertex
    float *ipart;              // [items][32]
    uint64_t icap;             // items the buffers hold
};

__global__ void k_wq_count(DevGraph g, uint32_t *__restrict__ first) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < g.n; v += gridDim.x * blockDim.x) {
        const uint32_t fill = g.vtx[v].y;
        first[v] = fill > WQ_LIGHT_FILL ? (blocks_for(fill, g.logB) + 31u) >> 5 : 0u;
    }
}

__global__ void k_wq_fill(uint32_t n, const uint32_t *__restrict__ first, uint32_t *__restrict__ ivert, uint64_t icap) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        for (uint32_t i = first[v]; i < first[v + 1] && i < icap; ++i) ivert[i] = v;
}

// x0 = e_source per query and its contributions; a vertex with no slots
// takes its final value (1 - alpha at its own query's source, else 0) in both
// iterate buffers here and is left out of the sweeps.
__global__ void k_wq_init(DevGraph g, const uint32_t *__restrict__ sources, uint32_t k, float alpha,
                          float *__restrict__ x, float *__restrict__ c, float *__restrict__ x_other,
                          float *__restrict__ c_other) {
    const size_t total = (size_t)g.n * k;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t v = (uint32_t)(i / k), j = (uint32_t)(i % k);
        const bool src = sources[j] == v;
        const uint4 rec = g.vtx[v];
        if (rec.y == 0) {
            const float xv = src ? 1.0f - alpha : 0.f;
            x[i] = xv;
            x_other[i] = xv;
            c[i] = 0.f;
            c_other[i] = 0.f;
            continue;
        }
        const float xv = src ? 1.f : 0.f;
        x[i] = xv;
        c[i] = rec.z ? xv / (float)rec.z : 0.f;
    }
}

__device__ __forceinline__ void wq_finish(const DevGraph &g, const WinQuery &a, uint32_t v, float acc, uint32_t lane,
                                          double &res) {
    if (lane >= a.k) return;
    const float xv = ((a.sources[lane] == v) ? (1.0f - a.alpha) : 0.f) + a.alpha * acc;
    const size_t at = (size_t)v * a.k + lane;
    a.xnew[at] = xv;
    const uint32_t d = g.vtx[v].z;
    a.cnew[at] = d ? xv / (float)d : 0.f;
    res += (double)fabsf(xv - a.xold[at]);
}

// adds the contributions of entries [e0, e1) of a vertex whose blocks from
// kb0 on are held by the lanes (lane i: block kb0 + i)
__device__ __forceinline__ float wq_entries(const DevGraph &g, const WinQuery &a, uint32_t my_blk, uint32_t kb0,
                                            uint32_t e0, uint32_t e1, uint32_t lane) {
    float acc = 0.f;
    for (uint32_t q0 = e0; q0 < e1; q0 += 32) {
        const uint32_t el = q0 - (kb0 << g.logB) + lane;
        const uint32_t pb = __shfl_sync(GV_FULL_MASK, my_blk, (el >> g.logB) & 31u);
        const uint32_t u = (q0 + lane < e1) ? g.pool[((size_t)pb << g.logB) + (el & (g.B - 1))] : GV_TOMB;
        const uint32_t cnt = min(32u, e1 - q0);
#pragma unroll 8
        for (uint32_t j = 0; j < cnt; ++j) {
            const uint32_t w = __shfl_sync(GV_FULL_MASK, u, j);
            if (w != GV_TOMB && lane < a.k) acc += __ldg(a.gather + (size_t)w * a.k + lane);
        }
    }
    return acc;
}

__device__ __forceinline__ uint32_t wq_block(const DevGraph &g, uint4 rec, uint32_t kb0, uint32_t nb, uint32_t lane) {
    const uint32_t kk = kb0 + lane;
    if (kk >= nb) return GV_NIL;
    return kk == 0 ? rec.x : cbt_block(g.left, g.right, rec.x, kk);
}

// even CTAs: a warp per vertex of at most WQ_LIGHT_FILL entries (residual
// slot blockIdx / 2); odd CTAs: the items of the larger vertices
__global__ void __launch_bounds__(WQ_THREADS) k_wq_sweep(DevGraph g, WinQuery a) {
    __shared__ double red[WQ_THREADS / 32][32];
    if (a.state[0]) return;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t vb = blockIdx.x >> 1, vg = gridDim.x >> 1;
    const uint32_t nw = vg * (WQ_THREADS / 32);
    if ((blockIdx.x & 1u) == 0) {
        double res = 0.0;
        for (uint32_t v = vb * (WQ_THREADS / 32) + warp; v < g.n; v += nw) {
            const uint4 rec = g.vtx[v];
            if (rec.y == 0 || rec.y > WQ_LIGHT_FILL) continue;  // set once by k_wq_init / items
            const uint32_t nb = blocks_for(rec.y, g.logB);
            const float acc = wq_entries(g, a, wq_block(g, rec, 0, nb, lane), 0, 0, rec.y, lane);
            wq_finish(g, a, v, acc, lane, res);
        }
        red[warp][lane] = res;
        __syncthreads();
        if (warp == 0) {
            double t = 0.0;
            for (int w = 0; w < WQ_THREADS / 32; ++w) t += red[w][lane];
            a.partial[(size_t)vb * 32 + lane] = t;
        }
    } else {
        const uint64_t items = min((uint64_t)a.first[g.n], a.icap);
        for (uint64_t i = vb * (WQ_THREADS / 32) + warp; i < items; i += nw) {
            const uint32_t v = a.ivert[i];
            const uint4 rec = g.vtx[v];
            const uint32_t nb = blocks_for(rec.y, g.logB);
            const uint32_t kb0 = (uint32_t)(i - a.first[v]) << 5;
            const uint32_t e0 = kb0 << g.logB, e1 = min(rec.y, (kb0 + 32) << g.logB);
            const float acc = wq_entries(g, a, wq_block(g, rec, kb0, nb, lane), kb0, e0, e1, lane);
            a.ipart[i * 32 + lane] = acc;
        }
    }
}

__global__ void __launch_bounds__(WQ_THREADS) k_wq_fin(DevGraph g, WinQuery a) {
    __shared__ double red[WQ_THREADS / 32][32];
    if (a.state[0]) return;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t nw = gridDim.x * (WQ_THREADS / 32);
    double res = 0.0;
    // the warp on a vertex's first item adds that vertex's items in order
    const uint64_t items = min((uint64_t)a.first[g.n], a.icap);
    for (uint64_t i = blockIdx.x * (WQ_THREADS / 32) + warp; i < items; i += nw) {
        const uint32_t v = a.ivert[i];
        const uint32_t i0 = a.first[v], i1 = a.first[v + 1];
        if (i != i0) continue;
        float acc = 0.f;
        for (uint32_t t = i0; t < i1 && t < a.icap; ++t) acc += a.ipart[(size_t)t * 32 + lane];
        wq_finish(g, a, v, acc, lane, res);
    }
    red[warp][lane] = res;
    __syncthreads();
    if (warp == 0) {
        double t = 0.0;
        for (int w = 0; w < WQ_THREADS / 32; ++w) t += red[w][lane];
        a.partial[(size_t)(WQ_GRID + blockIdx.x) * 32 + lane] = t;
    }
}

// per query, the sum of its residual slots in a fixed order; done when every query is
__global__ void k_wq_done(const double *__restrict__ partial, uint32_t k, float eps, int *state) {
    __shared__ int all_ok;
    if (state[0]) return;
    if (threadIdx.x == 0) all_ok = 1;
    __syncthreads();
    if (threadIdx.x < k) {
        double t = 0.0;
        for (uint32_t p = 0; p < WQ_GRID + WQ_FIN; ++p) t += partial[(size_t)p * 32 + threadIdx.x];
        if (!(t < (double)eps)) atomicAnd(&all_ok, 0);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        state[1] += 1;
        if (all_ok) state[0] = 1;
    }
}

// the last iterate (sweep i, 1-based, wrote buffer i & 1) into the result
__global__ void k_wq_select(const float *__restrict__ x0, const float *__restrict__ x1, const int *__restrict__ state,
                            size_t total, float *__restrict__ out) {
    const float *src = (state[1] & 1) ? x1 : x0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x)
        out[i] = src[i];
}

// A captured window graph and what it was captured against: it is replayed
// while the buffers, the store arrays and the capacity are unchanged.
struct WinGraph {
    uint64_t E = 0, nb_cap = 0;
    uint32_t flags = 0;
    uint32_t qk = 0;            // queries captured with the window (0: none)
    int32_t qiters = 0;
    float qalpha = 0.f, qeps = 0.f;
    std::vector<const void *> ptrs;
    DevGraph d{};
    cudaGraphExec_t exec = nullptr;
    unsigned long long launches = 0;  // kernels per replay
};

struct WindowBufs {
    uint64_t cap_src = 0, cap_dst = 0, cap_vals = 0, cap_vals_alt = 0, cap_bstart = 0, cap_bsplit = 0, cap_tiles = 0;
    uint32_t *src = nullptr, *dst = nullptr;  // device copies of host windows
    uint32_t *vals = nullptr, *vals_alt = nullptr;
    unsigned long long *bstart = nullptr, *bsplit = nullptr;
    uint32_t *tile_cnt = nullptr;  // tiles + 1 (the last slot holds the count)
    cudaStream_t cap_stream = nullptr;
    // persistent path: header, work queue and counts on the device
    void *wctl = nullptr;
    std::vector<WinGraph> graphs;
    unsigned long long captures = 0, replays = 0, persistent = 0, exact = 0;  // window counts by path
    // window queries: iterates, result, items, residuals (grown on demand)
    uint64_t cap_q = 0, cap_items = 0, cap_qn = 0;
    float *qbuf = nullptr;      // x0 | x1 | c0 | c1 | result, n * k each
    uint32_t *qfirst = nullptr; // n + 1
    uint32_t *qivert = nullptr; // items
    float *qipart = nullptr;    // items * 32
    double *qpartial = nullptr; // (WQ_GRID + WQ_FIN) * 32
    int *qstate = nullptr;      // 4
    uint32_t *qsrc = nullptr;   // 32
    WinHeader *hdr() const { return (WinHeader *)wctl; }
    unsigned long long *queue() const { return (unsigned long long *)((char *)wctl + 16); }
    uint32_t *net_count() const { return (uint32_t *)((char *)wctl + 48); }
    uint32_t *nseg_total() const { return (uint32_t *)((char *)wctl + 52); }
};

std::mutex win_mu;
std::vector<std::pair<gv_graph *, std::unique_ptr<WindowBufs>>> g_windows;

WindowBufs &window_bufs(gv_graph *g) {
    std::lock_guard<std::mutex> lk(win_mu);
    for (auto &w : g_windows)
        if (w.first == g) return *w.second;
    g_windows.emplace_back(g, std::make_unique<WindowBufs>());
    return *g_windows.back().second;
}

template <typename T>
gv_status grow(T **p, uint64_t &cap, uint64_t want, size_t elem, const char *what) {
    if (want <= cap && *p) return GV_OK;
    if (*p) cudaFree((void *)*p);
    *p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc((void **)p, want * elem);
    if (e != cudaSuccess) return cuda_status(e, what);
    cap = want;
    return GV_OK;
}

}  // namespace

bool window_stat(gv_graph *g, const char *key, double *value) {
    const char *keys[4] = {"window_captures", "window_replays", "window_persistent", "window_exact"};
    int which = -1;
    for (int i = 0; i < 4; ++i)
        if (!std::strcmp(key, keys[i])) which = i;
    if (which < 0) return false;
    std::lock_guard<std::mutex> lk(win_mu);
    unsigned long long v = 0;
    for (auto &w : g_windows)
        if (w.first == g) {
            const WindowBufs &b = *w.second;
            v = which == 0 ? b.captures : which == 1 ? b.replays : which == 2 ? b.persistent : b.exact;
        }
    *value = (double)v;
    return true;
}

void release_window(gv_graph *g) {
    std::lock_guard<std::mutex> lk(win_mu);
    for (size_t i = 0; i < g_windows.size(); ++i)
        if (g_windows[i].first == g) {
            WindowBufs &b = *g_windows[i].second;
            for (WinGraph &wg : b.graphs)
                if (wg.exec) cudaGraphExecDestroy(wg.exec);
            for (void *p : {(void *)b.src, (void *)b.dst, (void *)b.vals, (void *)b.vals_alt, (void *)b.bstart,
                            (void *)b.bsplit, (void *)b.tile_cnt, b.wctl, (void *)b.qbuf, (void *)b.qfirst,
                            (void *)b.qivert, (void *)b.qipart, (void *)b.qpartial, (void *)b.qstate, (void *)b.qsrc})
                if (p) cudaFree(p);
            if (b.cap_stream) cudaStreamDestroy(b.cap_stream);
            g_windows.erase(g_windows.begin() + i);
            return;
        }
}

// Enqueues the device work of one window (no allocation, no host sync).
static void enqueue_window(gv_graph *g, WindowBufs &wb, uint32_t nb, const uint32_t *dsrc, const uint32_t *ddst,
                           uint64_t total, uint32_t flags, cudaStream_t s) {
    const bool sym = !g->cfg.directed;
    const uint64_t E = sym ? 2 * total : total;
    BatchScratch &bs = g->bs;
    const unsigned long long sent = (g->bitsn >= 32) ? ~0ull : ((1ull << (2 * g->bitsn)) - 1ull);
    GV_LAUNCH(k_window_expand, grid_for(total, 256, 148 * 16), 256, 0, s, dsrc, ddst, total,
              (const unsigned long long *)wb.bstart, (const unsigned long long *)wb.bsplit, nb, sym ? 1 : 0, g->d.n,
              g->bitsn, bs.keys, wb.vals, g->d.affected, g->d.ctl);
    const int which = radix_sort_u64(bs.keys, bs.keys_alt, wb.vals, wb.vals_alt, E, 2 * (int)g->bitsn, bs.rs_counts,
                                     bs.scan_tmp, s);
    const unsigned long long *K = which ? bs.keys_alt : bs.keys;
    const uint32_t *V = which ? wb.vals_alt : wb.vals;
    unsigned long long *out = which ? bs.keys : bs.keys_alt;
    const unsigned ntiles = (unsigned)((E + NET_TILE - 1) / NET_TILE);
    uint32_t *count = wb.tile_cnt + ntiles;
    for (uint32_t want = 1;; want = 0) {  // net inserts, then net deletes
        GV_LAUNCH(k_net_count, ntiles, NET_THREADS, 0, s, K, V, E, sent, want, wb.tile_cnt);
        scan_exclusive_u32(wb.tile_cnt, wb.tile_cnt, ntiles, count, bs.scan_tmp, s);
        GV_LAUNCH(k_net_write, ntiles, NET_THREADS, 0, s, K, V, E, sent, want, (const uint32_t *)wb.tile_cnt, out);
        GV_LAUNCH(k_fill_sent, grid_for(E, 256, 148 * 16), 256, 0, s, out, (const uint32_t *)count, E, sent);
        apply_sorted(g, out, nullptr, E, sym, nullptr, want == 0, want == 0, s);
        if (want == 0) break;
    }
    if (flags & GV_BATCH_COMPACT) run_compact(g, s);
}

// Enqueues the persistent-path window over capacity E (launch only, no
// allocation, no host sync, sizes read from the header): expand, sort, net
// effect over both operations, segments, then one persistent launch applies
// every segment (launch_window_apply) and compaction follows.
static void enqueue_window_persistent(gv_graph *g, WindowBufs &wb, uint64_t E, uint32_t flags, cudaStream_t s) {
    const bool sym = !g->cfg.directed;
    BatchScratch &bs = g->bs;
    const unsigned long long sent = (g->bitsn >= 32) ? ~0ull : ((1ull << (2 * g->bitsn)) - 1ull);
    cudaMemsetAsync(wb.queue(), 0, 24, s);
    const uint64_t per = sym ? 2 : 1;
    GV_LAUNCH(k_window_expand_dev, grid_for(E / per, 256, 148 * 16), 256, 0, s, (const uint32_t *)wb.src,
              (const uint32_t *)wb.dst, (const WinHeader *)wb.hdr(), E, (const unsigned long long *)wb.bstart,
              (const unsigned long long *)wb.bsplit, sym ? 1 : 0, g->d.n, g->bitsn, bs.keys, wb.vals, g->d.affected,
              g->d.ctl);
    int which;
    {
        ProfScope ps(PROF_RADIX, s);
        which = radix_sort_u64(bs.keys, bs.keys_alt, wb.vals, wb.vals_alt, E, 2 * (int)g->bitsn, bs.rs_counts,
                               bs.scan_tmp, s);
    }
    const unsigned long long *K = which ? bs.keys_alt : bs.keys;
    const uint32_t *V = which ? wb.vals_alt : wb.vals;
    unsigned long long *out = which ? bs.keys : bs.keys_alt;
    uint32_t *otype = which ? wb.vals : wb.vals_alt;
    const unsigned ntiles = (unsigned)((E + NET_TILE - 1) / NET_TILE);
    {
        ProfScope ps(PROF_SEGMENT, s);
        GV_LAUNCH(k_net_all_count, ntiles, NET_THREADS, 0, s, K, E, sent, wb.tile_cnt);
        scan_exclusive_u32(wb.tile_cnt, wb.tile_cnt, ntiles, wb.net_count(), bs.scan_tmp, s);
        GV_LAUNCH(k_net_all_write, ntiles, NET_THREADS, 0, s, K, V, E, sent, (const uint32_t *)wb.tile_cnt, out, otype);
        GV_LAUNCH(k_wseg_count, ntiles, NET_THREADS, 0, s, (const unsigned long long *)out,
                  (const uint32_t *)wb.net_count(), g->bitsn, wb.tile_cnt);
        scan_exclusive_u32(wb.tile_cnt, wb.tile_cnt, ntiles, wb.nseg_total(), bs.scan_tmp, s);
        GV_LAUNCH(k_wseg_write, ntiles, NET_THREADS, 0, s, (const unsigned long long *)out,
                  (const uint32_t *)wb.net_count(), g->bitsn, (const uint32_t *)wb.tile_cnt,
                  (const uint32_t *)wb.nseg_total(), bs.bdst, bs.found, bs.seg_vertex, bs.seg_start, g->d.ctl);
    }
    launch_window_apply(g, bs.seg_vertex, bs.seg_start, bs.bdst, otype, bs.found, bs.big_list, wb.queue(), s);
    if (flags & GV_BATCH_COMPACT) run_compact(g, s);
}

// Queries answered after a window (gv_batch_run_ppr).
struct QuerySpec {
    uint32_t k = 0;
    const uint32_t *sources = nullptr;  // host, k
    float alpha = 0.85f, eps = 1e-6f;
    int32_t max_iter = 0;
    float *x_out = nullptr;
    int mem = GV_MEM_HOST;
    int32_t *sweeps = nullptr;
};

static gv_status grow_queries(gv_graph *g, WindowBufs &wb, uint32_t k) {
    const uint64_t n = g->d.n;
    const uint64_t heavy_max = std::min<uint64_t>(n, g->d.P * (uint64_t)g->d.B / (WQ_LIGHT_FILL + 1));
    const uint64_t want_q = 5 * n * k, want_items = g->d.P / 32 + heavy_max + 1;
    gv_status st = GV_OK;
    if (want_q > wb.cap_q || !wb.qbuf) {
        if (wb.qbuf) cudaFree(wb.qbuf);
        wb.qbuf = nullptr;
        wb.cap_q = 0;
        cudaError_t e = cudaMalloc(&wb.qbuf, want_q * 4);
        if (e != cudaSuccess) return cuda_status(e, "window query iterates");
        wb.cap_q = want_q;
    }
    if (!wb.qfirst || wb.cap_items < want_items || wb.cap_qn < n) {
        for (void *p : {(void *)wb.qfirst, (void *)wb.qivert, (void *)wb.qipart, (void *)wb.qpartial,
                        (void *)wb.qstate, (void *)wb.qsrc})
            if (p) cudaFree(p);
        wb.qfirst = wb.qivert = wb.qsrc = nullptr;
        wb.qipart = nullptr;
        wb.qpartial = nullptr;
        wb.qstate = nullptr;
        wb.cap_items = wb.cap_qn = 0;
        cudaError_t e = cudaMalloc(&wb.qfirst, (n + 1) * 4);
        if (e == cudaSuccess) e = cudaMalloc(&wb.qivert, want_items * 4);
        if (e == cudaSuccess) e = cudaMalloc(&wb.qipart, want_items * 32 * 4);
        if (e == cudaSuccess) e = cudaMalloc(&wb.qpartial, (size_t)(WQ_GRID + WQ_FIN) * 32 * 8);
        if (e == cudaSuccess) e = cudaMalloc(&wb.qstate, 16);
        if (e == cudaSuccess) e = cudaMalloc(&wb.qsrc, 32 * 4);
        if (e != cudaSuccess) return cuda_status(e, "window query scratch");
        wb.cap_items = want_items;
        wb.cap_qn = n;
    }
    return st;
}

// Enqueues the queries' sweeps (launch only, no host sync; max_iter sweeps
// are launched and those after convergence exit at once), then the result
// copy into the result block.
static void enqueue_queries(gv_graph *g, WindowBufs &wb, uint32_t k, float alpha, float eps, int32_t max_iter,
                            cudaStream_t s) {
    const DevGraph d = g->d;
    const uint32_t n = d.n;
    const size_t nk = (size_t)n * k;
    float *x[2] = {wb.qbuf, wb.qbuf + nk};
    float *c[2] = {wb.qbuf + 2 * nk, wb.qbuf + 3 * nk};
    float *xr = wb.qbuf + 4 * nk;
    GV_LAUNCH(k_wq_count, grid_for(n, 256), 256, 0, s, d, wb.qfirst);
    scan_exclusive_u32(wb.qfirst, wb.qfirst, n, wb.qfirst + n, g->bs.scan_tmp, s);
    GV_LAUNCH(k_wq_fill, grid_for(n, 256), 256, 0, s, n, (const uint32_t *)wb.qfirst, wb.qivert, wb.cap_items);
    cudaMemsetAsync(wb.qstate, 0, 16, s);
    cudaMemsetAsync(wb.qpartial, 0, (size_t)(WQ_GRID + WQ_FIN) * 32 * 8, s);
    GV_LAUNCH(k_wq_init, grid_for(nk, 256, 148 * 16), 256, 0, s, d, (const uint32_t *)wb.qsrc, k, alpha, x[0], c[0],
              x[1], c[1]);
    int cur = 0;
    for (int32_t it = 0; it < max_iter; ++it) {
        WinQuery a{k, wb.qsrc, alpha, c[cur], x[cur], x[cur ^ 1], c[cur ^ 1], wb.qpartial, wb.qstate, wb.qfirst,
                   wb.qivert, wb.qipart, wb.cap_items};
        {
            ProfScope ps(PROF_PULL, s);
            GV_LAUNCH(k_wq_sweep, 2 * WQ_GRID, WQ_THREADS, 0, s, d, a);
            GV_LAUNCH(k_wq_fin, WQ_FIN, WQ_THREADS, 0, s, d, a);
        }
        GV_LAUNCH(k_wq_done, 1, 32, 0, s, (const double *)wb.qpartial, k, eps, wb.qstate);
        cur ^= 1;
    }
    GV_LAUNCH(k_wq_select, grid_for(nk, 256, 148 * 16), 256, 0, s, (const float *)x[0], (const float *)x[1],
              (const int *)wb.qstate, nk, xr);
}

// The buffers a persistent-path graph captures.
static std::vector<const void *> window_ptrs(gv_graph *g, WindowBufs &wb) {
    const BatchScratch &bs = g->bs;
    return {wb.src, wb.dst, wb.vals, wb.vals_alt, wb.bstart, wb.bsplit, wb.tile_cnt, wb.wctl, bs.keys, bs.keys_alt,
            bs.rs_counts, bs.scan_tmp, bs.bdst, bs.found, bs.seg_vertex, bs.seg_start, bs.big_list, wb.qbuf,
            wb.qfirst, wb.qivert, wb.qipart, wb.qpartial, wb.qstate, wb.qsrc};
}

// Runs the persistent-path window of capacity E on stream s: replays the
// graph captured for (E, batch capacity, flags) when the buffers and the
// store are those it was captured with, else captures it first.
static gv_status run_window_graph(gv_graph *g, WindowBufs &wb, uint64_t E, uint64_t nb_cap, uint32_t flags,
                                  const QuerySpec *q, cudaStream_t s) {
    const std::vector<const void *> ptrs = window_ptrs(g, wb);
    const uint32_t qk = q ? q->k : 0;
    const int32_t qit = q ? q->max_iter : 0;
    const float qa = q ? q->alpha : 0.f, qe = q ? q->eps : 0.f;
    WinGraph *hit = nullptr;
    for (WinGraph &wg : wb.graphs)
        if (wg.E == E && wg.nb_cap == nb_cap && wg.flags == flags && wg.ptrs == ptrs && wg.qk == qk &&
            wg.qiters == qit && wg.qalpha == qa && wg.qeps == qe && std::memcmp(&wg.d, &g->d, sizeof(DevGraph)) == 0)
            hit = &wg;
    if (!hit) {
        // graphs captured against buffers that have since moved are useless
        for (size_t i = 0; i < wb.graphs.size();) {
            if (wb.graphs[i].ptrs != ptrs || std::memcmp(&wb.graphs[i].d, &g->d, sizeof(DevGraph)) != 0) {
                if (wb.graphs[i].exec) cudaGraphExecDestroy(wb.graphs[i].exec);
                wb.graphs.erase(wb.graphs.begin() + i);
            } else {
                ++i;
            }
        }
        if (!wb.cap_stream) {
            cudaError_t e = cudaStreamCreateWithFlags(&wb.cap_stream, cudaStreamNonBlocking);
            if (e != cudaSuccess) return cuda_status(e, "capture stream");
        }
        const unsigned long long l0 = g_launches.load();
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamBeginCapture(wb.cap_stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            enqueue_window_persistent(g, wb, E, flags, wb.cap_stream);
            if (qk) enqueue_queries(g, wb, qk, qa, qe, qit, wb.cap_stream);
            e = cudaStreamEndCapture(wb.cap_stream, &graph);
        }
        WinGraph wg;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&wg.exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            if (wg.exec) cudaGraphExecDestroy(wg.exec);
            return cuda_status(e, "window graph capture");
        }
        wg.E = E;
        wg.nb_cap = nb_cap;
        wg.flags = flags;
        wg.qk = qk;
        wg.qiters = qit;
        wg.qalpha = qa;
        wg.qeps = qe;
        wg.ptrs = ptrs;
        wg.d = g->d;
        wg.launches = g_launches.load() - l0;
        g_launches.fetch_sub(wg.launches);  // counted when the graph runs
        wb.graphs.push_back(wg);
        hit = &wb.graphs.back();
        ++wb.captures;
    } else {
        ++wb.replays;
    }
    cudaError_t e = cudaGraphLaunch(hit->exec, s);
    if (e == cudaSuccess) g_launches.fetch_add(hit->launches);
    return cuda_status(e, "window graph launch");
}

static uint64_t pow2_at_least(uint64_t x, uint64_t lo) {
    uint64_t p = lo;
    while (p < x) p <<= 1;
    return p;
}

}  // namespace gv

using namespace gv;

static gv_status batch_run_impl(gv_graph *g, const gv_batch_desc *descs, uint32_t nbatches, const uint32_t *src,
                                const uint32_t *dst, int mem, uint32_t flags, void *stream, const QuerySpec *q) {
    if (!g || (nbatches && !descs)) { set_error("null argument"); return GV_ERR_INVALID; }
    if (g->parent) { set_error("a view is read-only"); return GV_ERR_STATE; }
    if (g->cfg.weighted) { set_error("gv_batch_run handles unweighted stores"); return GV_ERR_UNSUPPORTED; }
    if (nbatches == 0 && !q) return GV_OK;
    uint64_t total = 0;
    for (uint32_t i = 0; i < nbatches; ++i) {
        if (descs[i].offset != total) { set_error("batches must be laid out consecutively"); return GV_ERR_INVALID; }
        total += (uint64_t)descs[i].n_insert + descs[i].n_delete;
    }
    if (total == 0 && !q) return GV_OK;
    if (total && (!src || !dst)) { set_error("null src/dst"); return GV_ERR_INVALID; }
    if (total > 0x7FFFFFFFull) { set_error("window too large"); return GV_ERR_CAPACITY; }
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != g->cfg.device) cudaSetDevice(g->cfg.device);
    cudaStream_t s = (cudaStream_t)stream;
    WindowBufs &wb = window_bufs(g);
    const bool sym = !g->cfg.directed;
    const uint64_t per = sym ? 2 : 1;
    const uint64_t E = per * total;
    // Persistent path: capacity rounded up to a power of two so that windows
    // of similar size share one captured graph; its sizes live on the device.
    const uint64_t Ecap = pow2_at_least(E, 1ull << 16);
    const uint64_t nb_cap = pow2_at_least(nbatches, 64);
    const uint64_t pcap = Ecap / per;
    gv_status st = ensure_batch_scratch(g, Ecap, 1);
    const uint64_t ntiles = (Ecap + NET_TILE - 1) / NET_TILE;
    if (st == GV_OK) st = grow(&wb.vals, wb.cap_vals, Ecap, 4, "window vals");
    if (st == GV_OK) st = grow(&wb.vals_alt, wb.cap_vals_alt, Ecap, 4, "window vals");
    if (st == GV_OK) st = grow(&wb.bstart, wb.cap_bstart, nb_cap, 8, "window starts");
    if (st == GV_OK) st = grow(&wb.bsplit, wb.cap_bsplit, nb_cap, 8, "window splits");
    if (st == GV_OK) st = grow(&wb.tile_cnt, wb.cap_tiles, ntiles + 2, 4, "window tiles");
    if (st == GV_OK) st = grow(&wb.src, wb.cap_src, pcap, 4, "window src");
    if (st == GV_OK) st = grow(&wb.dst, wb.cap_dst, pcap, 4, "window dst");
    if (st == GV_OK && !wb.wctl) {
        cudaError_t e = cudaMalloc(&wb.wctl, 64);
        if (e != cudaSuccess) st = cuda_status(e, "window control");
    }
    if (st == GV_OK && q) st = grow_queries(g, wb, q->k);
    if (st == GV_OK && mem == GV_MEM_HOST) {
        const uint32_t n = g->d.n;
        for (uint64_t i = 0; i < total; ++i)
            if (src[i] >= n || dst[i] >= n) { set_error("vertex id out of range"); st = GV_ERR_INVALID; break; }
    }
    Ctl cc{};
    if (st == GV_OK) {
        const cudaMemcpyKind k = mem == GV_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
        cudaError_t e = cudaSuccess;
        if (total) e = cudaMemcpyAsync(wb.src, src, total * 4, k, s);
        if (e == cudaSuccess && total) e = cudaMemcpyAsync(wb.dst, dst, total * 4, k, s);
        if (e == cudaSuccess && q) e = cudaMemcpyAsync(wb.qsrc, q->sources, q->k * 4, cudaMemcpyHostToDevice, s);
        std::vector<unsigned long long> hs(nbatches), hp(nbatches);
        for (uint32_t i = 0; i < nbatches; ++i) {
            hs[i] = descs[i].offset;
            hp[i] = descs[i].offset + descs[i].n_insert;
        }
        WinHeader h{total, nbatches, 0};
        if (e == cudaSuccess && nbatches) e = cudaMemcpyAsync(wb.bstart, hs.data(), nbatches * 8, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && nbatches) e = cudaMemcpyAsync(wb.bsplit, hp.data(), nbatches * 8, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(wb.hdr(), &h, sizeof(h), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&cc, g->d.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
        // the host vectors and the header die here: wait for the copies before returning
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_status(e, "window inputs");
    }
    if (st == GV_OK) {
        // Admission for the persistent path: the free stack must hold the
        // worst case of the window, one block per touched vertex plus one
        // per B inserted entries; otherwise the two-stage path plans the
        // blocks exactly and rejects the window if they do not fit.
        const uint64_t worst = (E + g->d.B - 1) / g->d.B + std::min<uint64_t>(E, g->d.n);
        if (worst <= cc.free_top) {
            ++wb.persistent;
            if (flags & GV_BATCH_GRAPH) st = run_window_graph(g, wb, Ecap, nb_cap, flags, q, s);
            else {
                enqueue_window_persistent(g, wb, Ecap, flags, s);
                if (q) enqueue_queries(g, wb, q->k, q->alpha, q->eps, q->max_iter, s);
                st = cuda_status(cudaGetLastError(), "window launch");
            }
        } else {
            ++wb.exact;
            if (total) enqueue_window(g, wb, nbatches, wb.src, wb.dst, total, flags, s);
            if (q) enqueue_queries(g, wb, q->k, q->alpha, q->eps, q->max_iter, s);
            st = cuda_status(cudaGetLastError(), "window launch");
        }
    }
    if (st == GV_OK && q) {
        // the answers: the result block to the caller, and the sweeps run
        const size_t nk = (size_t)g->d.n * q->k;
        int32_t hs[2] = {0, 0};
        cudaError_t e = cudaMemcpyAsync(q->x_out, wb.qbuf + 4 * nk, nk * 4,
                                        q->mem == GV_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hs, wb.qstate, 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_status(e, "window queries");
        else if (q->sweeps) *q->sweeps = hs[1];
    }
    if (prev >= 0 && prev != g->cfg.device) cudaSetDevice(prev);
    return st;
}

extern "C" gv_status gv_batch_run(gv_graph *g, const gv_batch_desc *descs, uint32_t nbatches, const uint32_t *src,
                                  const uint32_t *dst, int mem, uint32_t flags, void *stream) {
    return batch_run_impl(g, descs, nbatches, src, dst, mem, flags, stream, nullptr);
}

extern "C" gv_status gv_batch_run_ppr(gv_graph *g, const gv_batch_desc *descs, uint32_t nbatches, const uint32_t *src,
                                      const uint32_t *dst, int mem, uint32_t flags, const uint32_t *sources,
                                      uint32_t k, float alpha, float epsilon, int32_t max_iter, float *x_out,
                                      int32_t *sweeps, void *stream) {
    if (!g || !sources || !x_out || k == 0 || k > 32 || max_iter < 0) { set_error("bad argument"); return GV_ERR_INVALID; }
    if (g->cfg.directed) { set_error("window queries need an undirected (symmetric) store"); return GV_ERR_STATE; }
    for (uint32_t j = 0; j < k; ++j)
        if (sources[j] >= g->d.n) { set_error("source out of range"); return GV_ERR_INVALID; }
    QuerySpec q;
    q.k = k;
    q.sources = sources;
    q.alpha = alpha;
    q.eps = epsilon;
    q.max_iter = max_iter;
    q.x_out = x_out;
    q.mem = mem;
    q.sweeps = sweeps;
    return batch_run_impl(g, descs, nbatches, src, dst, mem, flags, stream, &q);
}

// Autotuner: for every candidate (edge-block size x threads per vertex)
// builds the sample graph, times one window of batches and one PageRank
// with CUDA events, and repeats that on a fresh graph; the first round
// warms the candidate up (scratch growth) and is dropped, the median of the
// other rounds is kept.  The candidate with the smallest median total wins.
extern "C" gv_status gv_autotune(const gv_config *base, const uint32_t *src0, const uint32_t *dst0, uint64_t k0,
                                 const gv_batch_desc *descs, uint32_t nbatches, const uint32_t *bsrc,
                                 const uint32_t *bdst, int mem, gv_tune_result *results, uint32_t *nresults,
                                 gv_config *best) {
    if (!base || !best || (k0 && (!src0 || !dst0))) { set_error("null argument"); return GV_ERR_INVALID; }
    static const uint32_t blocks[] = {32, 64, 128};
    static const uint32_t tpvs[] = {4, 8, 16, 32};
    *best = *base;
    float best_ms = 1e30f;
    uint32_t nr = 0;
    cudaEvent_t e0, e1, e2;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    gv_status st = GV_OK;
    std::vector<float> x(base->num_vertices);
    constexpr int ROUNDS = 4;  // one warm-up, three timed
    for (uint32_t B : blocks)
        for (uint32_t T : tpvs) {
            gv_config c = *base;
            c.block_size = B;
            c.threads_per_vertex = T;
            std::vector<float> upd_ms, pr_ms;
            for (int r = 0; r < ROUNDS && st == GV_OK; ++r) {
                gv_graph *g = nullptr;
                st = gv_create(&c, &g);
                if (st != GV_OK) break;
                st = gv_insert_edges(g, src0, dst0, nullptr, k0, mem, nullptr);
                if (st == GV_OK) st = gv_synchronize(g, nullptr);
                float upd = 0.f, pr = 0.f;
                if (st == GV_OK) {
                    cudaEventRecord(e0, 0);
                    st = gv_batch_run(g, descs, nbatches, bsrc, bdst, mem, GV_BATCH_COMPACT, nullptr);
                    cudaEventRecord(e1, 0);
                    int32_t sw = 0;
                    if (st == GV_OK) st = gv_pagerank(g, 0.85f, 1e-6f, 100, x.data(), &sw, GV_MEM_HOST, nullptr);
                    cudaEventRecord(e2, 0);
                    cudaEventSynchronize(e2);
                    cudaEventElapsedTime(&upd, e0, e1);
                    cudaEventElapsedTime(&pr, e1, e2);
                }
                gv_destroy(g);
                if (r > 0) {
                    upd_ms.push_back(upd);
                    pr_ms.push_back(pr);
                }
            }
            if (st != GV_OK) break;
            std::sort(upd_ms.begin(), upd_ms.end());
            std::sort(pr_ms.begin(), pr_ms.end());
            const float upd = upd_ms[upd_ms.size() / 2], pr = pr_ms[pr_ms.size() / 2];
            if (results && nresults && nr < *nresults) results[nr] = {B, T, upd, pr};
            ++nr;
            if (upd + pr < best_ms) {
                best_ms = upd + pr;
                *best = c;
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    if (nresults) *nresults = nr;
    return st;
}
