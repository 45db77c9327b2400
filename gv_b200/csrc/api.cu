// C ABI of libgv: graph lifecycle, scratch management, host staging and the
// update entry points.  Replaces the host orchestration of class GraphVine
// (src/dynamicStructure/graphvine.cu:5-527) with stream-ordered calls that
// return status codes instead of exiting (include/util/cudaError.cuh:8-26).
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>
#include "store.cuh"
#include "prims.cuh"
#include "prof.hpp"
#include "launch.hpp"

namespace gv {

namespace {
thread_local std::string t_err;

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

__global__ void k_init_store(uint4 *vtx, uint32_t n, uint32_t *free_stack, unsigned long long P) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        vtx[i] = make_uint4(GV_NIL, 0u, 0u, GV_NIL);
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < P; i += stride)
        free_stack[i] = (uint32_t)(P - 1ull - i);
}

// src of every CSR entry (device-resident offsets): upper-bound search.
__global__ void k_csr_sources(const unsigned long long *__restrict__ off, uint32_t n, uint64_t m,
                              uint32_t *__restrict__ src) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = n;  // find largest u with off[u] <= i
        while (hi - lo > 1) {
            uint32_t mid = (lo + hi) >> 1;
            if (off[mid] <= i) lo = mid; else hi = mid;
        }
        src[i] = lo;
    }
}

template <typename T>
gv_status dmalloc(T **p, size_t bytes, const char *what) {
    *p = nullptr;
    if (bytes == 0) return GV_OK;
    cudaError_t e = cudaMalloc((void **)p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        t_err = std::string("cudaMalloc(") + what + ", " + std::to_string(bytes) + " B): " + cudaGetErrorString(e);
        *p = nullptr;
        return GV_ERR_NOMEM;
    }
    return GV_OK;
}

template <typename T>
void dfree(T *&p) {
    if (p) cudaFree((void *)p);
    p = nullptr;
}

void free_batch_entries(BatchScratch &bs) {
    dfree(bs.keys); dfree(bs.keys_alt); dfree(bs.vals); dfree(bs.vals_alt);
    dfree(bs.rs_counts); dfree(bs.scan_tmp); dfree(bs.tile_cnt); dfree(bs.bdst); dfree(bs.bw);
    dfree(bs.found); dfree(bs.seg_vertex); dfree(bs.seg_start); dfree(bs.seg_found);
    dfree(bs.seg_newblocks); dfree(bs.seg_blkbase); dfree(bs.big_list);
    bs.cap = 0;
}

void free_batch_inputs(BatchScratch &bs) {
    dfree(bs.in_src); dfree(bs.in_dst); dfree(bs.in_w);
    bs.in_cap = 0;
}

bool valid_block(uint32_t b) { return b == 32 || b == 64 || b == 128; }
bool valid_tpv(uint32_t t) { return t == 4 || t == 8 || t == 16 || t == 32; }

gv_status map_device_status(unsigned st) {
    if (st & GV_DEV_ERR_TIMEOUT) { t_err = "device wait timed out"; return GV_ERR_TIMEOUT; }
    if (st & GV_DEV_ERR_NOMEM) { t_err = "edge-block pool exhausted; batch rejected"; return GV_ERR_NOMEM; }
    if (st & GV_DEV_ERR_RANGE) { t_err = "vertex id out of range; batch rejected"; return GV_ERR_INVALID; }
    if (st & GV_DEV_ERR_CAP) { t_err = "scratch capacity exceeded"; return GV_ERR_CAPACITY; }
    return GV_OK;
}

}  // namespace

void set_error(const std::string &msg) { t_err = msg; }

gv_status cuda_status(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return GV_OK;
    t_err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? GV_ERR_NOMEM : GV_ERR_CUDA;
}

gv_status ensure_batch_scratch(gv_graph *g, uint64_t entries, uint64_t pairs) {
    BatchScratch &bs = g->bs;
    gv_status st = GV_OK;
    if (entries > bs.cap) {
        free_batch_entries(bs);
        const uint64_t E = entries;
        const bool w = g->cfg.weighted != 0;
        const uint64_t nseg_tiles = (E + 2047) / 2048 + 1;
        uint64_t scan_elems = radix_counts_elems(E);
        if (nseg_tiles > scan_elems) scan_elems = nseg_tiles;
        if ((uint64_t)g->d.n + 1 > scan_elems) scan_elems = (uint64_t)g->d.n + 1;
        if ((st = dmalloc(&bs.keys, E * 8, "keys")) != GV_OK) goto fail;
        if ((st = dmalloc(&bs.keys_alt, E * 8, "keys_alt")) != GV_OK) goto fail;
        if (w) {
            if ((st = dmalloc(&bs.vals, E * 4, "vals")) != GV_OK) goto fail;
            if ((st = dmalloc(&bs.vals_alt, E * 4, "vals_alt")) != GV_OK) goto fail;
            if ((st = dmalloc(&bs.bw, E * 4, "bw")) != GV_OK) goto fail;
        }
        if ((st = dmalloc(&bs.rs_counts, radix_counts_elems(E) * 4 + 16, "rs_counts")) != GV_OK) goto fail;
        if ((st = dmalloc((char **)&bs.scan_tmp, scan_scratch_bytes(scan_elems), "scan")) != GV_OK) goto fail;
        if ((st = dmalloc(&bs.tile_cnt, std::max<uint64_t>(nseg_tiles, 8) * 8, "tile_cnt")) != GV_OK) goto fail;
        if ((st = dmalloc(&bs.bdst, E * 4, "bdst")) != GV_OK) goto fail;
        if ((st = dmalloc(&bs.found, E, "found")) != GV_OK) goto fail;
        if ((st = dmalloc(&bs.seg_vertex, E * 4, "seg_vertex")) != GV_OK) goto fail;
        if ((st = dmalloc(&bs.seg_start, (E + 1) * 4, "seg_start")) != GV_OK) goto fail;
        if ((st = dmalloc(&bs.seg_found, E * 4, "seg_found")) != GV_OK) goto fail;
        if ((st = dmalloc(&bs.seg_newblocks, E * 4, "seg_newblocks")) != GV_OK) goto fail;
        if ((st = dmalloc(&bs.seg_blkbase, E * 4, "seg_blkbase")) != GV_OK) goto fail;
        if ((st = dmalloc(&bs.big_list, E * 4, "big_list")) != GV_OK) goto fail;
        bs.cap = E;
    }
    if (pairs > bs.in_cap) {
        free_batch_inputs(bs);
        if ((st = dmalloc(&bs.in_src, pairs * 4, "in_src")) != GV_OK) goto fail;
        if ((st = dmalloc(&bs.in_dst, pairs * 4, "in_dst")) != GV_OK) goto fail;
        if (g->cfg.weighted && (st = dmalloc(&bs.in_w, pairs * 4, "in_w")) != GV_OK) goto fail;
        bs.in_cap = pairs;
    }
    return GV_OK;
fail:
    free_batch_entries(bs);
    free_batch_inputs(bs);
    return st;
}

void *analytics_scratch(gv_graph *g, size_t bytes) {
    if (bytes > g->an_bytes) {
        if (g->an_buf) cudaFree(g->an_buf);
        g->an_buf = nullptr;
        g->an_bytes = 0;
        // a quarter more than asked, so calls of slightly different sizes
        // (and the device-wide stall of cudaFree) do not repeat
        size_t want = bytes + bytes / 4;
        if (cudaMalloc(&g->an_buf, want) != cudaSuccess) {
            cudaGetLastError();
            want = bytes;
            if (cudaMalloc(&g->an_buf, want) != cudaSuccess) {
                cudaGetLastError();
                g->an_buf = nullptr;
                t_err = "analytics scratch allocation of " + std::to_string(bytes) + " B failed";
                return nullptr;
            }
        }
        g->an_bytes = want;
    }
    return g->an_buf;
}

void release_analytics_scratch(gv_graph *g) {
    if (g->an_buf) cudaFree(g->an_buf);
    g->an_buf = nullptr;
    g->an_bytes = 0;
    for (int i = 0; i < gv_graph::AUX_SLOTS; ++i) {
        if (g->aux[i]) cudaFree(g->aux[i]);
        g->aux[i] = nullptr;
        g->aux_bytes[i] = 0;
    }
}

void *aux_scratch(gv_graph *g, int slot, size_t bytes) {
    if (bytes > g->aux_bytes[slot]) {
        if (g->aux[slot]) cudaFree(g->aux[slot]);
        g->aux[slot] = nullptr;
        g->aux_bytes[slot] = 0;
        const size_t want = bytes + bytes / 4;
        if (cudaMalloc(&g->aux[slot], want) != cudaSuccess) {
            cudaGetLastError();
            t_err = "auxiliary scratch allocation of " + std::to_string(want) + " B failed";
            return nullptr;
        }
        g->aux_bytes[slot] = want;
    }
    return g->aux[slot];
}

gv_status read_ctl(gv_graph *g, Ctl *out, cudaStream_t s) {
    cudaError_t e = cudaMemcpyAsync(out, g->d.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return cuda_status(e, "read control block");
}

// ----------------------------------------------------------------- profiler
namespace {
const char *const kProfNames[PROF_NSLOTS] = {"radix", "segment", "member", "apply", "compact",
                                             "pull", "tc_snapshot", "tc_count", "bfs_level", "bc_dep",
                                             "wpr_build", "wpr_sweep", "wpr_grad", "tc_core",
                                             "tc_probe", "tc_sort"};
struct ProfRec {
    int slot;
    cudaEvent_t a, b;
};
std::mutex prof_mu;
std::atomic<bool> prof_on{false};
std::vector<ProfRec> prof_recs;
std::vector<cudaEvent_t> prof_pool;
double prof_ms[PROF_NSLOTS];
unsigned long long prof_n[PROF_NSLOTS];

cudaEvent_t prof_event() {
    if (!prof_pool.empty()) {
        cudaEvent_t e = prof_pool.back();
        prof_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

void prof_collect_locked() {
    for (ProfRec &r : prof_recs) {
        float ms = 0.f;
        if (cudaEventSynchronize(r.b) == cudaSuccess && cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
            prof_ms[r.slot] += ms;
            prof_n[r.slot] += 1;
        }
        prof_pool.push_back(r.a);
        prof_pool.push_back(r.b);
    }
    prof_recs.clear();
}
}  // namespace

int prof_begin(int slot, cudaStream_t s) {
    if (!prof_on.load(std::memory_order_relaxed)) return -1;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return -1;
    std::lock_guard<std::mutex> lk(prof_mu);
    ProfRec r{slot, prof_event(), prof_event()};
    cudaEventRecord(r.a, s);
    prof_recs.push_back(r);
    return (int)prof_recs.size() - 1;
}

void prof_end(int token, cudaStream_t s) {
    if (token < 0) return;
    std::lock_guard<std::mutex> lk(prof_mu);
    if (token < (int)prof_recs.size()) cudaEventRecord(prof_recs[token].b, s);
}

}  // namespace gv

using namespace gv;

extern "C" {

const char *gv_version(void) { return "gv-b200 0.1 (sm_100a)"; }

const char *gv_last_error_string(void) { return t_err.c_str(); }

uint64_t gv_kernel_launches(void) { return g_launches.load(); }

gv_status gv_profile_enable(int32_t on) {
    std::lock_guard<std::mutex> lk(prof_mu);
    if (!on) prof_collect_locked();
    prof_on.store(on != 0);
    return GV_OK;
}

gv_status gv_profile_reset(void) {
    std::lock_guard<std::mutex> lk(prof_mu);
    prof_collect_locked();
    for (int i = 0; i < PROF_NSLOTS; ++i) {
        prof_ms[i] = 0.0;
        prof_n[i] = 0;
    }
    return GV_OK;
}

gv_status gv_profile_query(const char *name, double *total_ms, uint64_t *launches) {
    if (!name) return GV_ERR_INVALID;
    std::lock_guard<std::mutex> lk(prof_mu);
    prof_collect_locked();
    for (int i = 0; i < PROF_NSLOTS; ++i)
        if (std::strcmp(name, kProfNames[i]) == 0) {
            if (total_ms) *total_ms = prof_ms[i];
            if (launches) *launches = prof_n[i];
            return GV_OK;
        }
    set_error(std::string("unknown profile slot ") + name);
    return GV_ERR_INVALID;
}

gv_status gv_config_init(gv_config *cfg, uint32_t num_vertices) {
    if (!cfg) return GV_ERR_INVALID;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->num_vertices = num_vertices;
    cfg->block_size = 128;
    cfg->threads_per_vertex = 8;
    cfg->directed = 0;
    cfg->weighted = 0;
    cfg->device = 0;
    cfg->pool_blocks = 0;
    cfg->hbm_budget_bytes = 0;
    cfg->max_batch_pairs = 1ull << 22;
    return GV_OK;
}

gv_status gv_create(const gv_config *cfg, gv_graph **out) {
    if (!cfg || !out) { set_error("null argument"); return GV_ERR_INVALID; }
    *out = nullptr;
    if (cfg->num_vertices == 0 || cfg->num_vertices > 0xFFFFFFF0u) { set_error("num_vertices out of range"); return GV_ERR_INVALID; }
    if (!valid_block(cfg->block_size)) { set_error("block_size must be 32, 64 or 128"); return GV_ERR_INVALID; }
    if (!valid_tpv(cfg->threads_per_vertex)) { set_error("threads_per_vertex must be 4, 8, 16 or 32"); return GV_ERR_INVALID; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_error("no CUDA device is visible; libgv has no CPU path");
        return GV_ERR_CUDA;
    }
    if (cfg->device < 0 || cfg->device >= ndev) { set_error("device ordinal out of range"); return GV_ERR_INVALID; }
    DeviceGuard dg(cfg->device);
    gv_graph *g = new gv_graph();
    g->cfg = *cfg;
    if (g->cfg.max_batch_pairs == 0) g->cfg.max_batch_pairs = 1ull << 16;
    const uint32_t n = cfg->num_vertices;
    g->bitsn = (n <= 1) ? 1u : (uint32_t)(32 - __builtin_clz(n - 1));
    const uint32_t B = cfg->block_size;
    uint64_t P = cfg->pool_blocks;
    const uint64_t per_block = (uint64_t)B * 4 * (cfg->weighted ? 2 : 1) + 6 * 4;
    const uint64_t dict = (uint64_t)n * (16 + 1 + 1 + 4 + 4);
    if (P == 0) {
        uint64_t budget = cfg->hbm_budget_bytes;
        if (budget == 0) {
            size_t fr = 0, tot = 0;
            cudaMemGetInfo(&fr, &tot);
            budget = fr / 2;
        }
        P = budget > dict ? (budget - dict) / per_block : 0;
    }
    if (P > 0xFFFFFFF0ull) P = 0xFFFFFFF0ull;
    if (P == 0) { delete g; set_error("HBM budget leaves no room for edge blocks"); return GV_ERR_NOMEM; }
    DevGraph &d = g->d;
    d.n = n;
    g->n_cap = n;
    d.B = B;
    d.logB = (uint32_t)__builtin_ctz(B);
    d.weighted = cfg->weighted ? 1 : 0;
    d.P = P;
    gv_status st = GV_OK;
    if ((st = dmalloc(&d.vtx, (size_t)n * sizeof(uint4), "vtx")) != GV_OK) goto fail;
    if ((st = dmalloc(&d.left, P * 4, "left")) != GV_OK) goto fail;
    if ((st = dmalloc(&d.right, P * 4, "right")) != GV_OK) goto fail;
    if ((st = dmalloc(&d.pred, P * 4, "pred")) != GV_OK) goto fail;
    if ((st = dmalloc(&d.bcount, P * 4, "bcount")) != GV_OK) goto fail;
    if ((st = dmalloc(&d.owner, P * 4, "owner")) != GV_OK) goto fail;
    if ((st = dmalloc(&d.pool, P * B * 4, "pool")) != GV_OK) goto fail;
    if (cfg->weighted && (st = dmalloc(&d.wpool, P * B * 4, "wpool")) != GV_OK) goto fail;
    if ((st = dmalloc(&d.free_stack, P * 4, "free_stack")) != GV_OK) goto fail;
    if ((st = dmalloc(&d.affected, n, "affected")) != GV_OK) goto fail;
    if ((st = dmalloc(&d.dirty, n, "dirty")) != GV_OK) goto fail;
    if ((st = dmalloc(&d.dirty_list, (size_t)n * 4, "dirty_list")) != GV_OK) goto fail;
    if ((st = dmalloc(&d.vbig_list, (size_t)n * 4, "vbig_list")) != GV_OK) goto fail;
    if ((st = dmalloc(&d.ctl, sizeof(Ctl), "ctl")) != GV_OK) goto fail;
    {
        cudaMemset(d.affected, 0, n);
        cudaMemset(d.dirty, 0, n);
        Ctl c;
        std::memset(&c, 0, sizeof(c));
        c.free_top = P;
        cudaMemcpy(d.ctl, &c, sizeof(c), cudaMemcpyHostToDevice);
        GV_LAUNCH(k_init_store, grid_for(P > n ? P : n, 256, 148 * 16), 256, 0, 0, d.vtx, n, d.free_stack,
                  (unsigned long long)P);
        const uint64_t E = g->cfg.max_batch_pairs * (cfg->directed ? 1 : 2);
        if ((st = ensure_batch_scratch(g, E, g->cfg.max_batch_pairs)) != GV_OK) goto fail;
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) { st = cuda_status(e, "gv_create"); goto fail; }
    }
    *out = g;
    return GV_OK;
fail:
    gv_destroy(g);
    return st;
}

gv_status gv_view_create(gv_graph *g, gv_graph **out) {
    if (!g || !out) { set_error("null argument"); return GV_ERR_INVALID; }
    if (g->parent) g = g->parent;
    DeviceGuard dg(g->cfg.device);
    gv_graph *v = new gv_graph();
    v->cfg = g->cfg;
    v->bitsn = g->bitsn;
    v->d = g->d;
    v->parent = g;
    g->nviews.fetch_add(1);
    v->weighted_alloc = g->weighted_alloc;
    // analytics need a scan scratch and a few words of their own
    const uint64_t elems = (uint64_t)g->d.n + 2;
    gv_status st = dmalloc((char **)&v->bs.scan_tmp, scan_scratch_bytes(elems), "view scan");
    if (st == GV_OK) st = dmalloc(&v->bs.tile_cnt, 64, "view words");
    if (st != GV_OK) {
        dfree(v->bs.scan_tmp);
        delete v;
        return st;
    }
    *out = v;
    return GV_OK;
}

gv_status gv_destroy(gv_graph *g) {
    if (!g) return GV_OK;
    DeviceGuard dg(g->cfg.device);
    if (g->parent) {  // a view: free only its own scratch
        g->parent->nviews.fetch_sub(1);
        dfree(g->bs.scan_tmp);
        dfree(g->bs.tile_cnt);
        if (g->an_buf) cudaFree(g->an_buf);
        if (g->host_pinned) cudaFreeHost(g->host_pinned);
        for (int i = 0; i < gv_graph::AUX_SLOTS; ++i)
            if (g->aux[i]) cudaFree(g->aux[i]);
        delete g;
        return GV_OK;
    }
    release_window(g);
    DevGraph &d = g->d;
    dfree(d.vtx); dfree(d.left); dfree(d.right); dfree(d.pred); dfree(d.bcount); dfree(d.owner);
    dfree(d.pool); dfree(d.wpool); dfree(d.free_stack); dfree(d.affected); dfree(d.dirty);
    dfree(d.dirty_list); dfree(d.vbig_list); dfree(d.ctl);
    free_batch_entries(g->bs);
    free_batch_inputs(g->bs);
    if (g->an_buf) cudaFree(g->an_buf);
    for (int i = 0; i < gv_graph::AUX_SLOTS; ++i)
        if (g->aux[i]) cudaFree(g->aux[i]);
    if (g->host_pinned) cudaFreeHost(g->host_pinned);
    delete g;
    return GV_OK;
}

static gv_status stage_pairs(gv_graph *g, const uint32_t *src, const uint32_t *dst, const float *w,
                             uint64_t k, int mem, cudaStream_t s, const uint32_t **dsrc,
                             const uint32_t **ddst, const float **dw) {
    if (mem == GV_MEM_DEVICE) {
        *dsrc = src; *ddst = dst; *dw = w;
        return GV_OK;
    }
    const uint32_t n = g->d.n;
    for (uint64_t i = 0; i < k; ++i)
        if (src[i] >= n || dst[i] >= n) {
            set_error("vertex id out of range at pair " + std::to_string(i));
            return GV_ERR_INVALID;
        }
    cudaError_t e = cudaMemcpyAsync(g->bs.in_src, src, k * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(g->bs.in_dst, dst, k * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && w) e = cudaMemcpyAsync(g->bs.in_w, w, k * 4, cudaMemcpyHostToDevice, s);
    *dsrc = g->bs.in_src; *ddst = g->bs.in_dst; *dw = w ? g->bs.in_w : nullptr;
    return cuda_status(e, "stage batch");
}

static gv_status update_common(gv_graph *g, const uint32_t *src, const uint32_t *dst, const float *w,
                               uint64_t k, int mem, void *stream, bool is_delete, bool force_directed) {
    if (!g || (k && (!src || !dst))) { set_error("null argument"); return GV_ERR_INVALID; }
    if (g->parent) { set_error("a view is read-only"); return GV_ERR_STATE; }
    if (mem != GV_MEM_HOST && mem != GV_MEM_DEVICE) { set_error("bad mem flag"); return GV_ERR_INVALID; }
    if (!is_delete && g->cfg.weighted && k && !w) { set_error("weighted store needs weights"); return GV_ERR_INVALID; }
    if (!g->cfg.weighted) w = nullptr;
    if (k == 0) return GV_OK;
    if (k > 0x7FFFFFFFull) { set_error("batch too large"); return GV_ERR_CAPACITY; }
    DeviceGuard dg(g->cfg.device);
    cudaStream_t s = (cudaStream_t)stream;
    const bool sym = !force_directed && !g->cfg.directed;
    gv_status st = ensure_batch_scratch(g, sym ? 2 * k : k, k);
    if (st != GV_OK) return st;
    const uint32_t *dsrc, *ddst;
    const float *dw;
    st = stage_pairs(g, src, dst, w, k, mem, s, &dsrc, &ddst, &dw);
    if (st != GV_OK) return st;
    return run_update(g, dsrc, ddst, dw, k, sym, is_delete, s);
}

gv_status gv_insert_edges(gv_graph *g, const uint32_t *src, const uint32_t *dst, const float *weights,
                          uint64_t k, int mem, void *stream) {
    return update_common(g, src, dst, weights, k, mem, stream, false, false);
}

gv_status gv_delete_edges(gv_graph *g, const uint32_t *src, const uint32_t *dst, uint64_t k, int mem,
                          void *stream) {
    return update_common(g, src, dst, nullptr, k, mem, stream, true, false);
}

gv_status gv_bulk_build_csr(gv_graph *g, const uint64_t *offsets, const uint32_t *dst,
                            const float *weights, int mem, void *stream) {
    if (!g || !offsets) { set_error("null argument"); return GV_ERR_INVALID; }
    if (g->parent) { set_error("a view is read-only"); return GV_ERR_STATE; }
    DeviceGuard dg(g->cfg.device);
    cudaStream_t s = (cudaStream_t)stream;
    Ctl c;
    gv_status st = read_ctl(g, &c, s);
    if (st != GV_OK) return st;
    if (c.live_edges != 0 || c.free_top != g->d.P) { set_error("bulk build needs an empty graph"); return GV_ERR_STATE; }
    const uint32_t n = g->d.n;
    if (mem == GV_MEM_HOST) {
        const uint64_t m = offsets[n];
        if (m && !dst) { set_error("null dst"); return GV_ERR_INVALID; }
        std::vector<uint32_t> src(m);
        for (uint32_t u = 0; u < n; ++u) {
            if (offsets[u] > offsets[u + 1]) { set_error("offsets not monotone"); return GV_ERR_INVALID; }
            for (uint64_t i = offsets[u]; i < offsets[u + 1]; ++i) src[i] = u;
        }
        return update_common(g, src.data(), dst, weights, m, GV_MEM_HOST, stream, false, true);
    }
    unsigned long long m = 0;
    cudaError_t e = cudaMemcpyAsync(&m, offsets + n, 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "bulk build");
    if (m == 0) return GV_OK;
    uint32_t *src = nullptr;
    if ((st = dmalloc(&src, m * 4, "csr sources")) != GV_OK) return st;
    GV_LAUNCH(k_csr_sources, grid_for(m, 256), 256, 0, s, (const unsigned long long *)offsets, n, m, src);
    st = update_common(g, src, dst, weights, m, GV_MEM_DEVICE, stream, false, true);
    cudaStreamSynchronize(s);
    cudaFree(src);
    return st;
}

// Per-vertex arrays grow to the next power of two (the reference sizes its
// dictionary with computeNearestPowerOf2, graphvine.cu:42, but cannot grow).
gv_status gv_add_vertices(gv_graph *g, uint32_t k, uint32_t *first, void *stream) {
    if (!g) { set_error("null argument"); return GV_ERR_INVALID; }
    if (g->parent) { set_error("a view is read-only"); return GV_ERR_STATE; }
    if (g->nviews.load() > 0) { set_error("destroy the graph's views before adding vertices"); return GV_ERR_STATE; }
    DeviceGuard dg(g->cfg.device);
    cudaStream_t s = (cudaStream_t)stream;
    DevGraph &d = g->d;
    const uint64_t n = d.n, nn = n + k;
    if (nn > 0xFFFFFFF0ull) { set_error("vertex count out of range"); return GV_ERR_INVALID; }
    if (first) *first = (uint32_t)n;
    if (k == 0) return GV_OK;
    cudaError_t e = cudaStreamSynchronize(s);  // work in flight still uses the old arrays
    if (e != cudaSuccess) return cuda_status(e, "add vertices");
    if (nn > g->n_cap) {
        uint64_t cap = 1;
        while (cap < nn) cap <<= 1;
        if (cap > 0xFFFFFFF0ull) cap = nn;
        uint4 *vtx = nullptr;
        uint8_t *aff = nullptr, *dirty = nullptr;
        uint32_t *dl = nullptr, *vb = nullptr;
        gv_status st = dmalloc(&vtx, cap * sizeof(uint4), "vtx");
        if (st == GV_OK) st = dmalloc(&aff, cap, "affected");
        if (st == GV_OK) st = dmalloc(&dirty, cap, "dirty");
        if (st == GV_OK) st = dmalloc(&dl, cap * 4, "dirty_list");
        if (st == GV_OK) st = dmalloc(&vb, cap * 4, "vbig_list");
        if (st != GV_OK) {
            dfree(vtx); dfree(aff); dfree(dirty); dfree(dl); dfree(vb);
            return st;
        }
        e = cudaMemcpy(vtx, d.vtx, n * sizeof(uint4), cudaMemcpyDeviceToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(aff, d.affected, n, cudaMemcpyDeviceToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(dirty, d.dirty, n, cudaMemcpyDeviceToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(dl, d.dirty_list, n * 4, cudaMemcpyDeviceToDevice);
        if (e != cudaSuccess) {
            dfree(vtx); dfree(aff); dfree(dirty); dfree(dl); dfree(vb);
            return cuda_status(e, "add vertices copy");
        }
        dfree(d.vtx); dfree(d.affected); dfree(d.dirty); dfree(d.dirty_list); dfree(d.vbig_list);
        d.vtx = vtx; d.affected = aff; d.dirty = dirty; d.dirty_list = dl; d.vbig_list = vb;
        g->n_cap = (uint32_t)cap;
    }
    GV_LAUNCH(k_init_store, grid_for(k, 256, 148 * 16), 256, 0, s, d.vtx + n, k, nullptr, 0ull);
    cudaMemsetAsync(d.affected + n, 0, k, s);
    cudaMemsetAsync(d.dirty + n, 0, k, s);
    d.n = (uint32_t)nn;
    g->bitsn = (nn <= 1) ? 1u : (uint32_t)(32 - __builtin_clz((uint32_t)(nn - 1)));
    // the scan scratch is sized for n + 1 elements: rebuild the batch scratch
    const uint64_t cap_e = g->bs.cap, cap_p = g->bs.in_cap;
    free_batch_entries(g->bs);
    g->bs.cap = 0;
    gv_status st = ensure_batch_scratch(g, std::max<uint64_t>(cap_e, 1), std::max<uint64_t>(cap_p, 1));
    if (st != GV_OK) return st;
    e = cudaStreamSynchronize(s);
    return cuda_status(e, "add vertices");
}

gv_status gv_delete_vertices(gv_graph *g, const uint32_t *ids, uint64_t k, uint32_t flags, int mem, void *stream) {
    if (!g || (k && !ids)) { set_error("null argument"); return GV_ERR_INVALID; }
    if (g->parent) { set_error("a view is read-only"); return GV_ERR_STATE; }
    DeviceGuard dg(g->cfg.device);
    cudaStream_t s = (cudaStream_t)stream;
    const uint32_t n = g->d.n;
    std::vector<uint32_t> h;
    const uint32_t *hid = ids;
    if (mem == GV_MEM_DEVICE && k) {
        h.resize(k);
        cudaError_t e = cudaMemcpyAsync(h.data(), ids, k * 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e, "delete vertices ids");
        hid = h.data();
    }
    std::vector<uint8_t> mark(n, 0);
    for (uint64_t i = 0; i < k; ++i) {
        if (hid[i] >= n) { set_error("vertex id out of range"); return GV_ERR_INVALID; }
        mark[hid[i]] = 1;
    }
    if (k == 0) return GV_OK;
    uint8_t *del = (uint8_t *)aux_scratch(g, 0, n);
    if (!del) return GV_ERR_NOMEM;
    cudaError_t e = cudaMemcpyAsync(del, mark.data(), n, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_status(e, "delete vertices flags");
    gv_status st = run_vertex_delete(g, del, s);
    if (st == GV_OK && (flags & GV_UPDATE_COMPACT)) st = run_compact(g, s);
    if (st != GV_OK) return st;
    return cuda_status(cudaStreamSynchronize(s), "delete vertices");
}

gv_status gv_compact(gv_graph *g, void *stream) {
    if (!g) return GV_ERR_INVALID;
    if (g->parent) { set_error("a view is read-only"); return GV_ERR_STATE; }
    DeviceGuard dg(g->cfg.device);
    return run_compact(g, (cudaStream_t)stream);
}

gv_status gv_synchronize(gv_graph *g, void *stream) {
    if (!g) return GV_ERR_INVALID;
    DeviceGuard dg(g->cfg.device);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "synchronize");
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, "pending launch error");
    unsigned st = 0;
    e = cudaMemcpy(&st, &g->d.ctl->status, sizeof(st), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e, "read status");
    if (st) cudaMemset(&g->d.ctl->status, 0, sizeof(st));
    return map_device_status(st);
}

gv_status gv_num_vertices(const gv_graph *g, uint32_t *n) {
    if (!g || !n) return GV_ERR_INVALID;
    *n = g->d.n;
    return GV_OK;
}

gv_status gv_get_config(const gv_graph *g, gv_config *cfg) {
    if (!g || !cfg) return GV_ERR_INVALID;
    *cfg = g->cfg;
    cfg->pool_blocks = g->d.P;
    return GV_OK;
}

gv_status gv_num_edges(gv_graph *g, uint64_t *live) {
    if (!g || !live) return GV_ERR_INVALID;
    DeviceGuard dg(g->cfg.device);
    Ctl c;
    gv_status st = read_ctl(g, &c, 0);
    if (st == GV_OK) *live = c.live_edges;
    return st;
}

gv_status gv_pool_stats(gv_graph *g, uint64_t *capacity, uint64_t *free_blocks) {
    if (!g) return GV_ERR_INVALID;
    DeviceGuard dg(g->cfg.device);
    Ctl c;
    gv_status st = read_ctl(g, &c, 0);
    if (st != GV_OK) return st;
    if (capacity) *capacity = g->d.P;
    if (free_blocks) *free_blocks = c.free_top;
    return GV_OK;
}

gv_status gv_vertex_records(gv_graph *g, const void **records) {
    if (!g || !records) return GV_ERR_INVALID;
    *records = g->d.vtx;
    return GV_OK;
}

gv_status gv_degrees(gv_graph *g, uint32_t *deg, int mem, void *stream) {
    if (!g || !deg) return GV_ERR_INVALID;
    DeviceGuard dg(g->cfg.device);
    cudaStream_t s = (cudaStream_t)stream;
    if (mem == GV_MEM_DEVICE) {
        launch_degrees(g, deg, s);
        return cuda_status(cudaGetLastError(), "degrees");
    }
    uint32_t *tmp = nullptr;
    gv_status st = dmalloc(&tmp, (size_t)g->d.n * 4, "degrees");
    if (st != GV_OK) return st;
    launch_degrees(g, tmp, s);
    cudaError_t e = cudaMemcpyAsync(deg, tmp, (size_t)g->d.n * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(tmp);
    return cuda_status(e, "degrees");
}

gv_status gv_export_csr(gv_graph *g, uint64_t *offsets, uint32_t *dst, float *weights, uint64_t cap,
                        int mem, void *stream) {
    if (!g || !offsets) return GV_ERR_INVALID;
    if (weights && !g->cfg.weighted) { set_error("graph has no weights"); return GV_ERR_INVALID; }
    DeviceGuard dg(g->cfg.device);
    cudaStream_t s = (cudaStream_t)stream;
    const uint32_t n = g->d.n;
    uint32_t *deg = nullptr;
    unsigned long long *off = nullptr;
    gv_status st = dmalloc(&deg, (size_t)n * 4, "export deg");
    if (st != GV_OK) return st;
    if (mem == GV_MEM_DEVICE) off = (unsigned long long *)offsets;
    else if ((st = dmalloc(&off, ((size_t)n + 1) * 8, "export offsets")) != GV_OK) { cudaFree(deg); return st; }
    launch_degrees(g, deg, s);
    scan_exclusive_u32_to_u64(deg, off, n, off + n, g->bs.scan_tmp, s);
    unsigned long long m = 0;
    cudaError_t e = cudaMemcpyAsync(&m, off + n, 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { st = cuda_status(e, "export"); goto done; }
    if (m > cap) { set_error("export capacity " + std::to_string(cap) + " < " + std::to_string(m)); st = GV_ERR_CAPACITY; goto done; }
    if (m && !dst) { st = GV_ERR_INVALID; goto done; }
    if (mem == GV_MEM_DEVICE) {
        st = run_export(g, off, dst, weights, s);
        if (st == GV_OK) st = cuda_status(cudaStreamSynchronize(s), "export");
    } else {
        uint32_t *ddst = nullptr;
        float *dw = nullptr;
        if ((st = dmalloc(&ddst, m * 4 + 4, "export dst")) != GV_OK) goto done;
        if (weights && (st = dmalloc(&dw, m * 4 + 4, "export w")) != GV_OK) { cudaFree(ddst); goto done; }
        st = run_export(g, off, ddst, dw, s);
        if (st == GV_OK) {
            e = cudaMemcpyAsync(offsets, off, ((size_t)n + 1) * 8, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess && m) e = cudaMemcpyAsync(dst, ddst, m * 4, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess && weights && m) e = cudaMemcpyAsync(weights, dw, m * 4, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            st = cuda_status(e, "export copy");
        }
        cudaFree(ddst);
        if (dw) cudaFree(dw);
        cudaFree(off);
    }
done:
    cudaFree(deg);
    return st;
}

gv_status gv_affected(gv_graph *g, uint8_t *affected, int mem, void *stream) {
    if (!g || !affected) return GV_ERR_INVALID;
    DeviceGuard dg(g->cfg.device);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemcpyAsync(affected, g->d.affected, g->d.n,
                                    mem == GV_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && mem != GV_MEM_DEVICE) e = cudaStreamSynchronize(s);
    return cuda_status(e, "affected");
}

gv_status gv_clear_affected(gv_graph *g, void *stream) {
    if (!g) return GV_ERR_INVALID;
    DeviceGuard dg(g->cfg.device);
    return cuda_status(cudaMemsetAsync(g->d.affected, 0, g->d.n, (cudaStream_t)stream), "clear affected");
}

gv_status gv_last_stat(gv_graph *g, const char *key, double *value) {
    if (!g || !key || !value) return GV_ERR_INVALID;
    DeviceGuard dg(g->cfg.device);
    if (std::strcmp(key, "tc_work") == 0 || std::strcmp(key, "tc_oriented_edges") == 0 ||
        std::strcmp(key, "tc_probes") == 0 || std::strcmp(key, "tc_core") == 0) {
        if (key[3] == 'o') {
            *value = (double)g->last_tc_oriented;
            return GV_OK;
        }
        // work counters of the last count (per-graph scratch words): [1] merged
        // entries, [2] core bit probes, [3] core vertices
        const int word = key[3] == 'w' ? 1 : key[4] == 'r' ? 2 : 3;
        unsigned long long w = 0;
        cudaError_t e = cudaMemcpy(&w, (unsigned long long *)g->bs.tile_cnt + word, 8, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) *value = (double)w;
        return cuda_status(e, key);
    }
    if (std::strcmp(key, "tc_subset_local") == 0) {
        *value = (double)g->last_tc_local;
        return GV_OK;
    }
    if (std::strcmp(key, "sweeps") == 0) {
        *value = (double)g->last_sweeps;
        return GV_OK;
    }
    if (window_stat(g, key, value)) return GV_OK;
    set_error(std::string("unknown stat ") + key);
    return GV_ERR_INVALID;
}

gv_status gv_check(gv_graph *g, uint64_t *violations, uint32_t *first_code, uint32_t *first_vertex) {
    if (!g || !violations) return GV_ERR_INVALID;
    DeviceGuard dg(g->cfg.device);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_status(e, "check");
    return run_check(g, violations, first_code, first_vertex);
}

}  // extern "C"
