// Host-side definition of a graph and the launch helpers the C ABI calls.
#pragma once
#include <cstdint>
#include <atomic>
#include <string>
#include <cuda_runtime.h>
#include "../../include/gv.h"
#include "common.cuh"

namespace gv {

// Thresholds between the lane-group path and the CTA-per-vertex path.
constexpr uint32_t BIG_BLOCKS = 64;    // vertices with more blocks go to a whole CTA
constexpr uint32_t BIG_SEGMENT = 2048; // batch segments with more entries go to a whole CTA
constexpr int BIG_THREADS = 512;

struct BatchScratch {
    uint64_t cap = 0;  // directed entries
    unsigned long long *keys = nullptr, *keys_alt = nullptr;
    uint32_t *vals = nullptr, *vals_alt = nullptr;
    uint32_t *rs_counts = nullptr;
    void *scan_tmp = nullptr;
    unsigned long long *tile_cnt = nullptr;  // packed (uniq << 32 | heads) per tile
    uint32_t *bdst = nullptr;
    float *bw = nullptr;
    uint8_t *found = nullptr;
    uint32_t *seg_vertex = nullptr, *seg_start = nullptr, *seg_found = nullptr;
    uint32_t *seg_newblocks = nullptr, *seg_blkbase = nullptr, *big_list = nullptr;
    uint64_t in_cap = 0;  // pairs
    uint32_t *in_src = nullptr, *in_dst = nullptr;
    float *in_w = nullptr;
};

}  // namespace gv

struct gv_graph {
    gv_config cfg;
    uint32_t bitsn = 1;
    gv::DevGraph d{};
    gv::BatchScratch bs;
    bool weighted_alloc = false;
    // lazily allocated analytics scratch
    void *an_buf = nullptr;
    size_t an_bytes = 0;
    void *host_pinned = nullptr;
    size_t host_pinned_bytes = 0;
    // facts about the last analytics calls (gv_last_stat)
    uint64_t last_tc_oriented = 0;
    int32_t last_tc_local = 0;  // 1: the last subset count took the local path
    int32_t last_sweeps = 0;
    // independent auxiliary device buffers, grown on demand
    static constexpr int AUX_SLOTS = 16;
    void *aux[AUX_SLOTS] = {};
    size_t aux_bytes[AUX_SLOTS] = {};
    // a view shares the parent's store and owns only analytics scratch
    gv_graph *parent = nullptr;
    std::atomic<int> nviews{0};  // live views of this graph (growth waits for none)
    uint32_t n_cap = 0;          // vertices the per-vertex arrays hold
};

namespace gv {

void set_error(const std::string &msg);
gv_status cuda_status(cudaError_t e, const char *what);
gv_status ensure_batch_scratch(gv_graph *g, uint64_t entries, uint64_t pairs);
void *analytics_scratch(gv_graph *g, size_t bytes);
// Auxiliary buffer `slot` (0..AUX_SLOTS-1) of at least `bytes`, kept across calls.
void *aux_scratch(gv_graph *g, int slot, size_t bytes);
// Frees the analytics and auxiliary scratch (it is allocated again on demand).
void release_analytics_scratch(gv_graph *g);
// Device-to-host copy of the control block (synchronises the stream).
gv_status read_ctl(gv_graph *g, Ctl *out, cudaStream_t s);

// Update pipeline stages (launch only).
gv_status run_update(gv_graph *g, const uint32_t *dsrc, const uint32_t *ddst, const float *dw,
                     uint64_t k, bool symmetric, bool is_delete, cudaStream_t s);
// Segment + membership + apply from keys already sorted (src << bitsn | dst);
// V = original entry index per key (weighted inserts), else nullptr.
gv_status apply_sorted(gv_graph *g, const unsigned long long *K, const uint32_t *V, uint64_t E, bool symmetric,
                       const float *dw, bool is_delete, bool finish, cudaStream_t s);
void launch_commit_keep_abort(gv_graph *g, cudaStream_t s);
// One persistent launch applying a window's net segments (both operations;
// btype[i] = 1 for an insert), then the commit of its block allocation.
// queue[0..2] must be zero; big_list holds up to nseg entries.
gv_status launch_window_apply(gv_graph *g, const uint32_t *seg_vertex, const uint32_t *seg_start,
                              const uint32_t *bdst, const uint32_t *btype, uint8_t *found, uint32_t *big_list,
                              unsigned long long *queue, cudaStream_t s);
void launch_finish(gv_graph *g, cudaStream_t s);
void release_window(gv_graph *g);
// Window counters of gv_batch_run (keys window_captures, window_replays,
// window_persistent, window_exact); false for other keys.
bool window_stat(gv_graph *g, const char *key, double *value);
gv_status run_compact(gv_graph *g, cudaStream_t s);
// Tombstones every entry whose source or destination is flagged in del[n].
gv_status run_vertex_delete(gv_graph *g, const uint8_t *del, cudaStream_t s);
gv_status run_export(gv_graph *g, unsigned long long *offsets, uint32_t *dst, float *w,
                     cudaStream_t s);
gv_status run_check(gv_graph *g, uint64_t *violations, uint32_t *code, uint32_t *vertex);
void launch_degrees(gv_graph *g, uint32_t *deg, cudaStream_t s);
// PageRank (x_init / source as gv_pagerank's internals take them) over a
// degree-ordered padded CSR built for the call (prplan.cu).  *planned =
// false, with nothing done, when the graph does not qualify (directed or
// weighted stores, more than 2^32 padded entries, GV_PR_PLAN=0).
bool plan_pagerank_enabled(gv_graph *g);
gv_status plan_pagerank(gv_graph *g, float alpha, float eps, int max_iter, const float *x_init, int init_mem,
                        uint32_t source, float *x_out, int32_t *sweeps, int mem, cudaStream_t s, bool *planned);
// k personalised PageRank queries over the sweep plan (sources in src_mem
// memory); *planned false when the plan does not take them (k outside 2..32,
// or a graph the plan cannot hold).
gv_status plan_ppr_batch(gv_graph *g, const uint32_t *sources, int src_mem, uint32_t k, float alpha, float eps,
                         int max_iter, float *x_out, int32_t *sweeps, int mem, cudaStream_t s, bool *planned);
// Incident-triangle counts of the subset d_sub[ns] (device) into d_out[ns]
// from neighbour hash sets, without a whole-graph pass.  *done = false (and
// nothing written) when the subset's neighbourhoods are too large for that
// to pay, unless force.
gv_status tc_local_subset(gv_graph *g, const uint32_t *d_sub, uint64_t ns, unsigned long long *d_out,
                          cudaStream_t s, bool *done, bool force);

template <int T>
struct Tpv {
    static constexpr int value = T;
};

// Calls f(Tpv<t>{}) for the configured threads-per-vertex t.
template <typename F>
void dispatch_tpv(uint32_t tpv, F &&f) {
    switch (tpv) {
        case 4: f(Tpv<4>{}); break;
        case 8: f(Tpv<8>{}); break;
        case 16: f(Tpv<16>{}); break;
        default: f(Tpv<32>{}); break;
    }
}

// Grid size for grid-stride kernels: a few CTAs per SM.
unsigned grid_for(uint64_t work_items, unsigned per_cta, unsigned max_ctas = 148 * 8);

}  // namespace gv
