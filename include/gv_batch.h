/*
 * gv_batch.h — batched updates, batched queries and the autotuner.
 *
 * No direct reference counterpart: the reference applies one batch per
 * synchronous host call (GraphVine::batchInsert / batchDelete,
 * src/dynamicStructure/graphvine.cu:222-451) and answers one query per call.
 */
#ifndef GV_BATCH_H
#define GV_BATCH_H
#include "gv.h"
#ifdef __cplusplus
extern "C" {
#endif

/* One update batch of a window: pairs [offset, offset + n_insert) of the
 * window's src/dst arrays are inserted, then pairs
 * [offset + n_insert, offset + n_insert + n_delete) are deleted. */
typedef struct gv_batch_desc {
    uint64_t offset;
    uint32_t n_insert;
    uint32_t n_delete;
} gv_batch_desc;

enum {
    GV_BATCH_COMPACT = 1u, /* compact once after the window */
    GV_BATCH_GRAPH = 2u    /* run the window as a CUDA graph, captured once per capacity (entries
                              rounded up to a power of two) and replayed for later windows */
};

/* Applies nbatches batches in order; the final graph equals applying them
 * one by one with gv_insert_edges / gv_delete_edges.  The window is reduced
 * to the last operation per pair and applied by one persistent launch that
 * scans every touched vertex once (when the free blocks cover the window's
 * worst case; else by an exact two-stage pass, see batch.cu).
 * descs is host memory; src/dst are `mem` (total pairs = sum of the batch
 * sizes, batches laid out consecutively).  A window that names an id >= n
 * or exhausts the pool is rejected whole (gv_synchronize reports it).
 * Unweighted stores only. */
gv_status gv_batch_run(gv_graph *g, const gv_batch_desc *descs, uint32_t nbatches, const uint32_t *src,
                       const uint32_t *dst, int mem, uint32_t flags, void *stream);

/* A window of update batches, then k <= 32 personalised PageRank queries on
 * the graph the window leaves, as one unit of device work: with
 * GV_BATCH_GRAPH the window and the queries' sweeps are one CUDA graph,
 * captured once per (capacity, k, max_iter, alpha, epsilon) and replayed
 * for later windows (every size is read on the device).  max_iter sweeps
 * are issued; once every query's L1 step is below epsilon the remaining ones
 * return at once.  sources: host array of k ids.  x_out: n * k floats,
 * vertex-major (x_out[v * k + j] is query j at v), in `mem` memory like
 * src/dst; *sweeps gets the sweeps that ran.  nbatches may be 0 (queries
 * only).  Synchronous.  No reference counterpart (the reference answers one
 * query per host call). */
gv_status gv_batch_run_ppr(gv_graph *g, const gv_batch_desc *descs, uint32_t nbatches, const uint32_t *src,
                           const uint32_t *dst, int mem, uint32_t flags, const uint32_t *sources, uint32_t k,
                           float alpha, float epsilon, int32_t max_iter, float *x_out, int32_t *sweeps,
                           void *stream);

/* k personalised PageRank queries (k <= 32) in one pass per sweep: every
 * adjacency read serves all k sources.  x_out[v * k + j] is query j's value
 * at v (vertex-major), sweeps stop when every query's L1 step < epsilon.
 * Undirected unweighted stores take the degree-ordered sweep plan (one
 * query: its single-vector sweep); GV_PR_PLAN=0, directed and weighted
 * stores the store's batched sweep. */
gv_status gv_ppr_batch(gv_graph *g, const uint32_t *sources, uint32_t k, float alpha, float epsilon,
                       int32_t max_iter, float *x_out, int32_t *sweeps, int mem, void *stream);

/* Autotuner: times a sample workload (build from src0/dst0, one window of
 * batches, one PageRank) for every edge-block size {32, 64, 128} and
 * threads-per-vertex {4, 8, 16, 32}: one warm-up round, then the median of
 * three rounds, each on a freshly built graph; writes one result per
 * candidate and the fastest configuration into *best (base config
 * otherwise). */
typedef struct gv_tune_result {
    uint32_t block_size;
    uint32_t threads_per_vertex;
    float update_ms;
    float pagerank_ms;
} gv_tune_result;

gv_status gv_autotune(const gv_config *base, const uint32_t *src0, const uint32_t *dst0, uint64_t k0,
                      const gv_batch_desc *descs, uint32_t nbatches, const uint32_t *bsrc, const uint32_t *bdst,
                      int mem, gv_tune_result *results, uint32_t *nresults, gv_config *best);

#ifdef __cplusplus
}
#endif
#endif
