/*
 * gv_serve.h — a request loop over a device-resident graph.
 *
 * Update batches and queries arrive over time.  The loop applies runs of
 * arrived updates as one coalesced window (gv_batch_run) and runs arrived
 * queries concurrently, each group on its own worker thread, stream and
 * read-only view, admitted while a slot is free and the group's scratch
 * estimate fits the HBM budget.  Queries that arrive while others run are
 * admitted as slots free up (continuous batching): arrived PPR queries are
 * merged into batched launches of up to ppr_batch, arrived triangle-subset
 * queries share one count per slot, arrived BC queries run in pairs whose
 * sources share one set of BFS passes (gv_bc_multi).  The kinds of one
 * dispatch take turns, shortest first (triangle counts, PPR, BC): a kind's
 * groups start once the previous kind's have finished.  A worker keeps its
 * scratch for its next group of the same kind, charged to the budget.
 * Epochs: with fresh = 0 a query sees exactly the updates
 * that arrived before it; with fresh = 1 (the default) it sees at least
 * those, so queries that arrive behind an update wait for it and run
 * together after it.  results[i].epoch names the updates each query saw (the
 * first epoch update requests in trace order).  No reference counterpart (the
 * reference has no serving path).
 */
#ifndef GV_SERVE_H
#define GV_SERVE_H
#include "gv_batch.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef enum gv_req_kind { GV_REQ_UPDATE = 0, GV_REQ_PPR = 1, GV_REQ_TC = 2, GV_REQ_BC = 3 } gv_req_kind;

typedef struct gv_request {
    uint32_t kind;     /* gv_req_kind                                                  */
    uint32_t count0;   /* update: inserts; TC / BC: vertices in the slice of qvert      */
    uint32_t count1;   /* update: deletes                                               */
    uint32_t source;   /* PPR source                                                    */
    uint64_t offset;   /* update: first pair in src/dst (updates laid out in trace
                          order); TC / BC: first vertex in qvert                        */
    double arrival_s;  /* seconds after the start of the trace                          */
} gv_request;

typedef struct gv_request_result {
    double start_s;    /* when its work was issued (seconds after the start)            */
    double done_s;     /* when its result was complete                                  */
    double latency_ms; /* done - arrival                                                */
    uint32_t epoch;    /* update requests applied before it ran                         */
    uint32_t status;   /* gv_status                                                     */
    uint32_t sweeps;   /* PPR sweeps                                                    */
    uint32_t group;    /* requests run together share a group id                       */
} gv_request_result;

typedef struct gv_serve_config {
    uint32_t slots;            /* concurrent query workers                              */
    uint32_t ppr_batch;        /* PPR queries per batched launch (<= 32)                */
    uint32_t max_coalesce;     /* update requests merged into one window                */
    uint32_t pace;             /* 1: honour arrival times, 0: everything arrives at 0   */
    uint64_t hbm_budget_bytes; /* admission budget for in-flight query scratch          */
    float alpha;
    float epsilon;
    int32_t max_iter;
    uint32_t fresh;            /* 1: a query sees at least the updates that arrived before it
                                  (the loop applies every arrived update, then runs every
                                  arrived query together); 0: exactly those updates       */
} gv_serve_config;

/* Optional host buffers for results, indexed by request (entries may be
 * NULL): ppr[i] n floats, tc[i] count0 incident-triangle counts, bc[i] n floats. */
typedef struct gv_serve_outputs {
    float **ppr;
    uint64_t **tc;
    float **bc;
} gv_serve_outputs;

gv_status gv_serve_config_init(gv_serve_config *cfg);

/* Runs the trace to completion on g (host arrays) and fills results[nreq]. */
gv_status gv_serve_trace(gv_graph *g, const gv_serve_config *cfg, const gv_request *reqs, uint32_t nreq,
                         const uint32_t *src, const uint32_t *dst, const uint32_t *qvert,
                         gv_request_result *results, const gv_serve_outputs *outs);

#ifdef __cplusplus
}
#endif
#endif
