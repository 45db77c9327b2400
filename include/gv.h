/*
 * gv.h — C ABI of libgv, a B200 (sm_100a) dynamic-graph store and the
 * analytics that traverse it.
 *
 * The store is GraphVine's per-vertex edge-block complete binary tree (CBT):
 * every vertex owns a tree of fixed-size edge blocks; block k of a vertex has
 * children 2k+1 and 2k+2 and a level-order predecessor k-1.  Blocks come from
 * one preallocated pool and return to it on compaction.
 *
 * Conventions (all entry points):
 *   - vertex ids are 0-based uint32_t (the reference keeps 1-based ids inside
 *     edge blocks; the C++ shim in graphvine.hpp converts);
 *   - every call returns a gv_status and never aborts the process;
 *   - device work is ordered on the caller's stream (`stream` is a
 *     cudaStream_t passed as void*, NULL = legacy default stream);
 *   - `mem` says where an input/output array lives: GV_MEM_HOST (pageable or
 *     pinned host memory; the call copies through its own staging) or
 *     GV_MEM_DEVICE (caller-owned device memory);
 *   - errors found on the device (pool exhausted, vertex id out of range) are
 *     latched in a device status word; gv_synchronize() waits for the stream
 *     and returns it.  A batch that would exhaust the pool is rejected as a
 *     whole and leaves the graph unchanged;
 *   - a gv_graph is not safe for concurrent use from several host threads
 *     without external locking.
 */
#ifndef GV_H
#define GV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gv_graph gv_graph;

typedef enum gv_status {
    GV_OK = 0,
    GV_ERR_INVALID = 1,     /* bad argument: null pointer, bad config, vertex id >= n */
    GV_ERR_NOMEM = 2,       /* block pool / HBM budget exhausted; graph unchanged      */
    GV_ERR_CUDA = 3,        /* CUDA runtime error; see gv_last_error_string()          */
    GV_ERR_TIMEOUT = 4,     /* a bounded device-side wait expired                       */
    GV_ERR_STATE = 5,       /* call not valid for this graph (e.g. TC on a directed store) */
    GV_ERR_UNSUPPORTED = 6, /* feature not built into this library                      */
    GV_ERR_CAPACITY = 7     /* batch larger than the scratch the graph was created with */
} gv_status;

enum { GV_MEM_HOST = 0, GV_MEM_DEVICE = 1 };

/* Update flag: compact after the deletes (gv_update_tc, gv_delete_vertices). */
#define GV_UPDATE_COMPACT 1u

/* Store configuration.  Replaces the reference's compile-time constants
 * (include/dynamicStructure/constants.cuh:4-19: EDGE_BLOCK_SIZE,
 * THREADS_PER_BLOCK, DIRECTED) and its "half of device memory" pool sizing
 * (src/dynamicStructure/graphvine.cu:466-491). */
typedef struct gv_config {
    uint32_t num_vertices;       /* n; vertex ids are [0, n)                               */
    uint32_t block_size;         /* entries per edge block: 32, 64 or 128                  */
    uint32_t threads_per_vertex; /* lanes that walk one vertex's blocks: 4, 8, 16 or 32    */
    uint32_t directed;           /* 0: gv_insert_edges/gv_delete_edges apply both (u,v),(v,u) */
    uint32_t weighted;           /* 1: every entry carries a float weight                  */
    int32_t device;              /* CUDA device ordinal                                    */
    uint64_t pool_blocks;        /* block pool capacity; 0 = derive from hbm_budget_bytes  */
    uint64_t hbm_budget_bytes;   /* bytes for pool + dictionary; 0 = half of free memory   */
    uint64_t max_batch_pairs;    /* scratch sized for update batches of up to this size    */
} gv_config;

/* Fills defaults for n vertices: block 128, 8 threads/vertex, undirected,
 * unweighted, device 0, budget = half of free memory, batches up to 2^22 pairs. */
gv_status gv_config_init(gv_config *cfg, uint32_t num_vertices);

/* Replaces GraphVine::GraphVine(CSR*) allocation half
 * (src/dynamicStructure/graphvine.cu:5-35, :38-130). */
gv_status gv_create(const gv_config *cfg, gv_graph **out);
/* The reference never frees (include/dynamicStructure/graphvine.cuh:32).
 * Destroying a view frees only the view. */
gv_status gv_destroy(gv_graph *g);

/* A read-only view of g: it shares g's device-resident store and owns its
 * own analytics scratch, so queries on different views (each on its own
 * stream and host thread) can run concurrently.  Updates through a view
 * return GV_ERR_STATE; the caller orders updates on g after queries on
 * views.  Destroy views before g.  No reference counterpart: the reference
 * keeps one global store per process (src/dynamicStructure/graphvine.cu:3). */
gv_status gv_view_create(gv_graph *g, gv_graph **view);

/* Bulk build from a CSR of directed entries: offsets[n+1] (uint64), dst[m].
 * Self-loops and duplicates are dropped, every other entry is stored as
 * given (no symmetrisation).  Replaces GraphVine::bulkBuild
 * (src/dynamicStructure/graphvine.cu:181-220).  Valid on an empty graph only. */
gv_status gv_bulk_build_csr(gv_graph *g, const uint64_t *offsets, const uint32_t *dst,
                            const float *weights, int mem, void *stream);

/* Set-union insert of k pairs (src[i], dst[i]); on an undirected graph both
 * directions are inserted.  Self-loops and pairs already present are no-ops,
 * and the first occurrence wins among duplicates in the batch (its weight is
 * kept).  Replaces GraphVine::batchInsert
 * (src/dynamicStructure/graphvine.cu:222-371). */
gv_status gv_insert_edges(gv_graph *g, const uint32_t *src, const uint32_t *dst,
                          const float *weights, uint64_t k, int mem, void *stream);

/* Set-difference delete of k pairs (both directions on an undirected graph):
 * matching entries are tombstoned until gv_compact.  Replaces
 * GraphVine::batchDelete (src/dynamicStructure/graphvine.cu:373-451). */
gv_status gv_delete_edges(gv_graph *g, const uint32_t *src, const uint32_t *dst,
                          uint64_t k, int mem, void *stream);

/* Adds k isolated vertices with ids n .. n + k - 1 (*first = n).  The vertex
 * table grows to the next power of two when it is full; the store's blocks
 * stay where they are.  The reference has no vertex insert (its menu option
 * 3, src/main.cu:80, :122-124, is empty) and sizes its dictionary once
 * (computeNearestPowerOf2, graphvine.cu:42).  Fails with GV_ERR_STATE while
 * views of g exist.  Synchronous. */
gv_status gv_add_vertices(gv_graph *g, uint32_t k, uint32_t *first, void *stream);

/* Removes every edge incident to the k listed vertices (their own entries
 * and every entry pointing at them, on directed stores too); the ids stay
 * valid, isolated.  flags & GV_UPDATE_COMPACT compacts afterwards.  No
 * reference counterpart (src/main.cu:122-124).  Synchronous. */
gv_status gv_delete_vertices(gv_graph *g, const uint32_t *ids, uint64_t k, uint32_t flags, int mem, void *stream);

/* Fills tombstone holes, returns emptied tail blocks to the pool and unlinks
 * them from their CBT parents; the neighbour set is unchanged.  Replaces
 * GraphVine::compaction (src/dynamicStructure/graphvine.cu:453-464). */
gv_status gv_compact(gv_graph *g, void *stream);

/* Waits for `stream` and returns (then clears) the latched device status. */
gv_status gv_synchronize(gv_graph *g, void *stream);

/* Graph facts.  Synchronous. */
gv_status gv_num_vertices(const gv_graph *g, uint32_t *n);
gv_status gv_num_edges(gv_graph *g, uint64_t *live_entries);     /* stored directed entries */
gv_status gv_pool_stats(gv_graph *g, uint64_t *capacity_blocks, uint64_t *free_blocks);
gv_status gv_get_config(const gv_graph *g, gv_config *cfg);

/* Per-vertex degree (live entries) into deg[n] (uint32). */
gv_status gv_degrees(gv_graph *g, uint32_t *deg, int mem, void *stream);

/* Device address of the vertex records: n records of four uint32 each,
 * {first block (pool index, 0xFFFFFFFF if none), filled slots, live
 * entries, last block}.  Read-only for the caller; valid until the next
 * call that adds vertices or destroys the graph.  Replaces
 * GraphVine::getVertexDictionary (graphvine.cu:493-495), whose
 * VertexDictionary the reference's algorithm kernels walk. */
gv_status gv_vertex_records(gv_graph *g, const void **records);

/* Snapshot of the live adjacency as CSR, each vertex's entries in storage
 * order.  offsets[n+1] (uint64), dst[cap], weights[cap] (nullable).
 * Synchronous; returns GV_ERR_CAPACITY if cap < live entries. */
gv_status gv_export_csr(gv_graph *g, uint64_t *offsets, uint32_t *dst, float *weights,
                        uint64_t cap, int mem, void *stream);

/* Applies one batch as gv_insert_edges, gv_delete_edges and (flags &
 * GV_UPDATE_COMPACT) gv_compact would, and returns the exact change of the
 * triangle counts it causes: *delta_total, and optionally delta_owner[n], the
 * change of the triangles each vertex owns (smallest id, as gv_tc counts
 * them).  Work is proportional to the degrees of the pairs that really
 * changed, not to the graph.  Undirected stores; the whole call is rejected
 * (graph unchanged) on an id >= n.  Replaces dynamic_tc
 * (src/algorithm/tc/tc.cu:29-64, tc_kernel.cu:76-147), which recounts only
 * the owned triangles of vertices touched by the batch and so misses
 * triangles whose owner was not touched.  Synchronous. */
gv_status gv_update_tc(gv_graph *g, const uint32_t *ins_src, const uint32_t *ins_dst, const float *ins_w,
                       uint64_t n_ins, const uint32_t *del_src, const uint32_t *del_dst, uint64_t n_del,
                       uint32_t flags, int64_t *delta_total, int64_t *delta_owner, int mem, void *stream);

/* Vertices touched by updates since the last gv_clear_affected (endpoints of
 * every inserted or deleted entry, duplicates included).  affected[n] uint8.
 * Replaces find_affected_nodes (src/dynamicStructure/kernels/insert_kernels.cu:182-198)
 * and GraphVine::getAffectedNodesPointer (graphvine.cu:501-503). */
gv_status gv_affected(gv_graph *g, uint8_t *affected, int mem, void *stream);
gv_status gv_clear_affected(gv_graph *g, void *stream);

/* Structural invariant check on the device: CBT child/predecessor links,
 * per-block counts, owners, live counts, and that used + free blocks cover
 * the pool exactly once.  Synchronous.  *violations = 0 on a sound store;
 * *first_code names the first failed check: 1 root/fill mismatch, 2 live >
 * fill, 3 block index out of the pool, 4 wrong owner, 5 wrong block count,
 * 6 wrong predecessor, 7/8 left/right child link disagrees with the CBT
 * shape, 9 last-block record wrong, 10 live count wrong, 11 block not used
 * or free exactly once, 12 free-stack entry out of the pool, 13 free-stack
 * size inconsistent. */
gv_status gv_check(gv_graph *g, uint64_t *violations, uint32_t *first_code,
                   uint32_t *first_vertex);

/* Facts about the last analytics call on this graph: "tc_work" = list
 * entries the last whole-graph triangle count read (|N+(u)| + |N+(v)| merged
 * per oriented edge; with GV_TC_PACKED=1 probes of N+(v) plus inserts of
 * N+(u)), "tc_probes" / "tc_core" (bit probes against the dense-core rows
 * and core vertices of the last total-only count; 0 when it merged every
 * edge), "tc_oriented_edges", "tc_subset_local" (1 if the last subset count
 * took the neighbour-hash path), "sweeps" (last PageRank), and counts of
 * gv_batch_run windows: "window_persistent" / "window_exact" (windows that
 * took the persistent one-launch apply / the two-stage exact path),
 * "window_captures" / "window_replays" (CUDA graphs captured / replayed).
 * Synchronous. */
gv_status gv_last_stat(gv_graph *g, const char *key, double *value);

/* ---- analytics ---------------------------------------------------------- */

/* PageRank: x0 = 1/n; x <- (1-alpha)/n + alpha * sum_{u->v} x_u / deg(u);
 * stops when sum|x' - x| < epsilon or after max_iter sweeps; no dangling-mass
 * redistribution.  x_out[n] float.  *sweeps = sweeps performed.  Replaces
 * static_pagerank (src/algorithm/pagerank/pagerank.cu:3-68,
 * src/algorithm/pagerank/pr_kernel.cu:3-48).  Synchronous (reads *sweeps). */
gv_status gv_pagerank(gv_graph *g, float alpha, float epsilon, int32_t max_iter,
                      float *x_out, int32_t *sweeps, int mem, void *stream);

/* Warm-started PageRank: starts from x_inout (the previous result) instead of
 * 1/n and converges to the same fixed point.  Replaces dynamic_pagerank
 * (src/algorithm/pagerank/pagerank.cu:70-132). */
gv_status gv_pagerank_dynamic(gv_graph *g, float alpha, float epsilon, int32_t max_iter,
                              float *x_inout, int32_t *sweeps, int mem, void *stream);

/* PageRank (same definition as gv_pagerank on an undirected store) that
 * allocates nothing.  No counterpart in the reference.  For callers that
 * cannot allocate device memory when they need the result: serving threads
 * that must not stall on an allocation (cudaMalloc may synchronise the
 * device), and hosts that hand all device memory to their own arena up
 * front.  Its scratch is one fixed file-scope device array (about 16 MiB,
 * held by every GPU that loads the library until exit), so graphs are
 * limited to 1048576 vertices (larger: GV_ERR_CAPACITY).  Undirected
 * (symmetric) stores only: a directed store gives GV_ERR_STATE (gv_pagerank
 * handles those through its transposed pull, which needs scratch).  x_out is
 * a caller-owned DEVICE buffer of n floats.  All calls on a device share the
 * array, which keeps the last call's contents: calls that overlap on the GPU
 * race and must be serialised by the caller.  The first call on a device
 * looks up the array's address with that device current and keeps it for
 * the process (not valid after cudaDeviceReset); make that first call before
 * any stream capture.  Synchronous: it reads the convergence flag back every
 * 8 sweeps and the sweep count at the end. */
gv_status gv_pagerank_noalloc(gv_graph *g, float alpha, float epsilon, int32_t max_iter,
                              float *x_out, int32_t *sweeps, void *stream);

/* Personalised PageRank from `source`: x0 = e_s;
 * x <- (1-alpha) e_s + alpha * sum_{u->v} x_u / deg(u). */
gv_status gv_ppr(gv_graph *g, uint32_t source, float alpha, float epsilon, int32_t max_iter,
                 float *x_out, int32_t *sweeps, int mem, void *stream);

/* Exact triangle count on an undirected store.  per_vertex[n] (nullable)
 * gets t(u) = #triangles {u<v<w} owned by their smallest vertex u, as the
 * reference counts them (src/algorithm/tc/tc_kernel.cu:3-74) but in uint64;
 * *total = sum.  Synchronous. */
gv_status gv_tc(gv_graph *g, uint64_t *per_vertex, uint64_t *total, int mem, void *stream);

/* Incident-triangle counts for a vertex subset: out[i] = #triangles that
 * contain subset[i].  Synchronous. */
gv_status gv_tc_subset(gv_graph *g, const uint32_t *subset, uint64_t ns, uint64_t *out,
                       int mem, void *stream);

/* Betweenness centrality (Brandes): bc[v] = sum over the given sources s != v
 * of delta_s(v), no halving for undirected graphs (as src/algorithm/bc/bc.cu:42-80
 * sums).  sources == NULL or ns == 0 means every vertex.  Path counts are
 * exact uint64, dependencies accumulate in fp64, bc_out[n] is fp32. */
gv_status gv_bc(gv_graph *g, const uint32_t *sources, uint64_t ns, float *bc_out,
                int mem, void *stream);

/* gv_bc for nreq requests at once: request r takes the sources
 * sources[offsets[r] .. offsets[r+1]) (an empty range: every vertex) and
 * gets bc_out[r*n .. (r+1)*n).  Sources run in passes of 64 that may hold
 * two requests (32 sources each), so two small requests share one set of
 * BFS sweeps; each request's scores equal its own gv_bc up to the order of
 * fp64 additions.  offsets (nreq + 1 entries, offsets[0] = 0) is host
 * memory; sources and bc_out follow mem.  New entry point: the reference
 * runs one bc call per request (src/algorithm/bc/bc.cu:3-88). */
gv_status gv_bc_multi(gv_graph *g, const uint32_t *sources, const uint64_t *offsets,
                      uint32_t nreq, float *bc_out, int mem, void *stream);

/* Single-source BFS level and exact shortest-path counts (the forward half
 * of gv_bc): dist[n] int32 (-1 unreachable), sigma[n] uint64. */
gv_status gv_bfs_sigma(gv_graph *g, uint32_t source, int32_t *dist, uint64_t *sigma,
                       int mem, void *stream);

/* ---- differentiation: weighted PageRank ----------------------------------
 * P_uv = w_uv / s_u with s_u = sum_v w_uv (row-normalised stored weights).
 * forward:  x = (1-alpha)/n + alpha P^T x  (x0 = 1/n, until L1 step < tol)
 * adjoint:  lambda = c + alpha P lambda    (lambda0 = c)
 * gradient of J = sum_i c_i x_i:
 *   mode 0 (raw weights):   dJ/dw_uv = x_u (alpha lambda_v - lambda_u + c_u) / s_u
 *   mode 1 (normalised P):  dJ/dP_uv = alpha x_u lambda_v
 * grad[] is aligned with gv_export_csr's entry order.  No reference
 * counterpart: Edge::weight is commented out in the reference
 * (include/dynamicStructure/graphStructures.cuh:21). */
gv_status gv_wpr_forward(gv_graph *g, float alpha, float tol, int32_t max_iter,
                         float *x_out, int32_t *sweeps, int mem, void *stream);
gv_status gv_wpr_backward(gv_graph *g, float alpha, float tol, int32_t max_iter,
                          const float *x, const float *c, int32_t mode,
                          float *grad, uint64_t cap, float *lambda_out,
                          int32_t *sweeps, int mem, void *stream);

/* ---- misc --------------------------------------------------------------- */

/* Number of kernels this library has launched in this process. */
uint64_t gv_kernel_launches(void);

/* Per-kernel device timing with CUDA events recorded on the launching
 * stream (replaces the reference's wall-clock Profiler,
 * src/util/profiler.cu:20-40).  Slots: "radix", "segment", "member",
 * "apply", "compact", "pull", "tc_snapshot", "tc_count", "bfs_level",
 * "bc_dep".  gv_profile_query synchronises the recorded events. */
gv_status gv_profile_enable(int32_t on);
gv_status gv_profile_reset(void);
gv_status gv_profile_query(const char *name, double *total_ms, uint64_t *launches);
/* Message for the last failing call on this host thread. */
const char *gv_last_error_string(void);
/* Library version string. */
const char *gv_version(void);

#ifdef __cplusplus
}
#endif

#endif /* GV_H */
