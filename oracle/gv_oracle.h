/*
 * gv_oracle — CPU restatement of GraphVine's dynamic-graph hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load this library, and only
 * as the checker or the timed CPU baseline; the product (libgv) never calls
 * it and has no CPU fallback.
 *
 * It restates the reference's intended semantics in exact integers and
 * fp64.  Parity pin: the reference ships no tests, golden vectors or
 * fixtures (it has no test directory at all), so this oracle is pinned
 * against (a) networkx / scipy on small graphs (tests/test_oracle.py,
 * tests/golden/make_golden.py) and (b) the reference's own CUDA code, built
 * from its sources by oracle/ref_build.sh and run on a B200 in the regimes
 * where the reference is well defined (tests/test_ref_pin.py).
 */
#ifndef GV_ORACLE_H
#define GV_ORACLE_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_graph or_graph;

or_graph *or_create(uint32_t n, int directed, int weighted);
void or_destroy(or_graph *g);
int or_set_threads(int nthreads);

/* Set-union insert of k pairs (both directions unless directed); self-loops
 * dropped; first occurrence wins (its weight is kept); existing entries keep
 * their weight.  Returns 0, or -1 on an out-of-range id (graph unchanged). */
int or_insert(or_graph *g, const uint32_t *src, const uint32_t *dst, const float *w, uint64_t k);
/* Same as or_insert but never symmetrises (bulk build from directed entries). */
int or_insert_directed(or_graph *g, const uint32_t *src, const uint32_t *dst, const float *w, uint64_t k);
/* Set-difference delete of k pairs (both directions unless directed). */
int or_delete(or_graph *g, const uint32_t *src, const uint32_t *dst, uint64_t k);

uint64_t or_num_edges(const or_graph *g);
/* offsets[n+1]; dst[] sorted per vertex; w[] aligned (nullable). */
void or_export(const or_graph *g, uint64_t *offsets, uint32_t *dst, float *w);

/* PageRank as src/algorithm/pagerank/pagerank.cu:3-68 computes it, in fp64.
 * x0 = x_init (nullable -> 1/n).  fixed_sweeps > 0 runs exactly that many
 * sweeps and ignores epsilon.  Returns sweeps performed. */
int or_pagerank(const or_graph *g, double alpha, double epsilon, int max_iter, const double *x_init,
                int fixed_sweeps, double *x_out);
/* Personalised PageRank from source (x0 = e_s, teleport to s). */
int or_ppr(const or_graph *g, uint32_t source, double alpha, double epsilon, int max_iter,
           int fixed_sweeps, double *x_out);

/* Triangles owned by their smallest vertex, the reference's formula
 * (src/algorithm/tc/tc_kernel.cu:3-74): t(u) = #{(v, w): v in N(u), v > u,
 * w in N(v), w > v, u in N(w)}.  Returns the total. */
uint64_t or_tc(const or_graph *g, uint64_t *per_vertex);
/* Incident-triangle counts of a subset (symmetric graphs). */
void or_tc_incident(const or_graph *g, const uint32_t *subset, uint64_t ns, uint64_t *out);

/* Brandes betweenness, exact uint64 path counts, fp64 dependencies, summed
 * over the sources without halving (src/algorithm/bc/bc.cu:42-80, with the
 * defects of src/algorithm/bc/bc_kernel.cu:19-119 corrected). */
void or_bc(const or_graph *g, const uint32_t *sources, uint64_t ns, double *bc);
void or_bfs_sigma(const or_graph *g, uint32_t source, int32_t *dist, uint64_t *sigma);

/* Weighted PageRank (row-normalised weights) and its adjoint. */
int or_wpr_forward(const or_graph *g, double alpha, double tol, int max_iter, double *x);
int or_wpr_adjoint(const or_graph *g, double alpha, double tol, int max_iter, const double *c, double *lambda);
/* Gradient per entry in or_export order.  mode 0: raw weights, 1: normalised. */
void or_wpr_gradient(const or_graph *g, double alpha, const double *x, const double *lambda,
                     const double *c, int mode, double *grad);
/* J = sum c_i x_i after replacing the raw weight of entry (u, v) by w_uv + delta. */
double or_wpr_objective(const or_graph *g, double alpha, double tol, int max_iter, const double *c,
                        uint32_t u, uint32_t v, double delta);

/* Central finite differences (J(w + h) - J(w - h)) / 2h of J = sum c_i x_i
 * with respect to the raw weights of the k entries (eu[i], ev[i]), in fp64.
 * Each perturbed objective is evaluated exactly through the rank-one form of
 * the perturbed fixed point (one forward-direction solve per entry, shared
 * by +h and -h, all k solves sharing each sweep), so no perturbed solve is
 * cut short and no two nearly equal objectives are subtracted.  tol bounds
 * the unperturbed solve's L1 step.  Returns the unperturbed sweeps. */
int or_wpr_fd(const or_graph *g, double alpha, double tol, int max_iter, const double *c, const uint32_t *eu,
              const uint32_t *ev, uint32_t k, double h, double *fd);

/* Seeded R-MAT pairs, the same generator libgv uses (gv_b200/csrc/rmat.h). */
void or_rmat_pairs(uint32_t scale, uint64_t num_pairs, uint64_t seed, uint32_t *src, uint32_t *dst);
/* Seeded uniform pairs u != v over [0, n), the same generator libgv uses
 * (gv_uniform_pair in gv_b200/csrc/rmat.h). */
void or_uniform_pairs(uint32_t n, uint64_t num_pairs, uint64_t seed, uint32_t *src, uint32_t *dst);

#ifdef __cplusplus
}
#endif
#endif
