/*
 * gv_gen.h — seeded synthetic workload generators exported by libgv.
 *
 * The reference reads Matrix-Market files (src/reader/marketReader.cu:3-121)
 * and draws update batches with srand/rand (src/dynamicStructure/csr.cu:80-125);
 * no dataset ships with it.  These generators stand in for both: R-MAT with
 * a/b/c/d = 0.57/0.19/0.19/0.05, counter-based so host and device produce the
 * same pairs for the same seed.
 */
#ifndef GV_GEN_H
#define GV_GEN_H
#include "gv.h"
#ifdef __cplusplus
extern "C" {
#endif

/* Pairs i in [first, first+count) of the R-MAT stream (scale, seed). */
gv_status gv_gen_rmat(uint32_t scale, uint64_t first, uint64_t count, uint64_t seed,
                      uint32_t *src, uint32_t *dst, int mem, void *stream);

/* count uniform pairs u != v over [0, n) (stream seed). */
gv_status gv_gen_uniform(uint32_t n, uint64_t count, uint64_t seed, uint32_t *src, uint32_t *dst,
                         int mem, void *stream);

#ifdef __cplusplus
}
#endif
#endif
