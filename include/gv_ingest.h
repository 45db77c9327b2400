/*
 * gv_ingest.h — Matrix-Market ingest on the device and graph snapshots.
 *
 * gv_mtx_parse replaces the reference's host reader readFile
 * (src/reader/marketReader.cu:3-121) and CSR::readGraph
 * (src/dynamicStructure/csr.cu:55-78).  gv_snapshot_save / gv_snapshot_load
 * have no reference counterpart (the reference cannot save a store); they
 * write and read a checksummed CSR of the store.
 */
#ifndef GV_INGEST_H
#define GV_INGEST_H
#include "gv.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct gv_mtx_info {
    uint64_t rows, cols, entries; /* the size line */
    uint32_t pattern;             /* banner field "pattern": no values */
    uint32_t symmetric;           /* banner symmetry "symmetric" / "hermitian" */
} gv_mtx_info;

/* Parses Matrix-Market coordinate text (len bytes; host or device memory
 * as `mem` says) on the device: the first line not starting with '%' is
 * "rows cols entries"; every later line "src dst [value]" (1-based) becomes
 * src[i] = src - 1, dst[i] = dst - 1 and, when values != NULL, values[i]
 * (1 for pattern files); blank and '%' lines are skipped.  With src == NULL
 * only *info is filled (and *count = 0).  Entries beyond `cap` return
 * GV_ERR_CAPACITY with *count set; an id outside [1, rows] x [1, cols]
 * returns GV_ERR_INVALID.  Outputs live in the same memory kind as the
 * text.  Synchronous; allocates device scratch. */
gv_status gv_mtx_parse(const char *text, uint64_t len, int mem, gv_mtx_info *info, uint32_t *src, uint32_t *dst,
                       float *values, uint64_t cap, uint64_t *count, void *stream);

/* Reads a Matrix-Market file and builds a graph of `rows` vertices from it
 * (base: configuration template, or NULL for defaults).  An undirected
 * store keeps every entry in both directions, as the reference's reader
 * symmetrises for !DIRECTED; a weighted store takes the file's values. */
gv_status gv_graph_from_mtx(const char *path, const gv_config *base, gv_graph **out);

/* Writes g (vertex count, flags, block size, CSR of the stored entries and
 * their weights) with an FNV-1a checksum of the payload. */
gv_status gv_snapshot_save(gv_graph *g, const char *path);

/* Reads a snapshot, checks it (magic, version, checksum, ids) and builds a
 * new graph with the same entries (base: configuration template for pool
 * and batch sizes, or NULL for the saved block size and defaults). */
gv_status gv_snapshot_load(const char *path, const gv_config *base, gv_graph **out);

#ifdef __cplusplus
}
#endif
#endif
