// Device-wide primitives written for this library (no CUB/Thrust on the hot
// path): exclusive scan and a stable LSD radix sort of 64-bit batch keys.
// They replace the reference's thrust::exclusive_scan call sites
// (src/dynamicStructure/graphvine.cu:197, :291, :329).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gv {

// Scratch a scan of n elements needs (bytes).
size_t scan_scratch_bytes(uint64_t n);

// out[i] = sum_{j<i} in[j]; out may alias in.  If total != nullptr the grand
// total is written there (device pointer).  Launch-only (no host sync).
void scan_exclusive_u32(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *total,
                        void *scratch, cudaStream_t s);
void scan_exclusive_u32_to_u64(const uint32_t *in, unsigned long long *out, uint64_t n,
                               unsigned long long *total, void *scratch, cudaStream_t s);
void scan_exclusive_u64(const unsigned long long *in, unsigned long long *out, uint64_t n,
                        unsigned long long *total, void *scratch, cudaStream_t s);

// Stable LSD radix sort of keys[0, n) over bits [0, nbits) with optional
// uint32 values carried along.  keys/vals are sorted using alt buffers of the
// same size; the result lands in whichever buffer the returned index names
// (0 = keys/vals, 1 = keys_alt/vals_alt).  counts must hold
// radix_counts_elems(n) uint32; scratch scan_scratch_bytes(radix_counts_elems(n)).
uint64_t radix_counts_elems(uint64_t n);
int radix_sort_u64(unsigned long long *keys, unsigned long long *keys_alt, uint32_t *vals,
                   uint32_t *vals_alt, uint64_t n, int nbits, uint32_t *counts, void *scratch,
                   cudaStream_t s);

}  // namespace gv
