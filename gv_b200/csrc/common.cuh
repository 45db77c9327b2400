// Device-side layout of the edge-block CBT store and the helpers every kernel
// shares.  Layout decisions (all B200-first; the reference equivalents are in
// include/dynamicStructure/graphStructures.cuh:19-120):
//   * a vertex record is one 16-byte uint4 {root, fill, live, last}, so a
//     traversal reads a vertex with a single vector load (the reference keeps
//     six 8-byte arrays plus pointers);
//   * edge blocks live in one pool of `P * B` uint32 entries; entries are
//     0-based destination ids, TOMB marks a deleted entry; slots past a
//     vertex's fill are never read (no "0 = end" convention, no reliance on
//     zeroed memory);
//   * block headers are SoA uint32 pool indices: left/right child, level-order
//     predecessor, used-slot count and owning vertex;
//   * block k of a vertex (level order) is found from the root by the binary
//     digits of k+1 (left = 0, right = 1), replacing the reference's decimal
//     path table bit_string_lookup[4096] (src/util/device_functions.cu:3,
//     :86-100, :153-169) and its 4096-block cap.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define GV_NIL 0xFFFFFFFFu
#define GV_TOMB 0xFFFFFFFFu
#define GV_FULL_MASK 0xFFFFFFFFu

// Latched device status bits (ctl->status); mapped to gv_status on the host.
#define GV_DEV_ERR_RANGE 0x1u   // vertex id >= n in a batch
#define GV_DEV_ERR_NOMEM 0x2u   // pool exhausted; batch rejected
#define GV_DEV_ERR_TIMEOUT 0x4u // a bounded spin-wait expired
#define GV_DEV_ERR_CAP 0x8u     // scratch capacity exceeded

namespace gv {

// Device control block: one per graph, in device memory.
struct Ctl {
    unsigned long long free_top;     // free_stack[0, free_top) holds free block ids
    unsigned long long need_blocks;  // blocks the pending batch needs
    unsigned long long alloc_cursor; // blocks handed out while applying a batch
    unsigned long long nuniq;        // unique entries in the pending batch
    unsigned long long nseg;         // touched vertices (segments) in the pending batch
    unsigned long long nbig;         // segments routed to the CTA-per-vertex path
    unsigned long long ndirty;       // vertices holding tombstones
    unsigned long long live_edges;   // stored live entries
    unsigned long long scratch0;     // per-algorithm scalars
    unsigned long long scratch1;
    unsigned int status;             // sticky GV_DEV_ERR_* bits
    unsigned int batch_abort;        // pending batch rejected (range error or pool exhausted)
    double acc[4];                   // per-iteration reductions (PageRank residual)
};

// Kernel-side view of a graph (passed by value).
struct DevGraph {
    uint32_t n;
    uint32_t B;        // entries per block (power of two)
    uint32_t logB;
    uint32_t weighted;
    uint64_t P;        // pool capacity in blocks
    uint4 *vtx;        // {root, fill, live, last} per vertex
    uint32_t *left;    // CBT child links (pool indices, GV_NIL if absent)
    uint32_t *right;
    uint32_t *pred;    // level-order predecessor (block k-1 of the same vertex)
    uint32_t *bcount;  // used slots in the block
    uint32_t *owner;   // owning vertex
    uint32_t *pool;    // P*B entries
    float *wpool;      // P*B weights (weighted stores only)
    uint32_t *free_stack;
    uint8_t *affected; // n flags
    uint8_t *dirty;    // n flags: vertex has tombstones
    uint32_t *dirty_list;
    uint32_t *vbig_list; // n entries: hub vertices routed to the CTA path by compaction
    Ctl *ctl;
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// Pool index of level-order block k of the tree rooted at `root`.
__device__ __forceinline__ uint32_t cbt_block(const uint32_t *__restrict__ left,
                                              const uint32_t *__restrict__ right,
                                              uint32_t root, uint32_t k) {
    uint32_t p = k + 1u;
    int d = 31 - __clz(p);
    uint32_t b = root;
    for (int i = d - 1; i >= 0; --i) b = ((p >> i) & 1u) ? right[b] : left[b];
    return b;
}

__device__ __forceinline__ uint32_t blocks_for(uint32_t fill, uint32_t logB) {
    return (fill + (1u << logB) - 1u) >> logB;
}

// Full-warp exclusive prefix of v, with one atomicAdd per warp on *ctr.
// All 32 lanes must call it.  Returns this lane's base.
__device__ __forceinline__ unsigned long long warp_agg_alloc(unsigned long long *ctr, uint32_t v) {
    const uint32_t lane = lane_id();
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(GV_FULL_MASK, incl, o);
        if (lane >= (uint32_t)o) incl += t;
    }
    uint32_t total = __shfl_sync(GV_FULL_MASK, incl, 31);
    unsigned long long base = 0;
    if (lane == 31 && total) base = atomicAdd(ctr, (unsigned long long)total);
    base = __shfl_sync(GV_FULL_MASK, base, 31);
    return base + (incl - v);
}

// Full-warp sum.
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(GV_FULL_MASK, v, o);
    return v;
}

// Lower bound of x in sorted a[0, len).
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t *a, uint32_t len, uint32_t x) {
    uint32_t lo = 0, hi = len;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

}  // namespace gv
