// Lane groups: TPV consecutive lanes of a warp cooperate on one vertex
// (threads-per-vertex, picked by the autotuner from {4, 8, 16, 32}).
#pragma once
#include "common.cuh"

namespace gv {

template <int TPV>
struct Group {
    uint32_t gl;    // lane within the group
    uint32_t gw;    // group index within the warp
    uint32_t mask;  // member lanes
    __device__ __forceinline__ Group() {
        const uint32_t lane = threadIdx.x & 31u;
        gl = lane % TPV;
        gw = lane / TPV;
        mask = (TPV == 32) ? GV_FULL_MASK : (((1u << TPV) - 1u) << (gw * TPV));
    }
    __device__ __forceinline__ void sync() const { __syncwarp(mask); }
    template <typename T>
    __device__ __forceinline__ T bcast(T v, int src) const {
        return __shfl_sync(mask, v, src, TPV);
    }
    template <typename T>
    __device__ __forceinline__ T sum(T v) const {
#pragma unroll
        for (int o = TPV / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, TPV);
        return v;
    }
    __device__ __forceinline__ uint32_t any(bool p) const {
        return __ballot_sync(mask, p) & mask;
    }
    // Exclusive prefix of v over the group; *total = group sum.
    __device__ __forceinline__ uint32_t excl_scan(uint32_t v, uint32_t &total) const {
        uint32_t incl = v;
#pragma unroll
        for (int o = 1; o < TPV; o <<= 1) {
            uint32_t t = __shfl_up_sync(mask, incl, o, TPV);
            if (gl >= (uint32_t)o) incl += t;
        }
        total = __shfl_sync(mask, incl, TPV - 1, TPV);
        return incl - v;
    }
};

// Fills tab[i] = pool index of block k0+i for i < cnt (threads t of nt stride).
__device__ __forceinline__ void fill_block_table(const DevGraph &g, uint32_t root, uint32_t k0,
                                                 uint32_t cnt, uint32_t *tab, uint32_t t,
                                                 uint32_t nt) {
    for (uint32_t i = t; i < cnt; i += nt) {
        const uint32_t k = k0 + i;
        tab[i] = (k == 0) ? root : cbt_block(g.left, g.right, root, k);
    }
}

// Block-wide exclusive scan for the CTA-per-vertex paths (NT threads).
template <typename T, int NT>
__device__ __forceinline__ T cta_excl_scan(T v, T *wtot /*[33]*/, T &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(GV_FULL_MASK, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) wtot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        constexpr int NW = NT / 32;
        T w = (lane < NW) ? wtot[lane] : T(0);
        T wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T t = __shfl_up_sync(GV_FULL_MASK, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < NW) wtot[lane] = wi - w;
        if (lane == 31) wtot[32] = wi;
    }
    __syncthreads();
    T res = wtot[warp] + incl - v;
    total = wtot[32];
    __syncthreads();
    return res;
}

template <typename T, int NT>
__device__ __forceinline__ T cta_sum(T v, T *wtot /*[33]*/) {
    T tot;
    cta_excl_scan<T, NT>(v, wtot, tot);
    return tot;
}

}  // namespace gv
