// Exclusive scan (reduce-then-scan) and stable LSD radix sort, hand-written
// for sm_100a.  The radix sort ranks each 4096-key tile with warp match_any
// multi-split in shared memory and stages the tile in digit order so that the
// global scatter writes contiguous runs.
#include "prims.cuh"
#include "common.cuh"
#include "launch.hpp"

namespace gv {

std::atomic<unsigned long long> g_launches{0};

namespace {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
constexpr int SCAN_TOP_THREADS = 1024;
constexpr int SCAN_TOP_ITEMS = 4;

// Block-wide exclusive scan of one value per thread; returns the exclusive
// prefix and writes the block total to *total_out (all threads see it).
template <typename T, int NT>
__device__ __forceinline__ T block_exclusive_scan(T v, T *warp_tot, T &total_out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(GV_FULL_MASK, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        constexpr int NW = NT / 32;
        T w = (lane < NW) ? warp_tot[lane] : T(0);
        T wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T t = __shfl_up_sync(GV_FULL_MASK, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < NW) warp_tot[lane] = wi - w;  // exclusive warp offsets
        if (lane == 31) warp_tot[32] = wi;       // block total
    }
    __syncthreads();
    T res = warp_tot[warp] + incl - v;
    total_out = warp_tot[32];
    __syncthreads();
    return res;
}

template <typename Tin, typename Tout>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(const Tin *__restrict__ in, uint64_t n,
                                                              Tout *__restrict__ tile_sums) {
    __shared__ Tout wt[33];
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE;
    Tout s = 0;
#pragma unroll
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        uint64_t i = base + (uint64_t)j * SCAN_THREADS + threadIdx.x;
        if (i < n) s += (Tout)in[i];
    }
    Tout tot;
    block_exclusive_scan<Tout, SCAN_THREADS>(s, wt, tot);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

template <typename Tout>
__global__ void __launch_bounds__(SCAN_TOP_THREADS) k_scan_top(Tout *__restrict__ sums, uint64_t ntiles,
                                                               Tout *__restrict__ total) {
    __shared__ Tout wt[33];
    Tout carry = 0;
    for (uint64_t cb = 0; cb < ntiles; cb += (uint64_t)SCAN_TOP_THREADS * SCAN_TOP_ITEMS) {
        Tout v[SCAN_TOP_ITEMS];
        Tout ts = 0;
#pragma unroll
        for (int j = 0; j < SCAN_TOP_ITEMS; ++j) {
            uint64_t i = cb + (uint64_t)threadIdx.x * SCAN_TOP_ITEMS + j;
            v[j] = (i < ntiles) ? sums[i] : Tout(0);
            ts += v[j];
        }
        Tout tot;
        Tout ex = block_exclusive_scan<Tout, SCAN_TOP_THREADS>(ts, wt, tot);
        Tout run = carry + ex;
#pragma unroll
        for (int j = 0; j < SCAN_TOP_ITEMS; ++j) {
            uint64_t i = cb + (uint64_t)threadIdx.x * SCAN_TOP_ITEMS + j;
            if (i < ntiles) sums[i] = run;
            run += v[j];
        }
        carry += tot;
    }
    if (total && threadIdx.x == 0) *total = carry;
}

template <typename Tin, typename Tout>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_down(const Tin *in, Tout *out, uint64_t n,
                                                            const Tout *__restrict__ tile_off) {
    __shared__ Tout buf[SCAN_TILE];
    __shared__ Tout wt[33];
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE;
#pragma unroll
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        uint64_t i = base + (uint64_t)j * SCAN_THREADS + threadIdx.x;
        buf[j * SCAN_THREADS + threadIdx.x] = (i < n) ? (Tout)in[i] : Tout(0);
    }
    __syncthreads();
    Tout v[SCAN_ITEMS];
    Tout ts = 0;
#pragma unroll
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        v[j] = buf[threadIdx.x * SCAN_ITEMS + j];
        ts += v[j];
    }
    Tout tot;
    Tout run = block_exclusive_scan<Tout, SCAN_THREADS>(ts, wt, tot) + tile_off[blockIdx.x];
#pragma unroll
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        buf[threadIdx.x * SCAN_ITEMS + j] = run;
        run += v[j];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        uint64_t i = base + (uint64_t)j * SCAN_THREADS + threadIdx.x;
        if (i < n) out[i] = buf[j * SCAN_THREADS + threadIdx.x];
    }
}

template <typename Tin, typename Tout>
void scan_exclusive_impl(const Tin *in, Tout *out, uint64_t n, Tout *total, void *scratch,
                         cudaStream_t s) {
    if (n == 0) {
        if (total) cudaMemsetAsync(total, 0, sizeof(Tout), s);
        return;
    }
    uint64_t ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    Tout *sums = static_cast<Tout *>(scratch);
    GV_LAUNCH((k_scan_reduce<Tin, Tout>), (unsigned)ntiles, SCAN_THREADS, 0, s, in, n, sums);
    GV_LAUNCH((k_scan_top<Tout>), 1, SCAN_TOP_THREADS, 0, s, sums, ntiles, total);
    GV_LAUNCH((k_scan_down<Tin, Tout>), (unsigned)ntiles, SCAN_THREADS, 0, s, in, out, n,
              (const Tout *)sums);
}

// ---------------------------------------------------------------- radix sort
constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;  // 4096 keys
constexpr int RS_RADIX = 256;

__global__ void __launch_bounds__(RS_THREADS) k_rs_upsweep(const unsigned long long *__restrict__ keys,
                                                           uint64_t n, int shift,
                                                           uint32_t *__restrict__ counts,
                                                           uint32_t ntiles) {
    __shared__ uint32_t hist[RS_RADIX];
    hist[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * RS_TILE;
#pragma unroll 4
    for (int j = 0; j < RS_ITEMS; ++j) {
        uint64_t i = base + (uint64_t)j * RS_THREADS + threadIdx.x;
        if (i < n) atomicAdd(&hist[(uint32_t)(keys[i] >> shift) & 0xFFu], 1u);
    }
    __syncthreads();
    counts[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = hist[threadIdx.x];
}

struct RsSmem {
    unsigned long long keys[RS_TILE];
    uint32_t vals[RS_TILE];
    uint32_t wcount[RS_WARPS][RS_RADIX];
    uint32_t run[RS_RADIX];
    uint32_t tstart[RS_RADIX];
    uint32_t gstart[RS_RADIX];
    uint32_t wt[33];
};

template <bool VALS>
__global__ void __launch_bounds__(RS_THREADS) k_rs_downsweep(const unsigned long long *__restrict__ kin,
                                                             unsigned long long *__restrict__ kout,
                                                             const uint32_t *__restrict__ vin,
                                                             uint32_t *__restrict__ vout, uint64_t n,
                                                             int shift,
                                                             const uint32_t *__restrict__ offsets,
                                                             uint32_t ntiles) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    RsSmem &S = *reinterpret_cast<RsSmem *>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t base = (uint64_t)blockIdx.x * RS_TILE;
    const uint64_t rem = n - base;
    const uint32_t tile_n = rem < (uint64_t)RS_TILE ? (uint32_t)rem : (uint32_t)RS_TILE;

    unsigned long long k[RS_ITEMS];
    uint32_t v[RS_ITEMS];
    uint32_t rank[RS_ITEMS];
#pragma unroll
    for (int j = 0; j < RS_ITEMS; ++j) {
        uint32_t li = (uint32_t)j * RS_THREADS + tid;
        k[j] = (li < tile_n) ? kin[base + li] : 0ull;
        if (VALS) v[j] = (li < tile_n) ? vin[base + li] : 0u;
    }
    S.run[tid] = 0;
#pragma unroll
    for (int w = 0; w < RS_WARPS; ++w) S.wcount[w][tid] = 0;
    __syncthreads();

    const uint32_t lt_mask = (1u << lane) - 1u;
#pragma unroll
    for (int j = 0; j < RS_ITEMS; ++j) {
        uint32_t li = (uint32_t)j * RS_THREADS + tid;
        bool valid = li < tile_n;
        uint32_t d = valid ? ((uint32_t)(k[j] >> shift) & 0xFFu) : 0x100u;
        uint32_t peers = __match_any_sync(GV_FULL_MASK, d);
        uint32_t r = __popc(peers & lt_mask);
        if (valid && r == 0) S.wcount[warp][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            uint32_t acc = S.run[d] + r;
            for (int w = 0; w < warp; ++w) acc += S.wcount[w][d];
            rank[j] = acc;
        }
        __syncthreads();
        {
            uint32_t sum = 0;
#pragma unroll
            for (int w = 0; w < RS_WARPS; ++w) {
                sum += S.wcount[w][tid];
                S.wcount[w][tid] = 0;
            }
            S.run[tid] += sum;
        }
        __syncthreads();
    }
    // Tile-local digit starts and global digit starts for this tile.
    uint32_t tot;
    uint32_t ex = block_exclusive_scan<uint32_t, RS_THREADS>(S.run[tid], S.wt, tot);
    S.tstart[tid] = ex;
    S.gstart[tid] = offsets[(uint64_t)tid * ntiles + blockIdx.x];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < RS_ITEMS; ++j) {
        uint32_t li = (uint32_t)j * RS_THREADS + tid;
        if (li < tile_n) {
            uint32_t d = (uint32_t)(k[j] >> shift) & 0xFFu;
            uint32_t pos = S.tstart[d] + rank[j];
            S.keys[pos] = k[j];
            if (VALS) S.vals[pos] = v[j];
        }
    }
    __syncthreads();
    for (uint32_t i = tid; i < tile_n; i += RS_THREADS) {
        unsigned long long key = S.keys[i];
        uint32_t d = (uint32_t)(key >> shift) & 0xFFu;
        uint64_t pos = (uint64_t)S.gstart[d] + (i - S.tstart[d]);
        kout[pos] = key;
        if (VALS) vout[pos] = S.vals[i];
    }
}

}  // namespace

size_t scan_scratch_bytes(uint64_t n) {
    uint64_t ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    return (size_t)(ntiles + 1) * sizeof(unsigned long long);
}

void scan_exclusive_u32(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *total,
                        void *scratch, cudaStream_t s) {
    scan_exclusive_impl<uint32_t, uint32_t>(in, out, n, total, scratch, s);
}

void scan_exclusive_u32_to_u64(const uint32_t *in, unsigned long long *out, uint64_t n,
                               unsigned long long *total, void *scratch, cudaStream_t s) {
    scan_exclusive_impl<uint32_t, unsigned long long>(in, out, n, total, scratch, s);
}

void scan_exclusive_u64(const unsigned long long *in, unsigned long long *out, uint64_t n,
                        unsigned long long *total, void *scratch, cudaStream_t s) {
    scan_exclusive_impl<unsigned long long, unsigned long long>(in, out, n, total, scratch, s);
}

uint64_t radix_counts_elems(uint64_t n) {
    uint64_t ntiles = (n + RS_TILE - 1) / RS_TILE;
    return ntiles * RS_RADIX;
}

int radix_sort_u64(unsigned long long *keys, unsigned long long *keys_alt, uint32_t *vals,
                   uint32_t *vals_alt, uint64_t n, int nbits, uint32_t *counts, void *scratch,
                   cudaStream_t s) {
    if (n <= 1 || nbits <= 0) return 0;
    static bool attr_set = false;
    const size_t smem = sizeof(RsSmem);
    if (!attr_set) {
        cudaFuncSetAttribute(k_rs_downsweep<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        cudaFuncSetAttribute(k_rs_downsweep<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        attr_set = true;
    }
    const uint32_t ntiles = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
    const uint64_t ncounts = (uint64_t)ntiles * RS_RADIX;
    unsigned long long *kin = keys, *kout = keys_alt;
    uint32_t *vin = vals, *vout = vals_alt;
    int cur = 0;
    for (int shift = 0; shift < nbits; shift += 8) {
        GV_LAUNCH(k_rs_upsweep, ntiles, RS_THREADS, 0, s, kin, n, shift, counts, ntiles);
        scan_exclusive_u32(counts, counts, ncounts, nullptr, scratch, s);
        if (vals)
            GV_LAUNCH(k_rs_downsweep<true>, ntiles, RS_THREADS, smem, s, kin, kout, vin, vout, n,
                      shift, counts, ntiles);
        else
            GV_LAUNCH(k_rs_downsweep<false>, ntiles, RS_THREADS, smem, s, kin, kout, nullptr,
                      nullptr, n, shift, counts, ntiles);
        std::swap(kin, kout);
        std::swap(vin, vout);
        cur ^= 1;
    }
    return cur;
}

}  // namespace gv
