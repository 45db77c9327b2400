// Seeded generators (see include/gv_gen.h).  Host and device share
// gv_b200/csrc/rmat.h, so a pair depends only on (scale, seed, index).
#include "../../include/gv_gen.h"
#include "store.cuh"
#include "rmat.h"
#include "launch.hpp"

namespace gv {
namespace {

__global__ void k_rmat(uint32_t scale, uint64_t first, uint64_t count, uint64_t seed, uint32_t *src, uint32_t *dst) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x)
        gv_rmat_pair(seed, first + i, scale, &src[i], &dst[i]);
}

__global__ void k_uniform(uint32_t n, uint64_t count, uint64_t seed, uint32_t *src, uint32_t *dst) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x)
        gv_uniform_pair(n, seed, i, &src[i], &dst[i]);
}

}  // namespace
}  // namespace gv

using namespace gv;

extern "C" {

gv_status gv_gen_rmat(uint32_t scale, uint64_t first, uint64_t count, uint64_t seed, uint32_t *src, uint32_t *dst,
                      int mem, void *stream) {
    if ((count && (!src || !dst)) || scale == 0 || scale > 32) return GV_ERR_INVALID;
    if (mem == GV_MEM_DEVICE) {
        GV_LAUNCH(k_rmat, grid_for(count, 256, 148 * 16), 256, 0, (cudaStream_t)stream, scale, first, count, seed, src, dst);
        return cuda_status(cudaGetLastError(), "gen rmat");
    }
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)count; ++i) gv_rmat_pair(seed, first + (uint64_t)i, scale, &src[i], &dst[i]);
    return GV_OK;
}

gv_status gv_gen_uniform(uint32_t n, uint64_t count, uint64_t seed, uint32_t *src, uint32_t *dst, int mem, void *stream) {
    if ((count && (!src || !dst)) || n < 2) return GV_ERR_INVALID;
    if (mem == GV_MEM_DEVICE) {
        GV_LAUNCH(k_uniform, grid_for(count, 256, 148 * 16), 256, 0, (cudaStream_t)stream, n, count, seed, src, dst);
        return cuda_status(cudaGetLastError(), "gen uniform");
    }
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)count; ++i) gv_uniform_pair(n, seed, (uint64_t)i, &src[i], &dst[i]);
    return GV_OK;
}

}  // extern "C"
