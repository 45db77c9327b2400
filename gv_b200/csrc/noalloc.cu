// PageRank that allocates nothing: gv_pagerank_noalloc.
//
// Some callers cannot call cudaMalloc at the moment they need a result:
// serving threads on a latency budget (a device allocation may synchronise
// the device and stall the other streams' work), and hosts that hand all
// device memory to their own arena up front, so that a later cudaMalloc
// fails or takes memory the arena counts on.  This entry point serves them:
// its scratch is a file-scope __device__ array of fixed size, so the call
// itself never allocates; the caller passes the graph and a device output
// buffer.
//
// Limits and rules:
//   * undirected (symmetric) stores only (a directed store -> GV_ERR_STATE);
//   * graphs of at most GV_NOALLOC_MAX_VERTICES vertices (larger -> GV_ERR_CAPACITY);
//   * every GPU that loads libgv holds the array (about 16 MiB) until exit;
//   * all calls on a device share the one array, which keeps the last call's
//     contents: calls that overlap on the GPU (different streams, or
//     different graphs at the same time) race and must be serialised by the
//     caller;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current and keeps it for the
//     life of the process; make that first call before any stream capture.
//     The kept address does not survive cudaDeviceReset: a process that
//     resets the device must not call this entry point afterwards.
//   * the call synchronises on `stream`: every 8 sweeps it reads the
//     convergence flag back to the host.
#include <mutex>
#include "store.cuh"
#include "group.cuh"
#include "launch.hpp"

#define GV_NOALLOC_MAX_VERTICES (1u << 20)

namespace gv {
namespace {

constexpr unsigned NA_GRID = 148 * 4;
constexpr int NA_THREADS = 256;
constexpr size_t NA_VEC = (size_t)GV_NOALLOC_MAX_VERTICES * sizeof(float);
// layout: x0 | x1 | c0 | c1 | partial[NA_GRID] (fp64) | state[4] (int) | residual (fp64)
constexpr size_t NA_PARTIAL = 4 * NA_VEC;
constexpr size_t NA_STATE = NA_PARTIAL + NA_GRID * sizeof(double);
constexpr size_t NA_RES = NA_STATE + 4 * sizeof(int);
constexpr size_t NA_BYTES = NA_RES + sizeof(double);

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

constexpr int NA_MAX_DEVICES = 64;
std::mutex na_mu;
void *na_ptr[NA_MAX_DEVICES] = {nullptr};

__global__ void k_na_init(DevGraph g, float *__restrict__ x0, float *__restrict__ c0) {
    const float x = 1.0f / (float)g.n;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < g.n; v += gridDim.x * blockDim.x) {
        x0[v] = x;
        const uint32_t d = g.vtx[v].z;
        c0[v] = d ? x / (float)d : 0.f;
    }
}

// One lane group per vertex for every degree: block tables of 64 blocks are
// walked chunk by chunk, so the kernel needs no work lists.
template <int TPV>
__global__ void __launch_bounds__(NA_THREADS) k_na_pull(DevGraph g, const float *__restrict__ gather,
                                                        const float *__restrict__ xold, float *__restrict__ xnew,
                                                        float *__restrict__ cnew, float alpha, float base,
                                                        double *__restrict__ partial, const int *__restrict__ state) {
    constexpr int GPC = NA_THREADS / TPV;
    __shared__ uint32_t tabs[GPC][BIG_BLOCKS];
    __shared__ double red[NA_THREADS / 32];
    if (state[0]) return;
    Group<TPV> G;
    uint32_t *tab = tabs[threadIdx.x / TPV];
    double res = 0.0;
    for (uint32_t v = blockIdx.x * GPC + threadIdx.x / TPV; v < g.n; v += gridDim.x * GPC) {
        const uint4 rec = g.vtx[v];
        const uint32_t fill = rec.y, nb = blocks_for(fill, g.logB);
        float sum = 0.f;
        for (uint32_t k0 = 0; k0 < nb; k0 += BIG_BLOCKS) {
            const uint32_t kc = min((uint32_t)BIG_BLOCKS, nb - k0);
            fill_block_table(g, rec.x, k0, kc, tab, G.gl, TPV);
            G.sync();
            const uint32_t e0 = k0 << g.logB, e1 = min(fill, (k0 + kc) << g.logB);
            for (uint32_t e = e0 + G.gl * 4; e < e1; e += TPV * 4) {
                const size_t at = ((size_t)tab[(e >> g.logB) - k0] << g.logB) + (e & (g.B - 1));
                const uint4 q = *reinterpret_cast<const uint4 *>(g.pool + at);
                const uint32_t ev[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (e + j < e1 && ev[j] != GV_TOMB) sum += __ldg(gather + ev[j]);
            }
            G.sync();
        }
        sum = G.sum(sum);
        if (G.gl == 0) {
            const float xv = base + alpha * sum;
            xnew[v] = xv;
            cnew[v] = rec.z ? xv / (float)rec.z : 0.f;
            res += (double)fabsf(xv - xold[v]);
        }
    }
    res = warp_sum(res);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = res;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < NA_THREADS / 32; ++i) t += red[i];
        partial[blockIdx.x] = t;
    }
}

__global__ void k_na_done(const double *__restrict__ partial, float eps, int *state, double *res) {
    __shared__ double red[32];
    if (state[0]) return;
    double t = 0.0;
    for (uint32_t i = threadIdx.x; i < NA_GRID; i += blockDim.x) t += partial[i];
    t = warp_sum(t);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < (int)(blockDim.x / 32); ++i) s += red[i];
        *res = s;
        state[1] += 1;
        if (s < (double)eps) state[0] = 1;
    }
}

// Device address of the scratch array on `dev` (looked up once per device,
// with that device current).
gv_status na_scratch(int dev, char **out) {
    if (dev < 0 || dev >= NA_MAX_DEVICES) { set_error("device ordinal beyond the no-alloc table"); return GV_ERR_INVALID; }
    std::lock_guard<std::mutex> lk(na_mu);
    if (!na_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(no-alloc scratch)");
        na_ptr[dev] = p;
    }
    *out = static_cast<char *>(na_ptr[dev]);
    return GV_OK;
}

}  // namespace
}  // namespace gv

using namespace gv;

extern "C" gv_status gv_pagerank_noalloc(gv_graph *g, float alpha, float epsilon, int32_t max_iter, float *x_out,
                                         int32_t *sweeps, void *stream) {
    if (!g || !x_out || max_iter < 0) { set_error("null argument"); return GV_ERR_INVALID; }
    const uint32_t n = g->d.n;
    if (n > GV_NOALLOC_MAX_VERTICES) {
        set_error("gv_pagerank_noalloc handles at most 1048576 vertices");
        return GV_ERR_CAPACITY;
    }
    if (g->cfg.directed) { set_error("PageRank pull needs an undirected (symmetric) store"); return GV_ERR_STATE; }
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != g->cfg.device) cudaSetDevice(g->cfg.device);
    char *base = nullptr;
    gv_status st = na_scratch(g->cfg.device, &base);
    if (st != GV_OK) {
        if (prev >= 0 && prev != g->cfg.device) cudaSetDevice(prev);
        return st;
    }
    cudaStream_t s = (cudaStream_t)stream;
    float *x[2] = {reinterpret_cast<float *>(base), reinterpret_cast<float *>(base + NA_VEC)};
    float *c[2] = {reinterpret_cast<float *>(base + 2 * NA_VEC), reinterpret_cast<float *>(base + 3 * NA_VEC)};
    double *partial = reinterpret_cast<double *>(base + NA_PARTIAL);
    int *state = reinterpret_cast<int *>(base + NA_STATE);
    double *res = reinterpret_cast<double *>(base + NA_RES);
    DevGraph d = g->d;
    // the array keeps the previous call's contents: clear what must start at zero
    cudaError_t e = cudaMemsetAsync(state, 0, 4 * sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(partial, 0, NA_GRID * sizeof(double), s);
    if (e == cudaSuccess) GV_LAUNCH(k_na_init, grid_for(n, 256), 256, 0, s, d, x[0], c[0]);
    const float b = (1.0f - alpha) / (float)n;
    int h_state[2] = {0, 0};
    int launched = 0, cur = 0;
    while (e == cudaSuccess && launched < max_iter) {
        const int chunk = max_iter - launched < 8 ? max_iter - launched : 8;
        for (int i = 0; i < chunk; ++i) {
            dispatch_tpv(g->cfg.threads_per_vertex, [&](auto t) {
                constexpr int T = decltype(t)::value;
                GV_LAUNCH((k_na_pull<T>), NA_GRID, NA_THREADS, 0, s, d, (const float *)c[cur], (const float *)x[cur],
                          x[cur ^ 1], c[cur ^ 1], alpha, b, partial, (const int *)state);
            });
            GV_LAUNCH(k_na_done, 1, 256, 0, s, (const double *)partial, epsilon, state, res);
            cur ^= 1;
        }
        launched += chunk;
        e = cudaMemcpyAsync(h_state, state, sizeof(h_state), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e == cudaSuccess && h_state[0]) break;
    }
    if (e == cudaSuccess) {
        // sweep i (1-based) wrote x[1] when i is odd
        e = cudaMemcpyAsync(x_out, x[h_state[1] & 1], (size_t)n * sizeof(float), cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (sweeps) *sweeps = h_state[1];
    if (prev >= 0 && prev != g->cfg.device) cudaSetDevice(prev);
    return cuda_status(e, "gv_pagerank_noalloc");
}
