/*
 * graphvine.hpp — header-only C++ shim that keeps the reference's host API
 * (sajidanis/GV) compiling on top of libgv's C ABI (gv.h).
 *
 * Reference interfaces kept, with their signatures and semantics:
 *   extern size_t BATCH_SIZE   include/dynamicStructure/constants.cuh:19 —
 *                        defined by the application (src/main.cu:18)
 *   struct GraphProperties include/dynamicStructure/graphStructures.cuh:8-17
 *   class CSR            include/dynamicStructure/csr.cuh:14-47 — host batch
 *                        container with 1-based destinations; readGraph
 *                        (csr.cu:6-17 + src/reader/marketReader.cu:3-121, both
 *                        directions of every line), computeGraphProperties,
 *                        initializeCSR, generate_random_batch (the same
 *                        srand/rand draw sequence as csr.cu:80-125), the
 *                        get_* accessors and the static h_graph_prop
 *   class GraphVine      include/dynamicStructure/graphvine.cuh:29-58 —
 *                        GraphVine(CSR*) builds the store from the CSR
 *                        (graphvine.cu:5-35); batchInsert / batchDelete /
 *                        compaction are synchronous like the reference
 *                        (graphvine.cu:367, :446, :461); the device accessors
 *                        return device arrays (see below)
 *   static_pagerank      include/algorithm/pagerank/pagerank.cuh:11 — result in v1
 *   dynamic_pagerank     include/algorithm/pagerank/pagerank.cuh:13 — warm start from v1
 *   static_tc, dynamic_tc include/algorithm/tc/tc.cuh:10-12 — float per-vertex counts
 *   bc                   include/algorithm/bc/bc.cuh:8 — every vertex as a
 *                        source (the reference ignores `source` too, bc.cu:42),
 *                        prints the first 40 scores like bc.cu:84 and returns nothing
 *
 * The algorithms take thrust::device_vector<float>& as in the reference when
 * the including file is compiled by nvcc (results stay on the device); any
 * host float container with data(), size() and resize() (std::vector,
 * thrust::host_vector) works too, from any C++17 compiler.
 *
 * Device accessors of GraphVine: getVertexDictionary() is libgv's vertex
 * record array (opaque VertexDictionary*, see gv_vertex_records);
 * getCsrOffsetNewPointer / getCsrEdgesNewPointer / getSourceDegreesNewPointer
 * hold the last batch as the reference keeps it on the device (n+1 offsets,
 * 1-based destinations, n degrees, unsigned long); getSourceVectorPointer
 * holds the last batch's offsets again (the reference's array of that name is
 * scratch of its delete kernels, graphvine.cu:283-295);
 * getAffectedNodesPointer holds n flags (1 = endpoint of an entry of a batch
 * since construction), refreshed after every batch.
 *
 * Differences a caller can see: errors throw gv::Error instead of exiting
 * (include/util/cudaError.cuh:8-16); the destructor frees the store (the
 * reference's is `= default` and leaks); the store is kept symmetric —
 * every entry of a batch is applied in both directions.  That is what the
 * reference's reader produces (both directions arrive as entries, and the
 * set union stores each once), and it is what PageRank and triangle
 * counting assume; a reference batch that is not symmetric
 * (generate_random_batch) becomes symmetric here.  The affected flags mark
 * the 0-based endpoints (the reference's find_affected_nodes marks
 * destination + 1, insert_kernels.cu:190-193).  Nothing is printed except
 * by bc() and printDeviceVertexDictionary().
 *
 * Needs the CUDA runtime (cuda_runtime.h, -lcudart) for the device arrays.
 */
#ifndef GV_GRAPHVINE_HPP
#define GV_GRAPHVINE_HPP

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "gv.h"

#if defined(__CUDACC__)
#include <thrust/copy.h>
#include <thrust/device_vector.h>
#include <thrust/fill.h>
#include <thrust/host_vector.h>
#endif

// Batch size of the application, as in the reference (defined by the program).
extern size_t BATCH_SIZE;

namespace gv {

struct Error : std::runtime_error {
    gv_status status;
    Error(gv_status st, const std::string &where)
        : std::runtime_error(where + ": " + gv_last_error_string()), status(st) {}
};

inline void check(gv_status st, const char *where) {
    if (st != GV_OK) throw Error(st, where);
}

inline void check_cuda(cudaError_t e, const char *where) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(where) + ": " + cudaGetErrorString(e));
}

#if defined(__CUDACC__)
template <typename T>
using host_vector = thrust::host_vector<T>;
#else
template <typename T>
using host_vector = std::vector<T>;
#endif

// Device array of unsigned long owned by the shim.
class DeviceArray {
  public:
    DeviceArray() = default;
    ~DeviceArray() { release(); }
    DeviceArray(const DeviceArray &) = delete;
    DeviceArray &operator=(const DeviceArray &) = delete;
    void assign(const unsigned long *host, size_t count) {
        if (count > cap_) {
            release();
            check_cuda(cudaMalloc((void **)&p_, count * sizeof(unsigned long)), "device array");
            cap_ = count;
        }
        if (count) check_cuda(cudaMemcpy(p_, host, count * sizeof(unsigned long), cudaMemcpyHostToDevice), "copy");
        size_ = count;
    }
    unsigned long *data() const { return p_; }
    size_t size() const { return size_; }

  private:
    void release() {
        if (p_) cudaFree(p_);
        p_ = nullptr;
        cap_ = size_ = 0;
    }
    unsigned long *p_ = nullptr;
    size_t cap_ = 0, size_ = 0;
};

}  // namespace gv

// Graph sizes of the last file or batch the CSR held (graphStructures.cuh:8-17).
struct GraphProperties {
    unsigned long xDim = 0;
    unsigned long yDim = 0;
    unsigned long total_edges = 0;
    unsigned long max_degree = 0;
    unsigned long sum_degree = 0;
    unsigned long total_batches = 0;
    unsigned long batch_size = 0;
};

// Opaque: libgv's vertex records on the device (gv_vertex_records).
struct VertexDictionary;

// Host CSR with 1-based destinations (reference csr.cuh:14-47).
class CSR {
  public:
    CSR() = default;
    ~CSR() = default;

    // Shared by every CSR, as the reference's static member (csr.cu:3).
    inline static GraphProperties *h_graph_prop = new GraphProperties();

    // Matrix-Market file: header "rows cols entries", then 1-based
    // "src dst" lines, each stored in both directions (marketReader.cu:52-63).
    void readGraph(const char *fileLocation) {
        FILE *f = std::fopen(fileLocation, "r");
        if (!f) throw std::runtime_error(std::string("cannot open ") + fileLocation);
        char line[512];
        bool header = false;
        unsigned long idx = 0;
        while (std::fgets(line, sizeof line, f)) {
            if (line[0] == '%') continue;
            unsigned long a = 0, b = 0, c = 0;
            if (!header) {
                if (std::sscanf(line, "%lu %lu %lu", &a, &b, &c) != 3) continue;
                h_graph_prop->xDim = a;
                h_graph_prop->yDim = b;
                h_graph_prop->total_edges = 2 * c;
                h_source.assign(2 * c, 0);
                h_destination.assign(2 * c, 0);
                h_source_degrees.assign(a, 0);
                header = true;
                continue;
            }
            if (std::sscanf(line, "%lu %lu", &a, &b) != 2) continue;
            if (idx + 2 > h_source.size() || a == 0 || b == 0 || a > h_graph_prop->xDim || b > h_graph_prop->xDim) {
                std::fclose(f);
                throw std::runtime_error("Matrix-Market entry out of range");
            }
            h_source[idx] = a;
            h_destination[idx++] = b;
            h_source_degrees[a - 1]++;
            h_source[idx] = b;
            h_destination[idx++] = a;
            h_source_degrees[b - 1]++;
        }
        std::fclose(f);
        h_source.resize(idx);
        h_destination.resize(idx);
        h_graph_prop->total_edges = idx;
        computeGraphProperties();
        initializeCSR();
    }

    // Degree statistics and the number of BATCH_SIZE batches (csr.cu:20-55).
    void computeGraphProperties() {
        const unsigned long vs = h_graph_prop->xDim;
        h_graph_prop->max_degree = 0;
        h_graph_prop->sum_degree = 0;
        for (unsigned long i = 0; i < vs && i < h_source_degrees.size(); ++i) {
            h_graph_prop->max_degree = std::max(h_graph_prop->max_degree, h_source_degrees[i]);
            h_graph_prop->sum_degree += h_source_degrees[i];
        }
        const unsigned long bs = BATCH_SIZE ? BATCH_SIZE : 1;
        h_graph_prop->total_batches = (h_graph_prop->total_edges + bs - 1) / bs;
        h_source_degrees_new.assign(vs, 0);
        h_csr_offset_new.assign(vs + 1, 0);
    }

    // CSR of (h_source, h_destination) in input order per source (csr.cu:58-79).
    void initializeCSR() {
        const unsigned long vs = h_graph_prop->xDim;
        h_csr_offset_new.assign(vs + 1, 0);
        for (unsigned long v = 0; v < vs; ++v) h_csr_offset_new[v + 1] = h_csr_offset_new[v] + h_source_degrees[v];
        h_csr_edges_new.assign(h_source.size(), 0);
        std::vector<unsigned long> cur(h_csr_offset_new.begin(), h_csr_offset_new.end() - 1);
        for (size_t i = 0; i < h_source.size(); ++i) h_csr_edges_new[cur[h_source[i] - 1]++] = h_destination[i];
    }

    // batch_size entries drawn with srand(batch_number + 1) / rand(): per
    // entry the source (rand() % n) and then the 1-based destination
    // (rand() % n + 1), the reference's draw sequence (csr.cu:80-125), so
    // the same batch number gives the same batch with the same C library.
    void generate_random_batch(size_t batch_size, size_t batch_number) {
        const unsigned long vs = h_graph_prop->xDim;
        if (vs == 0) throw std::runtime_error("generate_random_batch needs the vertex count (read a graph first)");
        h_graph_prop->batch_size = batch_size;
        h_source_degrees.assign(vs, 0);
        h_source.assign(batch_size, 0);
        h_destination.assign(batch_size, 0);
        std::srand((unsigned)(batch_number + 1));
        for (size_t i = 0; i < batch_size; ++i) {
            const unsigned long src = (unsigned long)std::rand() % vs;
            h_source[i] = src + 1;
            h_destination[i] = (unsigned long)std::rand() % vs + 1;
            h_source_degrees[src]++;
        }
        h_graph_prop->total_edges = batch_size;
        computeGraphProperties();
        initializeCSR();
    }

    gv::host_vector<unsigned long> get_source_degree() const { return to_host(h_source_degrees); }
    gv::host_vector<unsigned long> get_source_degree_new() const { return to_host(h_source_degrees_new); }
    gv::host_vector<unsigned long> get_csr_offset() const { return to_host(h_csr_offset_new); }
    gv::host_vector<unsigned long> get_csr_edges() const { return to_host(h_csr_edges_new); }

    // --- used by the shim's GraphVine -------------------------------------
    unsigned long getVertexSize() const { return h_graph_prop->xDim; }
    const std::vector<unsigned long> &offsets() const { return h_csr_offset_new; }
    const std::vector<unsigned long> &edges() const { return h_csr_edges_new; }
    const std::vector<unsigned long> &degrees() const { return h_source_degrees; }

    // 0-based (src, dst) arrays for the C ABI.
    void toPairs(std::vector<uint32_t> &src, std::vector<uint32_t> &dst) const {
        const unsigned long vs = h_csr_offset_new.empty() ? 0 : h_csr_offset_new.size() - 1;
        src.resize(h_csr_edges_new.size());
        dst.resize(h_csr_edges_new.size());
        for (unsigned long u = 0; u < vs; ++u)
            for (unsigned long i = h_csr_offset_new[u]; i < h_csr_offset_new[u + 1]; ++i) {
                src[i] = (uint32_t)u;
                dst[i] = (uint32_t)(h_csr_edges_new[i] - 1);
            }
    }

  private:
    static gv::host_vector<unsigned long> to_host(const std::vector<unsigned long> &v) {
        return gv::host_vector<unsigned long>(v.begin(), v.end());
    }
    std::vector<unsigned long> h_source, h_destination;  // 1-based, input order
    std::vector<unsigned long> h_source_degrees;         // per 0-based source
    std::vector<unsigned long> h_source_degrees_new;
    std::vector<unsigned long> h_csr_offset_new;         // n + 1
    std::vector<unsigned long> h_csr_edges_new;          // 1-based destinations
};

class GraphVine {
  public:
    explicit GraphVine(CSR *csr, uint32_t block_size = 128, uint32_t threads_per_vertex = 8, int device = 0,
                       uint64_t hbm_budget_bytes = 0)
        : h_csr_(csr), n_(csr->getVertexSize()) {
        gv_config cfg;
        gv::check(gv_config_init(&cfg, (uint32_t)n_), "gv_config_init");
        cfg.block_size = block_size;
        cfg.threads_per_vertex = threads_per_vertex;
        cfg.directed = 0;  // symmetric store (see the header comment)
        cfg.device = device;
        cfg.hbm_budget_bytes = hbm_budget_bytes;
        gv::check(gv_create(&cfg, &g_), "gv_create");
        initiateVertexDictionary();
        initiateEdgeBlocks();
        initiateDeviceVectors();
        copyGraphDataFromHostToDevice();
        bulkBuild();
    }
    ~GraphVine() { gv_destroy(g_); }
    GraphVine(const GraphVine &) = delete;
    GraphVine &operator=(const GraphVine &) = delete;

    // gv_create allocated the vertex records and the block pool; these keep
    // the reference's construction steps callable (graphvine.cu:38-130).
    void initiateVertexDictionary() {}
    void initiateEdgeBlocks() {}
    void initiateDeviceVectors() {
        std::vector<unsigned long> zeros(n_ + 1, 0);
        affected_.assign(zeros.data(), n_);
        csr_offset_.assign(zeros.data(), n_ + 1);
        source_vector_.assign(zeros.data(), n_ + 1);
        source_degrees_.assign(zeros.data(), n_);
    }
    // The CSR's current batch into the device arrays (graphvine.cu:171-179).
    void copyGraphDataFromHostToDevice() { copy_batch(h_csr_); }

    void bulkBuild() { bulkBuild(h_csr_); }
    void bulkBuild(CSR *csr) { apply(csr, true, "bulkBuild"); }
    // kk is the batch number, unused as in the reference's insert path.
    void batchInsert(CSR *csr, size_t /*kk*/) { apply(csr, true, "batchInsert"); }
    void batchDelete(CSR *csr, size_t /*kk*/) { apply(csr, false, "batchDelete"); }
    void compaction() {
        gv::check(gv_compact(g_, nullptr), "compaction");
        gv::check(gv_synchronize(g_, nullptr), "compaction");
    }

    VertexDictionary *getVertexDictionary() {
        const void *p = nullptr;
        gv::check(gv_vertex_records(g_, &p), "getVertexDictionary");
        return (VertexDictionary *)const_cast<void *>(p);
    }
    unsigned long *getSourceVectorPointer() { return source_vector_.data(); }
    unsigned long *getAffectedNodesPointer() { return affected_.data(); }
    unsigned long *getCsrEdgesNewPointer() { return csr_edges_.data(); }
    unsigned long *getSourceDegreesNewPointer() { return source_degrees_.data(); }
    unsigned long *getCsrOffsetNewPointer() { return csr_offset_.data(); }
    unsigned long getVertexSize() const { return n_; }

    // One line per vertex: id, live entries (graphvine.cu:517-523 prints the dictionary).
    void printDeviceVertexDictionary() {
        std::vector<uint32_t> deg(n_);
        gv::check(gv_degrees(g_, deg.data(), GV_MEM_HOST, nullptr), "printDeviceVertexDictionary");
        std::printf("[Vertex Dictionary] ->\n");
        for (unsigned long v = 0; v < n_; ++v) std::printf("%lu: %u\n", v, deg[v]);
    }

    gv_graph *handle() const { return g_; }
    // Affected-vertex flags on the host (uint8 per vertex).
    std::vector<uint8_t> getAffectedNodes() {
        std::vector<uint8_t> a(n_);
        gv::check(gv_affected(g_, a.data(), GV_MEM_HOST, nullptr), "affected");
        return a;
    }

  private:
    void copy_batch(const CSR *csr) {
        const auto &off = csr->offsets();
        const auto &edg = csr->edges();
        const auto &deg = csr->degrees();
        if (off.size() == n_ + 1) {
            csr_offset_.assign(off.data(), off.size());
            source_vector_.assign(off.data(), off.size());
        }
        if (!edg.empty()) csr_edges_.assign(edg.data(), edg.size());
        if (deg.size() == n_) source_degrees_.assign(deg.data(), deg.size());
    }
    void refresh_affected() {
        std::vector<uint8_t> a(n_);
        gv::check(gv_affected(g_, a.data(), GV_MEM_HOST, nullptr), "affected");
        std::vector<unsigned long> w(a.begin(), a.end());
        affected_.assign(w.data(), w.size());
    }
    void apply(CSR *csr, bool insert, const char *where) {
        std::vector<uint32_t> s, d;
        csr->toPairs(s, d);
        gv_status st = insert ? gv_insert_edges(g_, s.data(), d.data(), nullptr, s.size(), GV_MEM_HOST, nullptr)
                              : gv_delete_edges(g_, s.data(), d.data(), s.size(), GV_MEM_HOST, nullptr);
        gv::check(st, where);
        gv::check(gv_synchronize(g_, nullptr), where);
        copy_batch(csr);
        refresh_affected();
    }

    CSR *h_csr_;
    unsigned long n_;
    gv_graph *g_ = nullptr;
    gv::DeviceArray affected_, csr_offset_, csr_edges_, source_degrees_, source_vector_;
};

// ---------------------------------------------------------------- algorithms
// Host containers: result in v1 (pagerank.cu:64); v2 is the reference's
// work vector and is left untouched.
template <typename Vec>
inline void static_pagerank(GraphVine *graph, float alpha, float epsilon, int max_iter, Vec &v1, Vec & /*v2*/) {
    v1.resize(graph->getVertexSize());
    int32_t sweeps = 0;
    gv::check(gv_pagerank(graph->handle(), alpha, epsilon, max_iter, v1.data(), &sweeps, GV_MEM_HOST, nullptr),
              "static_pagerank");
}

// Warm start from v1 (the previous result), converging to the same fixed point.
template <typename Vec>
inline void dynamic_pagerank(GraphVine *graph, float alpha, float epsilon, int max_iter, Vec &v1, Vec & /*v2*/) {
    if (v1.size() != graph->getVertexSize()) {  // no previous result: start from 1/n
        v1.resize(graph->getVertexSize());
        std::fill(v1.begin(), v1.end(), 1.0f / (float)graph->getVertexSize());
    }
    int32_t sweeps = 0;
    gv::check(gv_pagerank_dynamic(graph->handle(), alpha, epsilon, max_iter, v1.data(), &sweeps, GV_MEM_HOST,
                                  nullptr),
              "dynamic_pagerank");
}

// Per-vertex counts as float, the reference's output type (tc.cuh:10).
template <typename Vec>
inline void static_tc(GraphVine *graph, Vec &counts) {
    std::vector<uint64_t> pv(graph->getVertexSize());
    uint64_t total = 0;
    gv::check(gv_tc(graph->handle(), pv.data(), &total, GV_MEM_HOST, nullptr), "static_tc");
    counts.resize(pv.size());
    for (size_t i = 0; i < pv.size(); ++i) counts[i] = (float)pv[i];
}

// The exact count after the batches (the reference's dynamic_tc recounts
// only the triangles owned by affected vertices, tc.cu:29-64).
template <typename Vec>
inline void dynamic_tc(GraphVine *graph, Vec &counts) { static_tc(graph, counts); }

#if defined(__CUDACC__)
// Device vectors, the reference's signatures: results stay on the device.
inline void static_pagerank(GraphVine *graph, float alpha, float epsilon, int max_iter,
                            thrust::device_vector<float> &d_pageRankVector_1,
                            thrust::device_vector<float> & /*d_pageRankVector_2*/) {
    d_pageRankVector_1.resize(graph->getVertexSize());
    int32_t sweeps = 0;
    gv::check(gv_pagerank(graph->handle(), alpha, epsilon, max_iter,
                          thrust::raw_pointer_cast(d_pageRankVector_1.data()), &sweeps, GV_MEM_DEVICE, nullptr),
              "static_pagerank");
}

inline void dynamic_pagerank(GraphVine *graph, float alpha, float epsilon, int max_iter,
                             thrust::device_vector<float> &d_pageRankVector_1,
                             thrust::device_vector<float> & /*d_pageRankVector_2*/) {
    const size_t n = graph->getVertexSize();
    if (d_pageRankVector_1.size() != n) {
        d_pageRankVector_1.resize(n);
        thrust::fill(d_pageRankVector_1.begin(), d_pageRankVector_1.end(), 1.0f / (float)n);
    }
    int32_t sweeps = 0;
    gv::check(gv_pagerank_dynamic(graph->handle(), alpha, epsilon, max_iter,
                                  thrust::raw_pointer_cast(d_pageRankVector_1.data()), &sweeps, GV_MEM_DEVICE,
                                  nullptr),
              "dynamic_pagerank");
}

inline void static_tc(GraphVine *graph, thrust::device_vector<float> &d_triangleCount) {
    thrust::device_vector<unsigned long long> pv(graph->getVertexSize());
    uint64_t total = 0;
    gv::check(gv_tc(graph->handle(), (uint64_t *)thrust::raw_pointer_cast(pv.data()), &total, GV_MEM_DEVICE,
                    nullptr),
              "static_tc");
    d_triangleCount.resize(pv.size());
    thrust::copy(pv.begin(), pv.end(), d_triangleCount.begin());  // uint64 -> float on the device
}

inline void dynamic_tc(GraphVine *graph, thrust::device_vector<float> &d_triangleCount) {
    static_tc(graph, d_triangleCount);
}
#endif

// Scores with every vertex as a source, summed without halving (bc.cu:42-80).
inline std::vector<float> bc_scores(GraphVine *graph) {
    std::vector<float> out(graph->getVertexSize());
    gv::check(gv_bc(graph->handle(), nullptr, 0, out.data(), GV_MEM_HOST, nullptr), "bc");
    return out;
}

// The reference's bc: computes the scores and prints the first 40 (bc.cu:84).
inline void bc(GraphVine *graph, int /*source*/) {
    const std::vector<float> s = bc_scores(graph);
    std::printf("[BC] -> ");
    for (size_t i = 0; i < s.size() && i < 40; ++i) std::printf("%f ", s[i]);
    std::printf("\n");
}

#endif  // GV_GRAPHVINE_HPP
