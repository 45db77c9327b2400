// Reference-style driver in the reference's own idiom (src/main.cu:40-119):
// a CSR read from a file, GraphVine(CSR*), random batches from
// CSR::generate_random_batch(BATCH_SIZE, kk) inserted and deleted, then the
// algorithms with thrust::device_vector<float> results
// (pagerank.cuh:11-13, tc.cuh:10-12) and the GraphVine device accessors.
// Built by nvcc against include/graphvine.hpp and libgv.
// Usage: compat_example_thrust <graph.mtx> <batch_size> <out_prefix>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include <thrust/device_vector.h>
#include <thrust/host_vector.h>

#include "graphvine.hpp"

size_t BATCH_SIZE = 10000000;

template <typename T>
static void dump(const std::string &path, const T *p, size_t count) {
    FILE *f = std::fopen(path.c_str(), "wb");
    std::fwrite(p, sizeof(T), count, f);
    std::fclose(f);
}

template <typename T>
static std::vector<T> from_device(const T *d, size_t count) {
    std::vector<T> h(count);
    gv::check_cuda(cudaMemcpy(h.data(), d, count * sizeof(T), cudaMemcpyDeviceToHost), "copy back");
    return h;
}

int main(int argc, char **argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s <graph.mtx> <batch_size> <out_prefix>\n", argv[0]);
        return 2;
    }
    BATCH_SIZE = std::strtoul(argv[2], nullptr, 10);
    const std::string pre = argv[3];
    try {
        CSR *csr = new CSR();
        csr->readGraph(argv[1]);
        GraphVine *dynGraph = new GraphVine(csr);
        const size_t vertex_size = CSR::h_graph_prop->xDim;
        size_t kk = 1;
        // insert batch kk, then delete batch kk + 1 (main.cu:90-105)
        csr->generate_random_batch(BATCH_SIZE, kk);
        thrust::host_vector<unsigned long> ins_off = csr->get_csr_offset();
        thrust::host_vector<unsigned long> ins_edges = csr->get_csr_edges();
        dynGraph->batchInsert(csr, kk);
        std::vector<unsigned long> aff = from_device(dynGraph->getAffectedNodesPointer(), vertex_size);
        dump(pre + ".ins_off", ins_off.data(), ins_off.size());
        dump(pre + ".ins_edges", ins_edges.data(), ins_edges.size());
        dump(pre + ".affected", aff.data(), aff.size());
        csr->generate_random_batch(BATCH_SIZE, kk + 1);
        dynGraph->batchDelete(csr, kk + 1);
        // the batch as the device accessors hold it
        std::vector<unsigned long> d_off = from_device(dynGraph->getCsrOffsetNewPointer(), vertex_size + 1);
        std::vector<unsigned long> d_edges = from_device(dynGraph->getCsrEdgesNewPointer(), (size_t)d_off[vertex_size]);
        std::vector<unsigned long> d_deg = from_device(dynGraph->getSourceDegreesNewPointer(), vertex_size);
        dump(pre + ".del_off", d_off.data(), d_off.size());
        dump(pre + ".del_edges", d_edges.data(), d_edges.size());
        dump(pre + ".del_deg", d_deg.data(), d_deg.size());
        dynGraph->compaction();

        thrust::device_vector<float> d_pageRankVector_1(vertex_size);
        thrust::device_vector<float> d_pageRankVector_2(vertex_size);
        static_pagerank(dynGraph, 0.85f, 1e-6f, 100, d_pageRankVector_1, d_pageRankVector_2);
        thrust::host_vector<float> pr = d_pageRankVector_1;
        dump(pre + ".pr", pr.data(), pr.size());
        // a warm start from the converged vector stays at the fixed point
        dynamic_pagerank(dynGraph, 0.85f, 1e-6f, 100, d_pageRankVector_1, d_pageRankVector_2);
        thrust::host_vector<float> pr_dyn = d_pageRankVector_1;
        dump(pre + ".pr_dyn", pr_dyn.data(), pr_dyn.size());

        thrust::device_vector<float> d_triangleCount(vertex_size);
        static_tc(dynGraph, d_triangleCount);
        thrust::host_vector<float> tc = d_triangleCount;
        dump(pre + ".tc", tc.data(), tc.size());
        dynamic_tc(dynGraph, d_triangleCount);
        thrust::host_vector<float> tc_dyn = d_triangleCount;
        dump(pre + ".tc_dyn", tc_dyn.data(), tc_dyn.size());

        if (dynGraph->getVertexDictionary() == nullptr) throw std::runtime_error("no vertex records");
        bc(dynGraph, 0);  // prints the first 40 scores
        std::printf("ok n=%zu\n", vertex_size);
        delete dynGraph;
        delete csr;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
