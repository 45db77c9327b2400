// Test-infrastructure driver for the reference implementation (sajidanis/GV),
// linked against the reference's own, unmodified CUDA sources by
// oracle/ref_build.py.  It runs the reference's public host API on a script
// of operations and writes what the reference's data structure holds, so the
// oracle can be pinned against the reference itself.
//
//   gv_ref_harness <script>
//
// Script lines (paths are Matrix-Market files with 1-based ids, each
// undirected edge listed once; the reference's reader symmetrises them,
// src/reader/marketReader.cu:58-64):
//   graph <mtx>                      CSR::readGraph + GraphVine(CSR*) (bulkBuild)
//   insert <mtx>                     GraphVine::batchInsert (graphvine.cu:222)
//   delete <mtx>                     GraphVine::batchDelete (graphvine.cu:373)
//   compact                          GraphVine::compaction (graphvine.cu:453)
//   dump <out>                       adjacency the store holds (0-based CSR)
//   pagerank <alpha> <eps> <max> <out>   static_pagerank (pagerank.cu:3)
//   tc <out>                         static_tc (tc.cu:3), float per vertex
//
// Only inputs inside the regimes where the reference is well defined are
// fed to it (see tests/test_ref_pin.py).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "graphvine.cuh"
#include "pagerank.cuh"
#include "tc.cuh"
#include "device_functions.cuh"

size_t BATCH_SIZE = 1 << 20;

namespace {

__global__ void dump_count(VertexDictionary *vd, unsigned long n, unsigned long long *cnt) {
    unsigned long v = blockIdx.x * (unsigned long)blockDim.x + threadIdx.x;
    if (v >= n) return;
    unsigned long nb = vd->edge_block_count[v];
    EdgeBlock *root = vd->edge_block_address[v];
    unsigned long long c = 0;
    if (root) {
        for (unsigned long i = 0; i < nb; ++i) {
            EdgeBlock *b = traverse_bit_string(root, bit_string_lookup[i]);
            if (!b) break;
            for (int j = 0; j < EDGE_BLOCK_SIZE; ++j) {
                unsigned long e = b->edge_block_entry[j].destination_vertex;
                if (e != 0 && e != INFTY) ++c;
            }
        }
    }
    cnt[v] = c;
}

__global__ void dump_fill(VertexDictionary *vd, unsigned long n, const unsigned long long *off, unsigned int *out) {
    unsigned long v = blockIdx.x * (unsigned long)blockDim.x + threadIdx.x;
    if (v >= n) return;
    unsigned long nb = vd->edge_block_count[v];
    EdgeBlock *root = vd->edge_block_address[v];
    unsigned long long w = off[v];
    if (!root) return;
    for (unsigned long i = 0; i < nb; ++i) {
        EdgeBlock *b = traverse_bit_string(root, bit_string_lookup[i]);
        if (!b) break;
        for (int j = 0; j < EDGE_BLOCK_SIZE; ++j) {
            unsigned long e = b->edge_block_entry[j].destination_vertex;
            if (e != 0 && e != INFTY && w < off[v + 1]) out[w++] = (unsigned int)(e - 1);
        }
    }
}

void check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "harness: %s: %s\n", what, cudaGetErrorString(e));
        std::exit(3);
    }
}

unsigned long count_lines(const std::string &mtx) {
    std::ifstream f(mtx);
    std::string line;
    unsigned long k = 0;
    bool header = false;
    while (std::getline(f, line)) {
        if (line.empty() || line[0] == '%') continue;
        if (!header) { header = true; continue; }
        ++k;
    }
    return k;
}

CSR *read_batch(const std::string &mtx) {
    CSR *c = new CSR();
    std::vector<char> path(mtx.begin(), mtx.end());
    path.push_back('\0');
    c->readGraph(path.data());
    // the reference sizes batch kernels from h_graph_prop->batch_size
    CSR::h_graph_prop->batch_size = 2 * count_lines(mtx);
    return c;
}

void dump(GraphVine *g, const std::string &out) {
    const unsigned long n = g->getVertexSize();
    unsigned long long *cnt = nullptr, *off = nullptr;
    check(cudaMalloc(&cnt, (n + 1) * 8), "malloc");
    check(cudaMalloc(&off, (n + 1) * 8), "malloc");
    dump_count<<<(n + 127) / 128, 128>>>(g->getVertexDictionary(), n, cnt);
    check(cudaDeviceSynchronize(), "dump_count");
    std::vector<unsigned long long> h(n + 1, 0), ho(n + 1, 0);
    check(cudaMemcpy(h.data(), cnt, n * 8, cudaMemcpyDeviceToHost), "copy");
    for (unsigned long v = 0; v < n; ++v) ho[v + 1] = ho[v] + h[v];
    check(cudaMemcpy(off, ho.data(), (n + 1) * 8, cudaMemcpyHostToDevice), "copy");
    unsigned int *dst = nullptr;
    check(cudaMalloc(&dst, (ho[n] + 1) * 4), "malloc");
    dump_fill<<<(n + 127) / 128, 128>>>(g->getVertexDictionary(), n, off, dst);
    check(cudaDeviceSynchronize(), "dump_fill");
    std::vector<unsigned int> hd(ho[n]);
    if (ho[n]) check(cudaMemcpy(hd.data(), dst, ho[n] * 4, cudaMemcpyDeviceToHost), "copy");
    FILE *f = std::fopen(out.c_str(), "wb");
    std::fwrite(&n, 8, 1, f);
    std::fwrite(ho.data(), 8, n + 1, f);
    if (ho[n]) std::fwrite(hd.data(), 4, ho[n], f);
    std::fclose(f);
    cudaFree(cnt);
    cudaFree(off);
    cudaFree(dst);
}

template <typename T>
void write_vec(const std::string &out, const thrust::device_vector<T> &v) {
    thrust::host_vector<T> h = v;
    FILE *f = std::fopen(out.c_str(), "wb");
    unsigned long n = h.size();
    std::fwrite(&n, 8, 1, f);
    std::fwrite(h.data(), sizeof(T), n, f);
    std::fclose(f);
}

}  // namespace

int main(int argc, char **argv) {
    if (argc != 2) {
        std::fprintf(stderr, "usage: %s <script>\n", argv[0]);
        return 2;
    }
    std::ifstream script(argv[1]);
    std::string line;
    CSR *csr = nullptr;
    GraphVine *g = nullptr;
    while (std::getline(script, line)) {
        std::istringstream is(line);
        std::string op;
        if (!(is >> op)) continue;
        if (op == "graph") {
            std::string p;
            is >> p;
            csr = read_batch(p);
            g = new GraphVine(csr);
        } else if (op == "insert" || op == "delete") {
            std::string p;
            is >> p;
            CSR *b = read_batch(p);
            if (op == "insert") g->batchInsert(b, 1);
            else g->batchDelete(b, 1);
        } else if (op == "compact") {
            g->compaction();
        } else if (op == "dump") {
            std::string p;
            is >> p;
            dump(g, p);
        } else if (op == "pagerank") {
            float alpha, eps;
            int mx;
            std::string p;
            is >> alpha >> eps >> mx >> p;
            const unsigned long n = g->getVertexSize();
            thrust::device_vector<float> v1(n), v2(n);
            static_pagerank(g, alpha, eps, mx, v1, v2);
            write_vec(p, v1);
        } else if (op == "tc") {
            std::string p;
            is >> p;
            thrust::device_vector<float> t(g->getVertexSize());
            static_tc(g, t);
            write_vec(p, t);
        } else {
            std::fprintf(stderr, "unknown op %s\n", op.c_str());
            return 2;
        }
        check(cudaDeviceSynchronize(), op.c_str());
        std::fprintf(stderr, "harness: %s done\n", op.c_str());
    }
    return 0;
}
