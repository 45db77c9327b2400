// Reference-style driver written against include/graphvine.hpp with host
// containers: the same calls src/main.cu:46-119 makes (readGraph,
// GraphVine(CSR*), batchInsert, batchDelete, compaction, static_pagerank,
// static_tc, bc), on libgv, built by a plain C++ compiler.
// Usage: compat_example <graph.mtx> <insert.mtx> <delete.mtx> <out_prefix>
#include <cstdio>
#include <vector>

#include "graphvine.hpp"

size_t BATCH_SIZE = 1000;  // the application defines it, as src/main.cu:18 does

int main(int argc, char **argv) {
    if (argc != 5) {
        std::fprintf(stderr, "usage: %s <graph.mtx> <insert.mtx> <delete.mtx> <out_prefix>\n", argv[0]);
        return 2;
    }
    try {
        CSR csr;
        csr.readGraph(argv[1]);
        GraphVine g(&csr, 128, 8, 0, 1ull << 30);
        CSR ins;
        ins.readGraph(argv[2]);
        g.batchInsert(&ins, 1);
        CSR del;
        del.readGraph(argv[3]);
        g.batchDelete(&del, 2);
        g.compaction();
        std::vector<float> pr1, pr2, tc;
        static_pagerank(&g, 0.85f, 1e-6f, 100, pr1, pr2);
        static_tc(&g, tc);
        std::vector<float> b = bc_scores(&g);
        const std::string pre = argv[4];
        auto dump = [&](const char *name, const std::vector<float> &v) {
            FILE *f = std::fopen((pre + name).c_str(), "wb");
            std::fwrite(v.data(), sizeof(float), v.size(), f);
            std::fclose(f);
        };
        dump(".pr", pr1);
        dump(".tc", tc);
        dump(".bc", b);
        std::printf("ok n=%lu\n", g.getVertexSize());
    } catch (const std::exception &e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
