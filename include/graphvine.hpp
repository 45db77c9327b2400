/*
 * graphvine.hpp — header-only C++ shim that keeps the reference's host API
 * (sajidanis/GV) compiling on top of libgv's C ABI (gv.h).
 *
 * Reference interfaces kept, with their semantics:
 *   class CSR            include/dynamicStructure/csr.cuh:14-47 — host batch
 *                        container; destinations are 1-based as in the
 *                        reference (src/dynamicStructure/csr.cu:55-78)
 *   class GraphVine      include/dynamicStructure/graphvine.cuh:29-58 —
 *                        GraphVine(CSR*) builds the store from the CSR
 *                        (graphvine.cu:5-35), batchInsert / batchDelete /
 *                        compaction are synchronous like the reference
 *                        (graphvine.cu:367, :446, :461)
 *   static_pagerank      include/algorithm/pagerank/pagerank.cuh:11 — result in v1
 *   dynamic_pagerank     include/algorithm/pagerank/pagerank.cuh:13 — warm start from v1
 *   static_tc            include/algorithm/tc/tc.cuh:10 — float per-vertex counts
 *   bc                   include/algorithm/bc/bc.cuh:8 — all sources; the
 *                        reference ignores `source` too (bc.cu:42)
 *
 * Differences a caller can see: errors throw gv::Error instead of exiting
 * (include/util/cudaError.cuh:8-16); the store is kept symmetric — every
 * entry of a batch is applied in both directions.  That is what the
 * reference's reader produces (both directions arrive as entries, and the
 * set union stores each once), and it is what PageRank and triangle
 * counting assume; a reference batch that is not symmetric
 * (generate_random_batch, csr.cu:93-117) becomes symmetric here.  Vectors
 * passed to the algorithms are host float containers with data(), size()
 * and resize() (std::vector, thrust::host_vector); results that must stay
 * on the device go through the C ABI with GV_MEM_DEVICE.
 */
#ifndef GV_GRAPHVINE_HPP
#define GV_GRAPHVINE_HPP

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "gv.h"

namespace gv {

struct Error : std::runtime_error {
    gv_status status;
    Error(gv_status st, const std::string &where)
        : std::runtime_error(where + ": " + gv_last_error_string()), status(st) {}
};

inline void check(gv_status st, const char *where) {
    if (st != GV_OK) throw Error(st, where);
}

}  // namespace gv

// Host CSR with 1-based destinations (reference csr.cuh:14-47).
class CSR {
  public:
    unsigned long n = 0;
    std::vector<unsigned long> offsets;  // n + 1
    std::vector<unsigned long> edges;    // 1-based destinations

    // Matrix-Market reader; symmetrises like src/reader/marketReader.cu:58-64.
    void readGraph(const char *path) {
        FILE *f = std::fopen(path, "r");
        if (!f) throw std::runtime_error(std::string("cannot open ") + path);
        char line[512];
        bool header = false;
        std::vector<std::pair<unsigned long, unsigned long>> e;
        while (std::fgets(line, sizeof line, f)) {
            if (line[0] == '%') continue;
            unsigned long a = 0, b = 0, c = 0;
            if (!header) {
                if (std::sscanf(line, "%lu %lu %lu", &a, &b, &c) == 3) {
                    n = a;
                    header = true;
                }
                continue;
            }
            if (std::sscanf(line, "%lu %lu", &a, &b) == 2) {
                e.push_back({a, b});
                e.push_back({b, a});
            }
        }
        std::fclose(f);
        fromEntries(e);
    }

    // Builds the CSR from (src, dst) entries, both 1-based.
    void fromEntries(const std::vector<std::pair<unsigned long, unsigned long>> &e) {
        offsets.assign(n + 1, 0);
        for (auto &p : e) offsets[p.first]++;  // count at src (1-based -> index src)
        for (unsigned long v = 0; v < n; ++v) offsets[v + 1] += offsets[v];
        edges.assign(e.size(), 0);
        std::vector<unsigned long> cur(offsets.begin(), offsets.end() - 1);
        for (auto &p : e) edges[cur[p.first - 1]++] = p.second;
    }

    // Random batch of `batch_size` entries seeded by batch_number, the shape
    // of src/dynamicStructure/csr.cu:80-125 (uniform sources and destinations).
    void generate_random_batch(size_t batch_size, size_t batch_number) {
        std::vector<std::pair<unsigned long, unsigned long>> e;
        e.reserve(batch_size);
        uint64_t x = 0x9E3779B97F4A7C15ull * (batch_number + 1);
        for (size_t i = 0; i < batch_size; ++i) {
            x ^= x << 13; x ^= x >> 7; x ^= x << 17;
            const unsigned long s = x % n;
            x ^= x << 13; x ^= x >> 7; x ^= x << 17;
            e.push_back({s + 1, (x % n) + 1});
        }
        fromEntries(e);
    }

    unsigned long getVertexSize() const { return n; }
    unsigned long numEntries() const { return edges.size(); }

    // 0-based (src, dst) arrays for the C ABI.
    void toPairs(std::vector<uint32_t> &src, std::vector<uint32_t> &dst) const {
        src.resize(edges.size());
        dst.resize(edges.size());
        for (unsigned long u = 0; u < n; ++u)
            for (unsigned long i = offsets[u]; i < offsets[u + 1]; ++i) {
                src[i] = (uint32_t)u;
                dst[i] = (uint32_t)(edges[i] - 1);
            }
    }
};

class GraphVine {
  public:
    explicit GraphVine(CSR *csr, uint32_t block_size = 128, uint32_t threads_per_vertex = 8, int device = 0,
                       uint64_t hbm_budget_bytes = 0)
        : n_(csr->getVertexSize()) {
        gv_config cfg;
        gv::check(gv_config_init(&cfg, (uint32_t)n_), "gv_config_init");
        cfg.block_size = block_size;
        cfg.threads_per_vertex = threads_per_vertex;
        cfg.directed = 0;  // symmetric store (see the header comment)
        cfg.device = device;
        cfg.hbm_budget_bytes = hbm_budget_bytes;
        gv::check(gv_create(&cfg, &g_), "gv_create");
        bulkBuild(csr);
    }
    ~GraphVine() { gv_destroy(g_); }
    GraphVine(const GraphVine &) = delete;
    GraphVine &operator=(const GraphVine &) = delete;

    void bulkBuild(CSR *csr) {
        std::vector<uint32_t> s, d;
        csr->toPairs(s, d);
        gv::check(gv_insert_edges(g_, s.data(), d.data(), nullptr, s.size(), GV_MEM_HOST, nullptr), "bulkBuild");
        gv::check(gv_synchronize(g_, nullptr), "bulkBuild");
    }
    // kk is the batch number (kept for signature compatibility).
    void batchInsert(CSR *csr, size_t /*kk*/) {
        std::vector<uint32_t> s, d;
        csr->toPairs(s, d);
        gv::check(gv_insert_edges(g_, s.data(), d.data(), nullptr, s.size(), GV_MEM_HOST, nullptr), "batchInsert");
        gv::check(gv_synchronize(g_, nullptr), "batchInsert");
    }
    void batchDelete(CSR *csr, size_t /*kk*/) {
        std::vector<uint32_t> s, d;
        csr->toPairs(s, d);
        gv::check(gv_delete_edges(g_, s.data(), d.data(), s.size(), GV_MEM_HOST, nullptr), "batchDelete");
        gv::check(gv_synchronize(g_, nullptr), "batchDelete");
    }
    void compaction() {
        gv::check(gv_compact(g_, nullptr), "compaction");
        gv::check(gv_synchronize(g_, nullptr), "compaction");
    }
    unsigned long getVertexSize() const { return n_; }
    gv_graph *handle() const { return g_; }
    // Affected-vertex flags (getAffectedNodesPointer, graphvine.cu:501-503), on the host.
    std::vector<uint8_t> getAffectedNodes() {
        std::vector<uint8_t> a(n_);
        gv::check(gv_affected(g_, a.data(), GV_MEM_HOST, nullptr), "affected");
        return a;
    }

  private:
    unsigned long n_;
    gv_graph *g_ = nullptr;
};

// Result in v1 (pagerank.cu:64); v2 is the reference's work vector and is
// left untouched.
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

template <typename Vec>
inline void dynamic_tc(GraphVine *graph, Vec &counts) { static_tc(graph, counts); }

// All sources, printed like the reference's bc (bc.cu:84); returns the scores.
inline std::vector<float> bc(GraphVine *graph, int /*source*/) {
    std::vector<float> out(graph->getVertexSize());
    gv::check(gv_bc(graph->handle(), nullptr, 0, out.data(), GV_MEM_HOST, nullptr), "bc");
    return out;
}

#endif  // GV_GRAPHVINE_HPP
