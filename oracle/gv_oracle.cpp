// CPU restatement of GraphVine's dynamic-graph hot path (test infrastructure;
// see gv_oracle.h).  Adjacency is kept as a sorted vector per vertex, so every
// operation states the set semantics directly.
#include "gv_oracle.h"

#include <omp.h>
#include <parallel/algorithm>

#include <algorithm>
#include <atomic>
#include <iterator>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "../gv_b200/csrc/rmat.h"

struct or_graph {
    uint32_t n;
    bool directed;
    bool weighted;
    std::vector<std::vector<uint32_t>> adj;
    std::vector<std::vector<float>> w;
};

namespace {

struct Entry {
    uint32_t s, d;
    float w;
    uint64_t order;
};

// Expanded batch in the order the reference's CSR would hold it: pair i gives
// (s, d) then, on an undirected graph, (d, s).
std::vector<Entry> expand(const uint32_t *src, const uint32_t *dst, const float *w, uint64_t k, bool sym) {
    std::vector<Entry> e;
    e.reserve(sym ? 2 * k : k);
    for (uint64_t i = 0; i < k; ++i) {
        if (src[i] == dst[i]) continue;  // self-loop (insert_kernels.cu:174)
        const float wi = w ? w[i] : 1.0f;
        e.push_back({src[i], dst[i], wi, sym ? 2 * i : i});
        if (sym) e.push_back({dst[i], src[i], wi, 2 * i + 1});
    }
    return e;
}

bool in_range(const or_graph *g, const uint32_t *src, const uint32_t *dst, uint64_t k) {
    for (uint64_t i = 0; i < k; ++i)
        if (src[i] >= g->n || dst[i] >= g->n) return false;
    return true;
}

// Groups sorted entries by source: returns [begin, end) ranges.
std::vector<std::pair<size_t, size_t>> groups(const std::vector<Entry> &e) {
    std::vector<std::pair<size_t, size_t>> r;
    size_t i = 0;
    while (i < e.size()) {
        size_t j = i;
        while (j < e.size() && e[j].s == e[i].s) ++j;
        r.push_back({i, j});
        i = j;
    }
    return r;
}

// Unweighted insert: duplicates are identical, so a parallel sort of packed
// (src << 32 | dst) keys states the same set union.
int insert_keys(or_graph *g, const uint32_t *src, const uint32_t *dst, uint64_t k, bool sym) {
    std::vector<uint64_t> keys;
    keys.reserve(sym ? 2 * k : k);
    for (uint64_t i = 0; i < k; ++i) {
        if (src[i] == dst[i]) continue;
        keys.push_back(((uint64_t)src[i] << 32) | dst[i]);
        if (sym) keys.push_back(((uint64_t)dst[i] << 32) | src[i]);
    }
    __gnu_parallel::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    std::vector<size_t> starts;
    for (size_t i = 0; i < keys.size(); ++i)
        if (i == 0 || (keys[i] >> 32) != (keys[i - 1] >> 32)) starts.push_back(i);
    starts.push_back(keys.size());
    const long ngroups = (long)starts.size() - 1;
#pragma omp parallel for schedule(dynamic, 256)
    for (long gi = 0; gi < ngroups; ++gi) {
        const uint32_t s = (uint32_t)(keys[starts[gi]] >> 32);
        std::vector<uint32_t> &a = g->adj[s];
        std::vector<uint32_t> add;
        add.reserve(starts[gi + 1] - starts[gi]);
        for (size_t q = starts[gi]; q < starts[gi + 1]; ++q) add.push_back((uint32_t)keys[q]);
        std::vector<uint32_t> na;
        na.reserve(a.size() + add.size());
        std::set_union(a.begin(), a.end(), add.begin(), add.end(), std::back_inserter(na));
        a.swap(na);
    }
    return 0;
}

int insert_impl(or_graph *g, const uint32_t *src, const uint32_t *dst, const float *w, uint64_t k, bool sym) {
    if (!in_range(g, src, dst, k)) return -1;
    if (!g->weighted) return insert_keys(g, src, dst, k, sym);
    std::vector<Entry> e = expand(src, dst, w, k, sym);
    std::stable_sort(e.begin(), e.end(), [](const Entry &a, const Entry &b) {
        return a.s != b.s ? a.s < b.s : (a.d != b.d ? a.d < b.d : a.order < b.order);
    });
    // keep the first occurrence of every (s, d)
    std::vector<Entry> u;
    u.reserve(e.size());
    for (size_t i = 0; i < e.size(); ++i)
        if (i == 0 || e[i].s != e[i - 1].s || e[i].d != e[i - 1].d) u.push_back(e[i]);
    auto gr = groups(u);
#pragma omp parallel for schedule(dynamic, 64)
    for (long gi = 0; gi < (long)gr.size(); ++gi) {
        const uint32_t s = u[gr[gi].first].s;
        std::vector<uint32_t> &a = g->adj[s];
        std::vector<uint32_t> na;
        std::vector<float> nw;
        na.reserve(a.size() + (gr[gi].second - gr[gi].first));
        size_t p = 0;
        for (size_t q = gr[gi].first; q < gr[gi].second; ++q) {
            const uint32_t d = u[q].d;
            while (p < a.size() && a[p] < d) {
                na.push_back(a[p]);
                if (g->weighted) nw.push_back(g->w[s][p]);
                ++p;
            }
            if (p < a.size() && a[p] == d) continue;  // already present: existing entry wins
            na.push_back(d);
            if (g->weighted) nw.push_back(u[q].w);
        }
        while (p < a.size()) {
            na.push_back(a[p]);
            if (g->weighted) nw.push_back(g->w[s][p]);
            ++p;
        }
        a.swap(na);
        if (g->weighted) g->w[s].swap(nw);
    }
    return 0;
}

// In-adjacency (transpose) for pull-style sweeps on directed graphs.
void transpose(const or_graph *g, std::vector<uint64_t> &off, std::vector<uint32_t> &src,
               std::vector<double> *pw, const std::vector<double> *rowscale) {
    const uint32_t n = g->n;
    off.assign(n + 1, 0);
    for (uint32_t u = 0; u < n; ++u)
        for (uint32_t v : g->adj[u]) off[v + 1]++;
    for (uint32_t v = 0; v < n; ++v) off[v + 1] += off[v];
    src.assign(off[n], 0);
    if (pw) pw->assign(off[n], 0.0);
    std::vector<uint64_t> cur(off.begin(), off.end() - 1);
    for (uint32_t u = 0; u < n; ++u)
        for (size_t i = 0; i < g->adj[u].size(); ++i) {
            const uint32_t v = g->adj[u][i];
            const uint64_t p = cur[v]++;
            src[p] = u;
            if (pw) (*pw)[p] = (double)g->w[u][i] * (*rowscale)[u];
        }
}

}  // namespace

extern "C" {

or_graph *or_create(uint32_t n, int directed, int weighted) {
    or_graph *g = new or_graph();
    g->n = n;
    g->directed = directed != 0;
    g->weighted = weighted != 0;
    g->adj.resize(n);
    if (g->weighted) g->w.resize(n);
    return g;
}

void or_destroy(or_graph *g) { delete g; }

int or_set_threads(int nthreads) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
    return omp_get_max_threads();
}

int or_insert(or_graph *g, const uint32_t *src, const uint32_t *dst, const float *w, uint64_t k) {
    return insert_impl(g, src, dst, w, k, !g->directed);
}

int or_insert_directed(or_graph *g, const uint32_t *src, const uint32_t *dst, const float *w, uint64_t k) {
    return insert_impl(g, src, dst, w, k, false);
}

int or_delete(or_graph *g, const uint32_t *src, const uint32_t *dst, uint64_t k) {
    if (!in_range(g, src, dst, k)) return -1;
    std::vector<Entry> e = expand(src, dst, nullptr, k, !g->directed);
    std::sort(e.begin(), e.end(), [](const Entry &a, const Entry &b) {
        return a.s != b.s ? a.s < b.s : a.d < b.d;
    });
    auto gr = groups(e);
#pragma omp parallel for schedule(dynamic, 64)
    for (long gi = 0; gi < (long)gr.size(); ++gi) {
        const uint32_t s = e[gr[gi].first].s;
        std::vector<uint32_t> &a = g->adj[s];
        std::vector<uint32_t> na;
        std::vector<float> nw;
        na.reserve(a.size());
        size_t q = gr[gi].first;
        for (size_t p = 0; p < a.size(); ++p) {
            while (q < gr[gi].second && e[q].d < a[p]) ++q;
            if (q < gr[gi].second && e[q].d == a[p]) continue;  // deleted
            na.push_back(a[p]);
            if (g->weighted) nw.push_back(g->w[s][p]);
        }
        a.swap(na);
        if (g->weighted) g->w[s].swap(nw);
    }
    return 0;
}

uint64_t or_num_edges(const or_graph *g) {
    uint64_t m = 0;
    for (const auto &a : g->adj) m += a.size();
    return m;
}

void or_export(const or_graph *g, uint64_t *offsets, uint32_t *dst, float *w) {
    uint64_t p = 0;
    for (uint32_t u = 0; u < g->n; ++u) {
        offsets[u] = p;
        for (size_t i = 0; i < g->adj[u].size(); ++i) {
            dst[p] = g->adj[u][i];
            if (w) w[p] = g->weighted ? g->w[u][i] : 1.0f;
            ++p;
        }
    }
    offsets[g->n] = p;
}

// One sweep x' = base + alpha * sum_{u->v} x_u / deg(u), pulled per v.
static void pr_sweep(const or_graph *g, const std::vector<uint64_t> *toff, const std::vector<uint32_t> *tsrc,
                     const std::vector<double> &contrib, double alpha, const std::vector<double> &base,
                     std::vector<double> &xn) {
    const long n = g->n;
#pragma omp parallel for schedule(dynamic, 1024)
    for (long v = 0; v < n; ++v) {
        double acc = 0.0;
        if (!g->directed) {
            for (uint32_t u : g->adj[v]) acc += contrib[u];
        } else {
            for (uint64_t i = (*toff)[v]; i < (*toff)[v + 1]; ++i) acc += contrib[(*tsrc)[i]];
        }
        xn[v] = base[v] + alpha * acc;
    }
}

static int pr_generic(const or_graph *g, double alpha, double epsilon, int max_iter, std::vector<double> x,
                      const std::vector<double> &base, int fixed_sweeps, double *x_out) {
    const uint32_t n = g->n;
    std::vector<uint64_t> toff;
    std::vector<uint32_t> tsrc;
    if (g->directed) transpose(g, toff, tsrc, nullptr, nullptr);
    std::vector<double> contrib(n), xn(n);
    int sweeps = 0;
    const int limit = fixed_sweeps > 0 ? fixed_sweeps : max_iter;
    for (int it = 0; it < limit; ++it) {
        for (uint32_t u = 0; u < n; ++u) {
            const size_t d = g->adj[u].size();
            contrib[u] = d ? x[u] / (double)d : 0.0;  // pr_kernel.cu:153 (no dangling redistribution)
        }
        pr_sweep(g, &toff, &tsrc, contrib, alpha, base, xn);
        double diff = 0.0;
#pragma omp parallel for reduction(+ : diff)
        for (long v = 0; v < (long)n; ++v) diff += std::fabs(xn[v] - x[v]);
        x.swap(xn);
        ++sweeps;
        if (fixed_sweeps <= 0 && diff < epsilon) break;  // pagerank.cu:56
    }
    std::memcpy(x_out, x.data(), n * sizeof(double));
    return sweeps;
}

int or_pagerank(const or_graph *g, double alpha, double epsilon, int max_iter, const double *x_init,
                int fixed_sweeps, double *x_out) {
    const uint32_t n = g->n;
    std::vector<double> x(n, 1.0 / n);  // pagerank.cu:17
    if (x_init) std::memcpy(x.data(), x_init, n * sizeof(double));
    std::vector<double> base(n, (1.0 - alpha) / n);  // pagerank.cu:22
    return pr_generic(g, alpha, epsilon, max_iter, x, base, fixed_sweeps, x_out);
}

int or_ppr(const or_graph *g, uint32_t source, double alpha, double epsilon, int max_iter, int fixed_sweeps,
           double *x_out) {
    const uint32_t n = g->n;
    std::vector<double> x(n, 0.0), base(n, 0.0);
    x[source] = 1.0;
    base[source] = 1.0 - alpha;
    return pr_generic(g, alpha, epsilon, max_iter, x, base, fixed_sweeps, x_out);
}

static bool has(const std::vector<uint32_t> &a, uint32_t x) {
    return std::binary_search(a.begin(), a.end(), x);
}

// Symmetric store: every triangle {a, b, c} is found once from its two
// lowest-ranked vertices under the order (degree, id) and credited to its
// smallest id, which is the reference's owner (tc_kernel.cu:25-30).
static uint64_t tc_symmetric(const or_graph *g, uint64_t *per_vertex) {
    const long n = g->n;
    auto less = [&](uint32_t a, uint32_t b) {
        const size_t da = g->adj[a].size(), db = g->adj[b].size();
        return da < db || (da == db && a < b);
    };
    std::vector<std::vector<uint32_t>> out(n);
#pragma omp parallel for schedule(dynamic, 256)
    for (long u = 0; u < n; ++u)
        for (uint32_t v : g->adj[u])
            if (less((uint32_t)u, v)) out[u].push_back(v);  // adj is sorted, so out[u] is sorted
    // per-vertex credits only when asked for (the atomics cost more than the merges)
    std::vector<std::atomic<uint64_t>> cnt(per_vertex ? n : 0);
    for (long u = 0; u < (long)cnt.size(); ++u) cnt[u].store(0, std::memory_order_relaxed);
    uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total)
    for (long u = 0; u < n; ++u) {
        const auto &A = out[u];
        for (uint32_t v : A) {
            const auto &Bv = out[v];
            auto a = A.begin();
            auto b = Bv.begin();
            while (a != A.end() && b != Bv.end()) {
                if (*a < *b) ++a;
                else if (*b < *a) ++b;
                else {
                    if (per_vertex) {
                        const uint32_t o = std::min<uint32_t>(std::min<uint32_t>((uint32_t)u, v), *a);
                        cnt[o].fetch_add(1, std::memory_order_relaxed);
                    }
                    ++total;
                    ++a;
                    ++b;
                }
            }
        }
    }
    if (per_vertex)
        for (long u = 0; u < n; ++u) per_vertex[u] = cnt[u].load();
    return total;
}

uint64_t or_tc(const or_graph *g, uint64_t *per_vertex) {
    if (!g->directed) return tc_symmetric(g, per_vertex);
    const long n = g->n;
    uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total)
    for (long u = 0; u < n; ++u) {
        uint64_t c = 0;
        const auto &Nu = g->adj[u];
        {
            // literal reference formula (tc_kernel.cu:25-65)
            for (uint32_t v : Nu) {
                if (v <= (uint32_t)u) continue;
                for (uint32_t w : g->adj[v])
                    if (w > v && has(g->adj[w], (uint32_t)u)) ++c;
            }
        }
        if (per_vertex) per_vertex[u] = c;
        total += c;
    }
    return total;
}

void or_tc_incident(const or_graph *g, const uint32_t *subset, uint64_t ns, uint64_t *out) {
#pragma omp parallel for schedule(dynamic, 16)
    for (long i = 0; i < (long)ns; ++i) {
        const uint32_t u = subset[i];
        const auto &Nu = g->adj[u];
        uint64_t c = 0;
        for (uint32_t v : Nu) {
            const auto &Nv = g->adj[v];
            auto a = Nu.begin();
            auto b = Nv.begin();
            while (a != Nu.end() && b != Nv.end()) {
                if (*a < *b) ++a;
                else if (*b < *a) ++b;
                else { ++c; ++a; ++b; }
            }
        }
        out[i] = c / 2;
    }
}

static void brandes_one(const or_graph *g, uint32_t s, std::vector<int32_t> &dist, std::vector<uint64_t> &sigma,
                        std::vector<double> &delta, std::vector<uint32_t> &order, double *bc) {
    const uint32_t n = g->n;
    std::fill(dist.begin(), dist.end(), -1);
    std::fill(sigma.begin(), sigma.end(), 0);
    order.clear();
    dist[s] = 0;
    sigma[s] = 1;
    order.push_back(s);
    for (size_t h = 0; h < order.size(); ++h) {
        const uint32_t v = order[h];
        for (uint32_t w : g->adj[v]) {
            if (dist[w] < 0) {
                dist[w] = dist[v] + 1;
                order.push_back(w);
            }
            if (dist[w] == dist[v] + 1) sigma[w] += sigma[v];
        }
    }
    if (!bc) return;
    for (uint32_t v : order) delta[v] = 0.0;
    for (size_t h = order.size(); h-- > 0;) {
        const uint32_t v = order[h];
        double dv = 0.0;
        for (uint32_t w : g->adj[v])
            if (dist[w] == dist[v] + 1) dv += ((double)sigma[v] / (double)sigma[w]) * (1.0 + delta[w]);
        delta[v] = dv;
        if (v != s) bc[v] += dv;
    }
    (void)n;
}

void or_bc(const or_graph *g, const uint32_t *sources, uint64_t ns, double *bc) {
    const uint32_t n = g->n;
    std::vector<uint32_t> all;
    if (!sources || ns == 0) {
        all.resize(n);
        std::iota(all.begin(), all.end(), 0u);
        sources = all.data();
        ns = n;
    }
    std::fill(bc, bc + n, 0.0);
#pragma omp parallel
    {
        std::vector<int32_t> dist(n);
        std::vector<uint64_t> sigma(n);
        std::vector<double> delta(n), local(n, 0.0);
        std::vector<uint32_t> order;
        order.reserve(n);
#pragma omp for schedule(dynamic, 1)
        for (long i = 0; i < (long)ns; ++i) brandes_one(g, sources[i], dist, sigma, delta, order, local.data());
#pragma omp critical
        for (uint32_t v = 0; v < n; ++v) bc[v] += local[v];
    }
}

void or_bfs_sigma(const or_graph *g, uint32_t source, int32_t *dist, uint64_t *sigma) {
    std::vector<int32_t> d(g->n);
    std::vector<uint64_t> s(g->n);
    std::vector<double> delta(g->n);
    std::vector<uint32_t> order;
    brandes_one(g, source, d, s, delta, order, nullptr);
    std::memcpy(dist, d.data(), g->n * sizeof(int32_t));
    std::memcpy(sigma, s.data(), g->n * sizeof(uint64_t));
}

static std::vector<double> row_inverse(const or_graph *g) {
    std::vector<double> r(g->n, 0.0);
    for (uint32_t u = 0; u < g->n; ++u) {
        double s = 0.0;
        for (size_t i = 0; i < g->adj[u].size(); ++i) s += g->weighted ? (double)g->w[u][i] : 1.0;
        r[u] = s > 0 ? 1.0 / s : 0.0;
    }
    return r;
}

static int wpr_forward_impl(const or_graph *g, double alpha, double tol, int max_iter, double *x_out,
                            uint32_t pu, uint32_t pv, double delta) {
    const uint32_t n = g->n;
    // raw weights with an optional perturbation of entry (pu, pv)
    std::vector<std::vector<double>> w(n);
    std::vector<double> rinv(n, 0.0);
    for (uint32_t u = 0; u < n; ++u) {
        w[u].resize(g->adj[u].size());
        double s = 0.0;
        for (size_t i = 0; i < g->adj[u].size(); ++i) {
            double wi = g->weighted ? (double)g->w[u][i] : 1.0;
            if (u == pu && g->adj[u][i] == pv) wi += delta;
            w[u][i] = wi;
            s += wi;
        }
        rinv[u] = s > 0 ? 1.0 / s : 0.0;
    }
    std::vector<uint64_t> toff(n + 1, 0);
    for (uint32_t u = 0; u < n; ++u)
        for (uint32_t v : g->adj[u]) toff[v + 1]++;
    for (uint32_t v = 0; v < n; ++v) toff[v + 1] += toff[v];
    std::vector<uint32_t> tsrc(toff[n]);
    std::vector<double> tw(toff[n]);
    std::vector<uint64_t> cur(toff.begin(), toff.end() - 1);
    for (uint32_t u = 0; u < n; ++u)
        for (size_t i = 0; i < g->adj[u].size(); ++i) {
            const uint64_t p = cur[g->adj[u][i]]++;
            tsrc[p] = u;
            tw[p] = w[u][i] * rinv[u];
        }
    std::vector<double> x(n, 1.0 / n), xn(n);
    const double base = (1.0 - alpha) / n;
    int sweeps = 0;
    for (int it = 0; it < max_iter; ++it) {
        double diff = 0.0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : diff)
        for (long v = 0; v < (long)n; ++v) {
            double acc = 0.0;
            for (uint64_t i = toff[v]; i < toff[v + 1]; ++i) acc += tw[i] * x[tsrc[i]];
            xn[v] = base + alpha * acc;
            diff += std::fabs(xn[v] - x[v]);
        }
        x.swap(xn);
        ++sweeps;
        if (diff < tol) break;
    }
    std::memcpy(x_out, x.data(), n * sizeof(double));
    return sweeps;
}

int or_wpr_forward(const or_graph *g, double alpha, double tol, int max_iter, double *x) {
    return wpr_forward_impl(g, alpha, tol, max_iter, x, UINT32_MAX, UINT32_MAX, 0.0);
}

int or_wpr_adjoint(const or_graph *g, double alpha, double tol, int max_iter, const double *c, double *lambda) {
    const uint32_t n = g->n;
    const std::vector<double> rinv = row_inverse(g);
    std::vector<double> l(c, c + n), ln(n);
    int sweeps = 0;
    for (int it = 0; it < max_iter; ++it) {
        double diff = 0.0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : diff)
        for (long u = 0; u < (long)n; ++u) {
            double acc = 0.0;
            for (size_t i = 0; i < g->adj[u].size(); ++i)
                acc += (g->weighted ? (double)g->w[u][i] : 1.0) * rinv[u] * l[g->adj[u][i]];
            ln[u] = c[u] + alpha * acc;
            diff += std::fabs(ln[u] - l[u]);
        }
        l.swap(ln);
        ++sweeps;
        if (diff < tol) break;
    }
    std::memcpy(lambda, l.data(), n * sizeof(double));
    return sweeps;
}

void or_wpr_gradient(const or_graph *g, double alpha, const double *x, const double *lambda, const double *c,
                     int mode, double *grad) {
    const std::vector<double> rinv = row_inverse(g);
    uint64_t p = 0;
    for (uint32_t u = 0; u < g->n; ++u)
        for (size_t i = 0; i < g->adj[u].size(); ++i) {
            const uint32_t v = g->adj[u][i];
            if (mode == 1) grad[p++] = alpha * x[u] * lambda[v];
            else grad[p++] = x[u] * (alpha * lambda[v] - lambda[u] + c[u]) * rinv[u];
        }
}

double or_wpr_objective(const or_graph *g, double alpha, double tol, int max_iter, const double *c, uint32_t u,
                        uint32_t v, double delta) {
    std::vector<double> x(g->n);
    wpr_forward_impl(g, alpha, tol, max_iter, x.data(), u, v, delta);
    double j = 0.0;
    for (uint32_t i = 0; i < g->n; ++i) j += c[i] * x[i];
    return j;
}

// Central differences (J(w + h e_uv) - J(w - h e_uv)) / 2h of J = sum c_i x_i
// for k raw-weight entries at once.  Changing the raw weight of (u, v) by d
// changes only row u of the normalised matrix, by r(d) q_u with r = d/(s_u+d)
// and q_u[j] = ([j == v] s_u - w_uj) / s_u over u's out-entries.  With
// y = a (I - a T)^-1 q_u (one forward-direction solve per entry, shared by
// both signs) the perturbed solve is exactly
//     x(d) - x0 = r x0[u] y / (1 - r y[u])          (rank-one update),
// so J(d) - J(0) = r x0[u] (c . y) / (1 - r y[u]) is evaluated without
// subtracting two nearly equal objectives and without stopping a perturbed
// solve early.  The k solves share each sweep over the transposed matrix
// (vertex-major rows of k values) and run until every right-hand side's L1
// step is below rel_tol of its norm.  `tol` bounds the base solve's L1 step.
int or_wpr_fd(const or_graph *g, double alpha, double tol, int max_iter, const double *c, const uint32_t *eu,
              const uint32_t *ev, uint32_t k, double h, double *fd) {
    const uint32_t n = g->n;
    if (k == 0) return 0;
    std::vector<uint64_t> toff(n + 1, 0);
    for (uint32_t u = 0; u < n; ++u)
        for (uint32_t v : g->adj[u]) toff[v + 1]++;
    for (uint32_t v = 0; v < n; ++v) toff[v + 1] += toff[v];
    std::vector<uint32_t> tsrc(toff[n]);
    std::vector<double> tw(toff[n]);
    std::vector<uint64_t> cur(toff.begin(), toff.end() - 1);
    const std::vector<double> rinv = row_inverse(g);
    auto raw = [&](uint32_t u, size_t i) { return g->weighted ? (double)g->w[u][i] : 1.0; };
    for (uint32_t u = 0; u < n; ++u)
        for (size_t i = 0; i < g->adj[u].size(); ++i) {
            const uint64_t p = cur[g->adj[u][i]]++;
            tsrc[p] = u;
            tw[p] = raw(u, i) * rinv[u];
        }
    // base solve x0 = (1-a)/n + a T x0
    const double base = (1.0 - alpha) / n;
    std::vector<double> x0(n, 1.0 / n), xn(n);
    int sweeps = 0;
    for (int it = 0; it < max_iter; ++it) {
        double diff = 0.0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : diff)
        for (long v = 0; v < (long)n; ++v) {
            double acc = 0.0;
            for (uint64_t i = toff[v]; i < toff[v + 1]; ++i) acc += tw[i] * x0[tsrc[i]];
            xn[v] = base + alpha * acc;
            diff += std::fabs(xn[v] - x0[v]);
        }
        x0.swap(xn);
        ++sweeps;
        if (diff < tol) break;
    }
    // forcing a q_e, sparse over the out-entries of u_e
    std::vector<double> s_of(k);
    std::vector<std::vector<std::pair<uint32_t, double>>> force(n);
    for (uint32_t e = 0; e < k; ++e) {
        const uint32_t u = eu[e];
        double s = 0.0;
        for (size_t i = 0; i < g->adj[u].size(); ++i) s += raw(u, i);
        s_of[e] = s;
        for (size_t i = 0; i < g->adj[u].size(); ++i) {
            const double q = ((g->adj[u][i] == ev[e] ? s : 0.0) - raw(u, i)) / s;
            force[g->adj[u][i]].push_back({e, alpha * q});
        }
    }
    const double rel_tol = 1e-11;
    std::vector<double> Y((size_t)n * k, 0.0), Yn((size_t)n * k);
    for (uint32_t v = 0; v < n; ++v)
        for (auto &f : force[v]) Y[(size_t)v * k + f.first] = f.second;
    std::vector<double> step(k), norm(k);
    for (int it = 0; it < 4 * max_iter; ++it) {
        std::fill(step.begin(), step.end(), 0.0);
        std::fill(norm.begin(), norm.end(), 0.0);
#pragma omp parallel
        {
            std::vector<double> acc(k), lstep(k, 0.0), lnorm(k, 0.0);
#pragma omp for schedule(dynamic, 512) nowait
            for (long v = 0; v < (long)n; ++v) {
                std::fill(acc.begin(), acc.end(), 0.0);
                for (uint64_t i = toff[v]; i < toff[v + 1]; ++i) {
                    const double t = alpha * tw[i];
                    const double *row = &Y[(size_t)tsrc[i] * k];
                    for (uint32_t j = 0; j < k; ++j) acc[j] += t * row[j];
                }
                for (auto &f : force[v]) acc[f.first] += f.second;
                double *out = &Yn[(size_t)v * k];
                const double *old = &Y[(size_t)v * k];
                for (uint32_t j = 0; j < k; ++j) {
                    lstep[j] += std::fabs(acc[j] - old[j]);
                    lnorm[j] += std::fabs(acc[j]);
                    out[j] = acc[j];
                }
            }
#pragma omp critical
            for (uint32_t j = 0; j < k; ++j) {
                step[j] += lstep[j];
                norm[j] += lnorm[j];
            }
        }
        Y.swap(Yn);
        bool done = true;
        for (uint32_t j = 0; j < k; ++j)
            if (step[j] > rel_tol * norm[j]) done = false;
        if (done) break;
    }
    std::vector<double> cy(k, 0.0);
    for (uint32_t v = 0; v < n; ++v)
        for (uint32_t j = 0; j < k; ++j) cy[j] += c[v] * Y[(size_t)v * k + j];
    for (uint32_t e = 0; e < k; ++e) {
        const uint32_t u = eu[e];
        const double yu = Y[(size_t)u * k + e];
        double dj[2];
        for (int side = 0; side < 2; ++side) {
            const double d = side == 0 ? h : -h;
            const double r = d / (s_of[e] + d);
            dj[side] = r * x0[u] * cy[e] / (1.0 - r * yu);
        }
        fd[e] = (dj[0] - dj[1]) / (2.0 * h);
    }
    return sweeps;
}

void or_uniform_pairs(uint32_t n, uint64_t num_pairs, uint64_t seed, uint32_t *src, uint32_t *dst) {
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)num_pairs; ++i) gv_uniform_pair(n, seed, (uint64_t)i, &src[i], &dst[i]);
}

void or_rmat_pairs(uint32_t scale, uint64_t num_pairs, uint64_t seed, uint32_t *src, uint32_t *dst) {
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)num_pairs; ++i) gv_rmat_pair(seed, (uint64_t)i, scale, &src[i], &dst[i]);
}

}  // extern "C"
