// Request loop over a device-resident graph (see include/gv_serve.h).
//
// One dispatcher (the calling thread) walks the trace in arrival order.  A
// run of arrived update requests becomes one coalesced window, applied once
// every query of the current epoch has finished.  Arrived queries are
// grouped (PPR queries into batched launches of up to ppr_batch, triangle
// subsets into one shared count, one BC per request) and handed to worker
// threads; each worker owns a read-only view of the graph and a stream, so
// groups run concurrently on the device.  A group is admitted when a worker
// is free and its scratch estimate fits the HBM budget.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>
#include "../../include/gv_serve.h"
#include "store.cuh"

namespace gv {
namespace {

using clk = std::chrono::steady_clock;

struct Job {
    uint32_t kind = 0;
    std::vector<uint32_t> reqs;  // request indices
    uint32_t epoch = 0;
    uint32_t group = 0;
    uint64_t mem = 0;
};

struct Server {
    gv_graph *g = nullptr;
    gv_serve_config cfg{};
    const gv_request *reqs = nullptr;
    const uint32_t *qvert = nullptr;
    gv_request_result *res = nullptr;
    const gv_serve_outputs *outs = nullptr;
    clk::time_point t0;
    std::mutex mu;
    std::condition_variable cv;
    std::vector<int> busy;        // per worker
    std::vector<Job> job;         // per worker
    uint64_t inflight_mem = 0;
    uint32_t inflight = 0;
    bool stop = false;
    gv_status first_error = GV_OK;

    double now() const { return std::chrono::duration<double>(clk::now() - t0).count(); }

    uint64_t estimate(uint32_t kind, uint32_t k) const {
        const uint64_t n = g->d.n;
        switch (kind) {
            case GV_REQ_PPR: return 16ull * n * k + 16ull * n;
            case GV_REQ_TC: return 64ull * n + 8ull * g->d.P * g->d.B / 2;
            default: return 256ull * n + 4ull * 32 * n + 40ull * n;  // BC: sigma rows, 32 level masks, lists
        }
    }

    void run_job(gv_graph *view, cudaStream_t s, Job &jb) {
        const uint32_t n = g->d.n;
        const double start = now();
        gv_status st = GV_OK;
        std::vector<uint32_t> sweeps(jb.reqs.size(), 0);
        if (jb.kind == GV_REQ_PPR) {
            std::vector<uint32_t> srcs;
            for (uint32_t r : jb.reqs) srcs.push_back(reqs[r].source);
            const uint32_t k = (uint32_t)srcs.size();
            std::vector<float> x((size_t)n * k);
            int32_t sw = 0;
            st = gv_ppr_batch(view, srcs.data(), k, cfg.alpha, cfg.epsilon, cfg.max_iter, x.data(), &sw, GV_MEM_HOST, s);
            for (uint32_t j = 0; j < k && st == GV_OK; ++j) {
                sweeps[j] = (uint32_t)sw;
                float *out = (outs && outs->ppr) ? outs->ppr[jb.reqs[j]] : nullptr;
                if (out)
                    for (uint32_t v = 0; v < n; ++v) out[v] = x[(size_t)v * k + j];
            }
        } else if (jb.kind == GV_REQ_TC) {
            std::vector<uint32_t> verts;
            for (uint32_t r : jb.reqs) verts.insert(verts.end(), qvert + reqs[r].offset, qvert + reqs[r].offset + reqs[r].count0);
            std::vector<uint64_t> cnt(verts.size());
            st = gv_tc_subset(view, verts.data(), verts.size(), cnt.data(), GV_MEM_HOST, s);
            size_t p = 0;
            for (uint32_t r : jb.reqs) {
                uint64_t *out = (outs && outs->tc) ? outs->tc[r] : nullptr;
                if (out && st == GV_OK) std::memcpy(out, cnt.data() + p, reqs[r].count0 * sizeof(uint64_t));
                p += reqs[r].count0;
            }
        } else {  // BC: one request per job
            const gv_request &q = reqs[jb.reqs[0]];
            std::vector<float> b(n);
            st = gv_bc(view, qvert + q.offset, q.count0, b.data(), GV_MEM_HOST, s);
            float *out = (outs && outs->bc) ? outs->bc[jb.reqs[0]] : nullptr;
            if (out && st == GV_OK) std::memcpy(out, b.data(), (size_t)n * sizeof(float));
        }
        const double done = now();
        for (size_t j = 0; j < jb.reqs.size(); ++j) {
            gv_request_result &rr = res[jb.reqs[j]];
            rr.start_s = start;
            rr.done_s = done;
            rr.latency_ms = (done - reqs[jb.reqs[j]].arrival_s) * 1e3;
            rr.epoch = jb.epoch;
            rr.status = (uint32_t)st;
            rr.sweeps = sweeps[j];
            rr.group = jb.group;
        }
        std::lock_guard<std::mutex> lk(mu);
        if (st != GV_OK && first_error == GV_OK) first_error = st;
    }

    void worker(int w) {
        gv_graph *view = nullptr;
        cudaSetDevice(g->cfg.device);
        cudaStream_t s = nullptr;
        cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        gv_status vs = gv_view_create(g, &view);
        for (;;) {
            Job jb;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return stop || busy[w] == 1; });
                if (busy[w] != 1 && stop) break;
                jb = job[w];
            }
            if (vs == GV_OK) run_job(view, s, jb);
            else {
                std::lock_guard<std::mutex> lk(mu);
                if (first_error == GV_OK) first_error = vs;
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                busy[w] = 0;
                inflight -= 1;
                inflight_mem -= jb.mem;
            }
            cv.notify_all();
        }
        if (view) gv_destroy(view);
        if (s) cudaStreamDestroy(s);
    }
};

}  // namespace
}  // namespace gv

using namespace gv;

extern "C" gv_status gv_serve_config_init(gv_serve_config *cfg) {
    if (!cfg) return GV_ERR_INVALID;
    cfg->slots = 4;
    cfg->ppr_batch = 32;
    cfg->max_coalesce = 64;
    cfg->pace = 1;
    cfg->hbm_budget_bytes = 32ull << 30;
    cfg->alpha = 0.85f;
    cfg->epsilon = 1e-6f;
    cfg->max_iter = 100;
    return GV_OK;
}

extern "C" gv_status gv_serve_trace(gv_graph *g, const gv_serve_config *cfg, const gv_request *reqs, uint32_t nreq,
                                    const uint32_t *src, const uint32_t *dst, const uint32_t *qvert,
                                    gv_request_result *results, const gv_serve_outputs *outs) {
    if (!g || !cfg || (nreq && (!reqs || !results))) { set_error("null argument"); return GV_ERR_INVALID; }
    if (g->parent) { set_error("serve on the graph, not a view"); return GV_ERR_STATE; }
    if (cfg->slots == 0 || cfg->ppr_batch == 0 || cfg->ppr_batch > 32 || cfg->max_coalesce == 0) {
        set_error("bad serve config");
        return GV_ERR_INVALID;
    }
    for (uint32_t i = 0; i < nreq; ++i) {
        if (i && reqs[i].arrival_s < reqs[i - 1].arrival_s) { set_error("requests must be in arrival order"); return GV_ERR_INVALID; }
        if (reqs[i].kind > GV_REQ_BC) { set_error("bad request kind"); return GV_ERR_INVALID; }
        if ((reqs[i].kind == GV_REQ_TC || reqs[i].kind == GV_REQ_BC) && !qvert) { set_error("qvert needed"); return GV_ERR_INVALID; }
        if (reqs[i].kind == GV_REQ_UPDATE && (!src || !dst)) { set_error("src/dst needed"); return GV_ERR_INVALID; }
    }
    std::memset(results, 0, sizeof(gv_request_result) * nreq);
    Server S;
    S.g = g;
    S.cfg = *cfg;
    S.reqs = reqs;
    S.qvert = qvert;
    S.res = results;
    S.outs = outs;
    const uint32_t W = cfg->slots;
    S.busy.assign(W, 0);
    S.job.assign(W, Job{});
    cudaSetDevice(g->cfg.device);
    cudaStream_t us = nullptr;
    cudaStreamCreateWithFlags(&us, cudaStreamNonBlocking);
    std::vector<std::thread> pool;
    S.t0 = clk::now();
    for (uint32_t w = 0; w < W; ++w) pool.emplace_back(&Server::worker, &S, (int)w);

    uint32_t next = 0, epoch = 0, group = 0;
    auto arrived = [&](uint32_t i) { return !cfg->pace || reqs[i].arrival_s <= S.now(); };
    gv_status st = GV_OK;
    while (next < nreq && st == GV_OK) {
        if (!arrived(next)) {
            const double wait = reqs[next].arrival_s - S.now();
            if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.0005)));
            continue;
        }
        if (reqs[next].kind == GV_REQ_UPDATE) {
            uint32_t j = next;
            while (j < nreq && reqs[j].kind == GV_REQ_UPDATE && arrived(j) && j - next < cfg->max_coalesce) ++j;
            {  // the window waits for every query of the current epoch
                std::unique_lock<std::mutex> lk(S.mu);
                S.cv.wait(lk, [&] { return S.inflight == 0; });
            }
            const double start = S.now();
            std::vector<gv_batch_desc> descs;
            const uint64_t base = reqs[next].offset;
            uint64_t p = 0;
            for (uint32_t i = next; i < j; ++i) {
                if (reqs[i].offset != base + p) { set_error("update pairs must follow trace order"); st = GV_ERR_INVALID; break; }
                descs.push_back({p, reqs[i].count0, reqs[i].count1});
                p += (uint64_t)reqs[i].count0 + reqs[i].count1;
            }
            gv_status us_st = GV_OK;
            if (st == GV_OK) {
                us_st = gv_batch_run(g, descs.data(), (uint32_t)descs.size(), src + base, dst + base, GV_MEM_HOST,
                                     GV_BATCH_COMPACT, us);
                if (us_st == GV_OK) us_st = gv_synchronize(g, us);
            }
            const double done = S.now();
            ++group;
            for (uint32_t i = next; i < j; ++i) {
                results[i].start_s = start;
                results[i].done_s = done;
                results[i].latency_ms = (done - reqs[i].arrival_s) * 1e3;
                results[i].epoch = epoch;
                results[i].status = (uint32_t)us_st;
                results[i].group = group;
            }
            epoch += j - next;
            next = j;
            continue;
        }
        // arrived queries of this epoch, in order, until an update or a future arrival
        uint32_t j = next;
        while (j < nreq && reqs[j].kind != GV_REQ_UPDATE && arrived(j)) ++j;
        std::vector<Job> jobs;
        Job ppr, tc;
        ppr.kind = GV_REQ_PPR;
        tc.kind = GV_REQ_TC;
        for (uint32_t i = next; i < j; ++i) {
            if (reqs[i].kind == GV_REQ_PPR) {
                ppr.reqs.push_back(i);
                if (ppr.reqs.size() == cfg->ppr_batch) {
                    jobs.push_back(ppr);
                    ppr.reqs.clear();
                }
            } else if (reqs[i].kind == GV_REQ_TC) {
                tc.reqs.push_back(i);
            } else {
                Job b;
                b.kind = GV_REQ_BC;
                b.reqs.push_back(i);
                jobs.push_back(b);
            }
        }
        if (!ppr.reqs.empty()) jobs.push_back(ppr);
        if (!tc.reqs.empty()) jobs.push_back(tc);
        for (Job &jb : jobs) {
            jb.epoch = epoch;
            jb.group = ++group;
            jb.mem = S.estimate(jb.kind, (uint32_t)jb.reqs.size());
            std::unique_lock<std::mutex> lk(S.mu);
            S.cv.wait(lk, [&] {
                if (S.inflight == 0) return true;  // always admit into an idle device
                if (S.inflight_mem + jb.mem > cfg->hbm_budget_bytes) return false;
                for (uint32_t w = 0; w < W; ++w)
                    if (!S.busy[w]) return true;
                return false;
            });
            for (uint32_t w = 0; w < W; ++w)
                if (!S.busy[w]) {
                    S.job[w] = jb;
                    S.busy[w] = 1;
                    S.inflight += 1;
                    S.inflight_mem += jb.mem;
                    break;
                }
            lk.unlock();
            S.cv.notify_all();
        }
        next = j;
    }
    {
        std::unique_lock<std::mutex> lk(S.mu);
        S.cv.wait(lk, [&] { return S.inflight == 0; });
        S.stop = true;
    }
    S.cv.notify_all();
    for (auto &t : pool) t.join();
    cudaStreamDestroy(us);
    if (st != GV_OK) return st;
    return S.first_error;
}
