// Request loop over a device-resident graph (see include/gv_serve.h).
//
// One dispatcher (the calling thread) walks the trace in arrival order.  A
// run of arrived update requests becomes one coalesced window, applied once
// every query of the current epoch has finished.  Arrived queries are
// grouped (PPR queries into batched launches of up to ppr_batch, triangle
// subsets into one shared count per worker, BC requests in pairs that share
// their BFS passes) and handed to worker threads; each worker owns a
// read-only view of the graph and a stream, so groups of one kind run
// concurrently on the device, the kinds taking turns.  A group is admitted
// when a worker is free and its scratch estimate fits the HBM budget.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
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
    // Scratch a worker keeps between jobs: its view's analytics buffers and
    // its result buffer stay allocated for the next job of the same kind, so
    // a job does not end in cudaFree (which waits for the whole device, the
    // other workers' jobs included).  held[w] charges it to the budget (the
    // estimate of the job that left it); it is released when the worker
    // takes a job of another kind, or when an admission needs the room.
    std::vector<gv_graph *> views;
    std::vector<int> held_kind;   // kind of the held scratch, -1: none
    std::vector<uint64_t> held;
    std::vector<int> release;     // the worker frees its scratch before its next job
    uint64_t held_mem = 0;        // sum of held
    uint64_t inflight_mem = 0;
    uint32_t inflight = 0;
    bool stop = false;
    gv_status first_error = GV_OK;
    std::string err;

    double now() const { return std::chrono::duration<double>(clk::now() - t0).count(); }

    uint64_t live_edges = 0;  // stored entries when the queries were grouped

    uint64_t estimate(uint32_t kind, uint32_t k) const {
        const uint64_t n = g->d.n;
        switch (kind) {
            case GV_REQ_PPR: return 20ull * n * k + 16ull * n;  // 4 iterate blocks + the result block
            // the whole-graph path: an oriented snapshot (two words per stored
            // entry), per-vertex arrays and the dense core's rows
            case GV_REQ_TC: return 64ull * n + 8ull * live_edges + (1ull << 30);
            default: return 512ull * n + 8ull * 32 * n + 48ull * n + 12ull * n * k;  // BC: sigma rows, 32 level masks, lists, scores
        }
    }

    // Device buffer of a worker, grown on demand (results stay on the device
    // unless the caller asked for them).
    struct DevBuf {
        void *p = nullptr;
        size_t bytes = 0;
        void *get(size_t want) {
            if (want <= bytes) return p;
            release();
            if (cudaMalloc(&p, want) != cudaSuccess) {
                cudaGetLastError();
                set_error("serving result buffer of " + std::to_string(want) + " B");
                return nullptr;
            }
            bytes = want;
            return p;
        }
        void release() {
            if (p) cudaFree(p);
            p = nullptr;
            bytes = 0;
        }
        ~DevBuf() { release(); }
    };

    void run_job(gv_graph *view, cudaStream_t s, DevBuf &buf, Job &jb) {
        const uint32_t n = g->d.n;
        const double start = now();
        gv_status st = GV_OK;
        cudaError_t e = cudaSuccess;
        std::vector<uint32_t> sweeps(jb.reqs.size(), 0);
        if (jb.kind == GV_REQ_PPR) {
            std::vector<uint32_t> srcs;
            for (uint32_t r : jb.reqs) srcs.push_back(reqs[r].source);
            const uint32_t k = (uint32_t)srcs.size();
            // sources to the device ahead of the vector block (gv_ppr_batch reads
            // them with the same memory kind as the output)
            float *x = (float *)buf.get((size_t)n * k * 4 + 256);  // k <= 32 sources fit in the tail
            int32_t sw = 0;
            if (!x) st = GV_ERR_NOMEM;
            uint32_t *dsrc = x ? (uint32_t *)((char *)x + (size_t)n * k * 4) : nullptr;
            if (st == GV_OK) e = cudaMemcpyAsync(dsrc, srcs.data(), k * 4, cudaMemcpyHostToDevice, s);
            if (st == GV_OK && e != cudaSuccess) st = cuda_status(e, "serve ppr sources");
            // one query: the single-vector sweeps; more: one lane per query
            if (st == GV_OK && k == 1)
                st = gv_ppr(view, srcs[0], cfg.alpha, cfg.epsilon, cfg.max_iter, x, &sw, GV_MEM_DEVICE, s);
            else if (st == GV_OK)
                st = gv_ppr_batch(view, dsrc, k, cfg.alpha, cfg.epsilon, cfg.max_iter, x, &sw, GV_MEM_DEVICE, s);
            for (uint32_t j = 0; j < k && st == GV_OK; ++j) {
                sweeps[j] = (uint32_t)sw;
                float *out = (outs && outs->ppr) ? outs->ppr[jb.reqs[j]] : nullptr;
                // column j of the n x k block
                if (out) e = cudaMemcpy2DAsync(out, 4, x + j, (size_t)k * 4, 4, n, cudaMemcpyDeviceToHost, s);
                if (e != cudaSuccess) st = cuda_status(e, "serve ppr out");
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
        } else {  // BC: up to two requests per job, sharing 64-source passes
            const uint32_t k = (uint32_t)jb.reqs.size();
            std::vector<uint64_t> off{0};
            for (uint32_t r : jb.reqs) off.push_back(off.back() + reqs[r].count0);
            // sources to the device behind the k score rows (gv_bc_multi reads
            // them with the same memory kind as its output)
            const size_t at = ((size_t)n * 4 * k + 255) & ~size_t(255);
            float *b = (float *)buf.get(at + (size_t)off.back() * 4 + 4);
            if (!b) st = GV_ERR_NOMEM;
            uint32_t *dsrc = b ? (uint32_t *)((char *)b + at) : nullptr;
            for (uint32_t j = 0; j < k && st == GV_OK; ++j) {
                const gv_request &q = reqs[jb.reqs[j]];
                if (!q.count0) continue;
                e = cudaMemcpyAsync(dsrc + off[j], qvert + q.offset, (size_t)q.count0 * 4, cudaMemcpyHostToDevice, s);
                if (e != cudaSuccess) st = cuda_status(e, "serve bc sources");
            }
            if (st == GV_OK) st = gv_bc_multi(view, dsrc, off.data(), k, b, GV_MEM_DEVICE, s);
            for (uint32_t j = 0; j < k && st == GV_OK; ++j) {
                float *out = (outs && outs->bc) ? outs->bc[jb.reqs[j]] : nullptr;
                if (!out) continue;
                e = cudaMemcpyAsync(out, b + (size_t)j * n, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, s);
                if (e != cudaSuccess) st = cuda_status(e, "serve bc out");
            }
        }
        if (st == GV_OK) {
            e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) st = cuda_status(e, "serve job");
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
        if (st != GV_OK && first_error == GV_OK) {
            first_error = st;
            err = gv_last_error_string();  // the message lives in this worker thread
        }
    }

    void worker(int w) {
        gv_graph *view = nullptr;
        cudaSetDevice(g->cfg.device);
        cudaStream_t s = nullptr;
        cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        gv_status vs = gv_view_create(g, &view);
        {
            std::lock_guard<std::mutex> lk(mu);
            views[w] = view;
        }
        DevBuf buf;
        for (;;) {
            Job jb;
            bool drop = false, have = false;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return stop || busy[w] == 1 || release[w] != 0; });
                drop = release[w] != 0;
                have = busy[w] == 1;
                if (!have && !drop && stop) break;
                if (have) jb = job[w];
            }
            if (drop && view) {  // another kind's scratch, or the budget wants it back
                release_analytics_scratch(view);
                buf.release();
            }
            if (drop) {
                {
                    std::lock_guard<std::mutex> lk(mu);
                    release[w] = 0;
                }
                cv.notify_all();
            }
            if (!have) continue;
            if (vs == GV_OK) {
                run_job(view, s, buf, jb);
            } else {
                std::lock_guard<std::mutex> lk(mu);
                if (first_error == GV_OK) first_error = vs;
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                busy[w] = 0;
                inflight -= 1;
                inflight_mem -= jb.mem;
                held[w] = jb.mem;
                held_kind[w] = (int)jb.kind;
                held_mem += jb.mem;
            }
            cv.notify_all();
        }
        if (view) gv_destroy(view);
        if (s) cudaStreamDestroy(s);
    }

    // Under mu: the idle worker for job jb, or -1 to wait.  A worker holding
    // scratch of jb's kind is preferred (it reuses it); a worker holding
    // another kind's frees it before the job.  Admitted when the jobs in
    // flight, the scratch held by the other workers and jb fit the budget,
    // or when nothing else runs; short of room, idle workers holding scratch
    // are woken to free it, and the job waits until they have.
    int pick_worker(const Job &jb, uint32_t W) {
        int best = -1;
        for (uint32_t w = 0; w < W; ++w) {
            if (release[w]) return -1;  // a release in progress: its memory is not back yet
            if (busy[w]) continue;
            if (best < 0 || (held_kind[w] == (int)jb.kind && held_kind[best] != (int)jb.kind)) best = (int)w;
        }
        if (best < 0) return -1;
        auto fits = [&](int w) { return inflight_mem + held_mem - held[w] + jb.mem <= cfg.hbm_budget_bytes; };
        if (fits(best)) return best;
        bool asked = false;
        for (uint32_t w = 0; w < W && !fits(best); ++w)
            if (!busy[w] && (int)w != best && held[w]) {
                held_mem -= held[w];
                held[w] = 0;
                held_kind[w] = -1;
                release[w] = 1;
                asked = true;
            }
        if (asked) {
            cv.notify_all();
            return -1;
        }
        return inflight == 0 ? best : -1;  // always admit into an otherwise idle device
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
    cfg->fresh = 1;
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
        if (reqs[i].kind == GV_REQ_PPR && reqs[i].source >= g->d.n) { set_error("PPR source out of range"); return GV_ERR_INVALID; }
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
    S.views.assign(W, nullptr);
    S.held_kind.assign(W, -1);
    S.held.assign(W, 0);
    S.release.assign(W, 0);
    cudaSetDevice(g->cfg.device);
    cudaStream_t us = nullptr;
    cudaStreamCreateWithFlags(&us, cudaStreamNonBlocking);
    std::vector<std::thread> pool;
    S.t0 = clk::now();
    for (uint32_t w = 0; w < W; ++w) pool.emplace_back(&Server::worker, &S, (int)w);

    uint32_t next = 0, epoch = 0, group = 0;
    auto arrived = [&](uint32_t i) { return !cfg->pace || reqs[i].arrival_s <= S.now(); };
    gv_status st = GV_OK;

    // Applies pending updates idx (trace order, contiguous pair ranges) in
    // windows of at most max_coalesce requests, after every query in flight
    // has finished.
    auto apply_updates = [&](const std::vector<uint32_t> &idx) {
        {
            std::unique_lock<std::mutex> lk(S.mu);
            S.cv.wait(lk, [&] { return S.inflight == 0; });
        }
        for (size_t w0 = 0; w0 < idx.size() && st == GV_OK; w0 += cfg->max_coalesce) {
            const size_t w1 = std::min(idx.size(), w0 + cfg->max_coalesce);
            const double start = S.now();
            std::vector<gv_batch_desc> descs;
            const uint64_t base = reqs[idx[w0]].offset;
            uint64_t p = 0;
            for (size_t q = w0; q < w1; ++q) {
                const gv_request &r = reqs[idx[q]];
                if (r.offset != base + p) {
                    set_error("update pairs must be laid out in trace order");
                    st = GV_ERR_INVALID;
                    return;
                }
                descs.push_back({p, r.count0, r.count1});
                p += (uint64_t)r.count0 + r.count1;
            }
            gv_status us_st = gv_batch_run(g, descs.data(), (uint32_t)descs.size(), src + base, dst + base,
                                           GV_MEM_HOST, GV_BATCH_COMPACT, us);
            if (us_st == GV_OK) us_st = gv_synchronize(g, us);
            const double done = S.now();
            ++group;
            for (size_t q = w0; q < w1; ++q) {
                gv_request_result &rr = results[idx[q]];
                rr.start_s = start;
                rr.done_s = done;
                rr.latency_ms = (done - reqs[idx[q]].arrival_s) * 1e3;
                rr.epoch = epoch;
                rr.status = (uint32_t)us_st;
                rr.group = group;
            }
            if (us_st != GV_OK && S.first_error == GV_OK) S.first_error = us_st;
            epoch += (uint32_t)(w1 - w0);
        }
    };

    // Groups queries idx (PPR into batches of at most ppr_batch, triangle
    // subsets into one count, BC in pairs) and hands the groups to free
    // workers as slots and HBM budget allow.
    auto dispatch_queries = [&](const std::vector<uint32_t> &idx) {
        std::vector<Job> jobs;
        Job ppr, tc, bc;
        ppr.kind = GV_REQ_PPR;
        tc.kind = GV_REQ_TC;
        bc.kind = GV_REQ_BC;
        for (uint32_t i : idx) {
            if (reqs[i].kind == GV_REQ_PPR) {
                ppr.reqs.push_back(i);
                if (ppr.reqs.size() == cfg->ppr_batch) {
                    jobs.push_back(ppr);
                    ppr.reqs.clear();
                }
            } else if (reqs[i].kind == GV_REQ_TC) {
                tc.reqs.push_back(i);
            } else {
                bc.reqs.push_back(i);
                if (bc.reqs.size() == 2) {
                    jobs.push_back(bc);
                    bc.reqs.clear();
                }
            }
        }
        if (!bc.reqs.empty()) jobs.push_back(bc);
        if (!ppr.reqs.empty()) jobs.push_back(ppr);
        // triangle subsets: one shared count per worker, the requests dealt
        // round-robin, so every slot takes part in the kind's turn
        const uint32_t ntc = std::min<uint32_t>((uint32_t)tc.reqs.size(), W);
        for (uint32_t j = 0; j < ntc; ++j) {
            Job part;
            part.kind = GV_REQ_TC;
            for (size_t r = j; r < tc.reqs.size(); r += ntc) part.reqs.push_back(tc.reqs[r]);
            jobs.push_back(part);
        }
        // shortest kinds first: the triangle counts and PPR start before the
        // BC passes, which would otherwise hold the slots and the HBM budget
        // while they queue
        std::stable_sort(jobs.begin(), jobs.end(), [](const Job &x, const Job &y) {
            auto rank = [](uint32_t k) { return k == GV_REQ_BC ? 2 : k == GV_REQ_PPR ? 1 : 0; };
            return rank(x.kind) < rank(y.kind);
        });
        if (ntc) {
            Ctl cc{};
            if (read_ctl(g, &cc, us) == GV_OK) S.live_edges = cc.live_edges;
            else S.live_edges = g->d.P * (uint64_t)g->d.B;  // fall back to the pool's capacity
        }
        const uint32_t first_group = group + 1;  // this dispatch's groups
        for (size_t j = 0; j < jobs.size(); ++j) {
            Job &jb = jobs[j];
            jb.epoch = epoch;
            jb.group = ++group;
            jb.mem = S.estimate(jb.kind, (uint32_t)jb.reqs.size());
            if (j && jobs[j - 1].kind != jb.kind) {
                // Each kind of the dispatch takes its turn: beside one another
                // the kinds ran several times slower (at scale 25 the triangle
                // count and PPR took 1.3 to 2.2 s beside BC passes, against
                // about 0.3 s each alone), which held every result back.
                // Groups of earlier dispatches keep running (their turn was
                // then), so arrivals do not queue behind them.
                std::unique_lock<std::mutex> lk(S.mu);
                S.cv.wait(lk, [&] {
                    for (uint32_t w = 0; w < W; ++w)
                        if (S.busy[w] && S.job[w].group >= first_group) return false;
                    return true;
                });
                if (S.inflight == 0) {
                    // The device is idle: the workers free the previous kinds'
                    // scratch now, while their cudaFree waits for nothing
                    // (later, it would wait for the new kind's groups).
                    for (uint32_t w = 0; w < W; ++w)
                        if (S.held[w] && S.held_kind[w] != (int)jb.kind) {
                            S.held_mem -= S.held[w];
                            S.held[w] = 0;
                            S.held_kind[w] = -1;
                            S.release[w] = 1;
                        }
                    S.cv.notify_all();
                    S.cv.wait(lk, [&] {
                        for (uint32_t w = 0; w < W; ++w)
                            if (S.release[w]) return false;
                        return true;
                    });
                }
            }
            std::unique_lock<std::mutex> lk(S.mu);
            int w = -1;
            S.cv.wait(lk, [&] { return (w = S.pick_worker(jb, W)) >= 0; });
            if (S.held_kind[w] != (int)jb.kind && S.held_kind[w] >= 0) S.release[w] = 1;
            S.held_mem -= S.held[w];
            S.held[w] = 0;
            S.held_kind[w] = -1;
            S.job[w] = jb;
            S.busy[w] = 1;
            S.inflight += 1;
            S.inflight_mem += jb.mem;
            lk.unlock();
            S.cv.notify_all();
        }
    };

    std::vector<uint32_t> pend_u, pend_q;  // arrived, not yet issued (trace order)
    while ((next < nreq || !pend_u.empty() || !pend_q.empty()) && st == GV_OK) {
        for (; next < nreq && arrived(next); ++next) {
            if (reqs[next].kind == GV_REQ_UPDATE) pend_u.push_back(next);
            else pend_q.push_back(next);
        }
        if (pend_u.empty() && pend_q.empty()) {
            const double wait = reqs[next].arrival_s - S.now();
            if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.0005)));
            continue;
        }
        // queries that arrived before the first pending update run on the current epoch
        const uint32_t first_u = pend_u.empty() ? nreq : pend_u.front();
        std::vector<uint32_t> now_q, later_q;
        for (uint32_t i : pend_q) (i < first_u ? now_q : later_q).push_back(i);
        if (!now_q.empty()) dispatch_queries(now_q);
        pend_q.swap(later_q);
        if (pend_u.empty()) continue;
        if (cfg->fresh) {
            // every arrived update, then every arrived query: a query sees at
            // least the updates that arrived before it
            apply_updates(pend_u);
            pend_u.clear();
            if (!pend_q.empty()) dispatch_queries(pend_q);
            pend_q.clear();
        } else {
            // the updates up to the next pending query, as one run
            const uint32_t first_q = pend_q.empty() ? nreq : pend_q.front();
            std::vector<uint32_t> run, rest;
            for (uint32_t i : pend_u) (i < first_q ? run : rest).push_back(i);
            apply_updates(run);
            pend_u.swap(rest);
        }
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
    if (S.first_error != GV_OK) set_error(S.err);
    return S.first_error;
}
