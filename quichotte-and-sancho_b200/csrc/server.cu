// server.cu -- a request loop over independent IV-point solves (qs_server_* of qsb200.h).
//
// The reference program solves one voltage after another for one model
// (src/quichotte.f90:125-143). Here requests -- a model, its energy grid and one voltage --
// arrive at any time and are served by continuous batching:
//   * admission by HBM budget: a request is admitted when a worker is free and the
//     estimated device bytes of its solve (qs_estimate_bytes, the allocations of
//     qs_create) fit into what the solves in flight leave of the budget; requests are
//     admitted in arrival order (the head of the queue waits for memory, so a large
//     request is not starved by later small ones);
//   * every admitted solve owns a handle -- its G, Sigma, Broyden history and stream stay
//     on the device until the solve ends -- and runs on its own worker thread, so the
//     kernels of different solves overlap on the device and one solve's host steps hide
//     behind another's kernels;
//   * a finished solve releases its memory (stream-ordered, no device-wide
//     synchronisation) and the next queued request is admitted at once.
// Each solve is the same computation as a stand-alone qs_create + qs_solve_scf (fresh
// start) + qs_current, on a handle of its own, so its result does not depend on what else
// is in flight.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "qs_common.cuh"

namespace {

struct Request {
    int64_t id = 0;
    double V = 0.0, t_arrival = 0.0, gib = 0.0;
    qs_problem p{};
    std::vector<double> H, GL, GR, U, omega;
    std::vector<int> atom_norb, atom_first;
};

}  // namespace

struct qs_server {
    qs_server_config cfg{};
    double budget_gib = 0.0, used_gib = 0.0;
    int inflight = 0;
    bool stop = false;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> queue;
    std::deque<qs_request_result> done;
    std::vector<std::thread> workers;
    std::chrono::steady_clock::time_point t0;
    int64_t n_pending = 0;  // submitted, not yet polled

    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }

    void work() {
        cudaSetDevice(cfg.device);
        for (;;) {
            Request *r = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] {
                    return stop || (!queue.empty() && used_gib + queue.front()->gib <= budget_gib);
                });
                if (queue.empty() || (stop && !(used_gib + queue.front()->gib <= budget_gib))) {
                    if (stop) return;
                    continue;
                }
                r = queue.front();
                queue.pop_front();
                used_gib += r->gib;
                inflight++;
            }
            qs_request_result res{};
            res.id = r->id;
            res.t_arrival = r->t_arrival;
            res.t_start = now();
            res.device_gib = r->gib;
            qs_handle *h = nullptr;
            int rc = qs_create(&r->p, &h);
            if (rc == 0) {
                qs_scf_result sr{};
                rc = qs_solve_scf(h, r->V, 1, &sr);
                if (rc == 0) {
                    res.converged = sr.converged;
                    res.n_iter = sr.n_iter;
                    res.n_mixed = sr.n_mixed;
                    res.fmax = sr.fmax;
                    res.solve_s = sr.seconds;
                    rc = qs_current(h, r->V, &res.J_up, &res.J_down);
                }
            }
            res.status = rc;
            if (rc && h) std::snprintf(res.error, sizeof(res.error), "%s", qs_last_error(h));
            qs_destroy(h);
            res.t_done = now();
            delete r;
            {
                std::lock_guard<std::mutex> lk(mu);
                used_gib -= res.device_gib;
                inflight--;
                done.push_back(res);
            }
            cv_work.notify_all();
            cv_done.notify_all();
        }
    }
};

extern "C" {

int qs_server_create(const qs_server_config *cfg, qs_server **out) {
    *out = nullptr;
    if (!cfg || cfg->max_inflight < 1 || cfg->max_inflight > 64) return -1;
    if (cudaSetDevice(cfg->device) != cudaSuccess) return -1;
    auto *s = new qs_server();
    s->cfg = *cfg;
    size_t freeb = 0, totb = 0;
    if (cudaMemGetInfo(&freeb, &totb) != cudaSuccess) {
        delete s;
        return -1;
    }
    const double free_gib = (double)freeb / (double)(1ull << 30);
    s->budget_gib = cfg->hbm_budget_gib > 0.0 ? std::min(cfg->hbm_budget_gib, 0.95 * free_gib) : 0.9 * free_gib;
    s->t0 = std::chrono::steady_clock::now();
    for (int k = 0; k < cfg->max_inflight; k++) s->workers.emplace_back([s] { s->work(); });
    *out = s;
    return 0;
}

double qs_server_budget_gib(const qs_server *s) { return s ? s->budget_gib : 0.0; }

double qs_server_clock(const qs_server *s) { return s ? s->now() : 0.0; }

int qs_server_submit(qs_server *s, const qs_problem *p, double V, int64_t id) {
    double gib = 0.0;
    int rc = qs_estimate_bytes(p, &gib);
    if (rc) return rc;
    gib += 0.5;  // the headroom qs_create keeps free
    if (gib > s->budget_gib) return QS_ERR_TOO_LARGE;
    auto *r = new Request();
    r->id = id;
    r->V = V;
    r->gib = gib;
    const size_t nn = (size_t)p->Norb * p->Norb;
    r->H.assign(p->H, p->H + 2 * nn);
    r->GL.assign(p->GammaL, p->GammaL + 2 * nn);
    r->GR.assign(p->GammaR, p->GammaR + 2 * nn);
    r->U.assign(p->U_site, p->U_site + p->Norb);
    r->omega.assign(p->omega, p->omega + p->n_omega);
    r->atom_norb.assign(p->atom_norb, p->atom_norb + p->N_atoms);
    r->atom_first.assign(p->atom_first, p->atom_first + p->N_atoms);
    r->p = *p;
    r->p.H = r->H.data();
    r->p.GammaL = r->GL.data();
    r->p.GammaR = r->GR.data();
    r->p.U_site = r->U.data();
    r->p.omega = r->omega.data();
    r->p.atom_norb = r->atom_norb.data();
    r->p.atom_first = r->atom_first.data();
    r->p.device = s->cfg.device;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->t_arrival = s->now();
        s->queue.push_back(r);
        s->n_pending++;
    }
    s->cv_work.notify_all();
    return 0;
}

int qs_server_poll(qs_server *s, qs_request_result *out, int cap, double timeout_s) {
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->done.empty() && timeout_s > 0.0)
        s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return !s->done.empty(); });
    int k = 0;
    while (k < cap && !s->done.empty()) {
        out[k++] = s->done.front();
        s->done.pop_front();
    }
    s->n_pending -= k;
    return k;
}

int qs_server_pending(qs_server *s) {
    std::lock_guard<std::mutex> lk(s->mu);
    return (int)s->n_pending;
}

void qs_server_destroy(qs_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        for (Request *r : s->queue) delete r;  // never admitted
        s->queue.clear();
    }
    s->cv_work.notify_all();
    for (auto &t : s->workers) t.join();
    delete s;
}

}  // extern "C"
