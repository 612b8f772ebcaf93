// sdot_server.cu -- a solve service: requests admitted by device-memory budget,
// solved concurrently on one GPU.
//
// The reference runs one SotSolver::solve at a time per process
// (src/solvers/SotSolver.cc:105-215; SemiDiscreteOT::run_sot drives
// epsilon scaling, SemiDiscreteOT.cc:878-922).  The service keeps a fixed
// number of slots, each a worker thread that owns one library context (its
// own CUDA stream and device buffers, reused across requests).  Requests wait
// in a FIFO queue and are admitted when a slot is free and the device-memory
// estimate of the request fits in the budget next to the requests already
// running; a request that arrives while others run starts as soon as a slot
// and memory free up, and its kernels overlap theirs on the device.  Every
// solve is deterministic (fixed-order reductions), so a request's result does
// not depend on what else is in flight.
//
// Per request: source (flattened quadrature data as sdot_set_source, or
// points only), targets, solver parameters, optional warm start, method
// (Newton with the tensor-core Hessian, or L-BFGS) and epsilon scaling.
#include <float.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "sdot_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b)
{
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Job {
    // request (copied)
    int dim = 0;
    int64_t nq = 0, ncells = 0, nt = 0;
    std::vector<double> x, jxw, density, centers, y, nu, psi;
    std::vector<int64_t> offsets;
    sdot_solver_params prm{};
    int method = SDOT_METHOD_AUTO, precision = SDOT_PREC_HYBRID, hessian_method = SDOT_HESS_AUTO;
    double eps_factor = 10.0, inter_tol = 0.0;
    int eps_steps = 1;
    size_t need = 0;
    // state and result
    enum { QUEUED, RUNNING, DONE } state = QUEUED;
    sdot_result res{};
    Clock::time_point t_submit, t_start, t_end;
};

}  // namespace

struct sdot_server {
    int device = 0;
    int n_slots = 1;
    size_t budget = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<int64_t> queue;
    std::unordered_map<int64_t, Job> jobs;
    int64_t next_ticket = 1;
    size_t in_use = 0, peak_in_use = 0;
    int running = 0, peak_running = 0;
    int64_t completed = 0, failed = 0;
    std::vector<double> latencies;
    bool stop = false;
    std::string err;
    std::vector<std::thread> workers;
    std::vector<sdot_ctx *> ctxs;
};

namespace {

// Device bytes a request may hold while it runs (sources, targets, evaluation
// buffers, solver history, and for Newton the FP32 Hessian with its tile data).
size_t estimate_bytes(const Job &j, bool newton)
{
    const double D = j.dim;
    double b = (double)j.nq * (D + 6.0) * 8.0 + (double)j.ncells * (D + 2.0) * 8.0;
    b += (double)j.nt * (D + 2.0 + sdot::TPACK + 64.0 + 6.0 + 12.0 + 8.0) * 8.0;
    b += 64.0 * 1024 * 1024;  // block-pair lists and small buffers
    if (newton) {
        b += (double)j.nt * (double)j.nt * 4.0;                  // FP32 Hessian
        b += (double)j.nq * 20.0 + 148.0 * 256.0 * 1024.0;       // per-point data, drain scratch
    } else if (j.prm.tau > 0.0) {
        b += 1024.0 * 1024.0 * 1024.0;                           // truncated-path gradient partials
    }
    return (size_t)b;
}

bool untruncated(const sdot_solver_params &p) { return p.tau <= 0.0 && p.threshold_type == SDOT_THRESH_POINTWISE; }

void run_job(sdot_server *s, sdot_ctx *c, Job &j)
{
    sdot_result &r = j.res;
    c->precision = j.precision;
    std::vector<int64_t> offs;
    std::vector<double> ctr;
    const int64_t *po = j.offsets.data();
    const double *pc = j.centers.data();
    int64_t ncells = j.ncells;
    if (ncells == 0) {
        // points only: each point is its own cell (the untruncated path never queries cells)
        ncells = j.nq;
        offs.resize(j.nq + 1);
        for (int64_t q = 0; q <= j.nq; ++q) offs[q] = q;
        po = offs.data();
        pc = j.x.data();
    }
    if (c->dim != j.dim) c->nt = 0;  // the slot's previous targets had another dimension
    sdot_status st = sdot_set_source(c, j.dim, j.nq, j.x.data(), j.jxw.data(), j.density.data(), ncells, po, pc);
    if (st == SDOT_OK) st = sdot_set_target(c, j.nt, j.y.data(), j.nu.data());
    int method = j.method;
    if (method == SDOT_METHOD_AUTO)
        method = (untruncated(j.prm) && c->w_nonneg && j.nt <= 46340) ? SDOT_METHOD_NEWTON : SDOT_METHOD_LBFGS;
    r.method = method;
    // Newton's steps need gradients below the tolerance: its evaluations are
    // FP64 (the reduced precision is in its tensor-core Hessian)
    if (method == SDOT_METHOD_NEWTON) c->precision = SDOT_PREC_FP64;
    const int levels = std::max(1, j.eps_steps);
    const double fac = j.eps_factor > 1.0 ? j.eps_factor : 2.0;
    unsigned iters = 0;
    int64_t evals = 0;
    for (int lev = 0; lev < levels && st == SDOT_OK; ++lev) {
        sdot_solver_params p = j.prm;
        p.epsilon = j.prm.epsilon * std::pow(fac, (double)(levels - 1 - lev));
        if (lev + 1 < levels && j.inter_tol > 0.0) p.tolerance = j.inter_tol;
        if (method == SDOT_METHOD_NEWTON) {
            sdot_newton_info ni{};
            st = sdot_solve_newton(c, j.psi.data(), &p, j.hessian_method, &ni);
            iters += ni.iterations;
            evals += ni.n_evaluations;
            r.last_value = ni.last_value;
            r.last_check_value = ni.last_check_value;
            r.converged = ni.converged;
        } else {
            sdot_solve_info si{};
            st = sdot_solve(c, j.psi.data(), &p, &si);
            iters += si.iterations;
            evals += si.n_evaluations;
            r.last_value = si.last_value;
            r.last_check_value = si.last_check_value;
            r.converged = si.converged;
        }
    }
    r.status = st;
    r.iterations = iters;
    r.n_evaluations = evals;
    if (st != SDOT_OK) {
        r.converged = 0;
        const char *m = sdot_last_error(c);
        strncpy(r.message, m ? m : "", sizeof(r.message) - 1);
        r.message[sizeof(r.message) - 1] = 0;
    }
    // with a budget, give back the per-request Hessian memory
    if (s->budget) {
        c->nt_H32.release();
        c->nt_H64.release();
        c->htc_scr.release();
    }
}

void worker(sdot_server *s, int slot)
{
    sdot_ctx *c = s->ctxs[slot];
    for (;;) {
        int64_t t = 0;
        Job *j = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] {
                if (s->stop) return true;
                if (s->queue.empty()) return false;
                const Job &h = s->jobs.at(s->queue.front());
                return s->budget == 0 || s->in_use + h.need <= s->budget || s->running == 0;
            });
            if (s->stop && s->queue.empty()) return;
            if (s->queue.empty()) continue;
            t = s->queue.front();
            j = &s->jobs.at(t);
            if (!(s->budget == 0 || s->in_use + j->need <= s->budget || s->running == 0)) continue;
            s->queue.pop_front();
            j->state = Job::RUNNING;
            j->t_start = Clock::now();
            s->in_use += j->need;
            s->peak_in_use = std::max(s->peak_in_use, s->in_use);
            ++s->running;
            s->peak_running = std::max(s->peak_running, s->running);
        }
        s->cv_work.notify_all();
        j->res.slot = slot;
        run_job(s, c, *j);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            j->t_end = Clock::now();
            j->res.queue_ms = ms_between(j->t_submit, j->t_start);
            j->res.run_ms = ms_between(j->t_start, j->t_end);
            j->res.latency_ms = ms_between(j->t_submit, j->t_end);
            j->state = Job::DONE;
            s->in_use -= j->need;
            --s->running;
            ++s->completed;
            if (j->res.status != SDOT_OK) ++s->failed;
            s->latencies.push_back(j->res.latency_ms);
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
}

double percentile(std::vector<double> v, double q)
{
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t i = (size_t)pos;
    const double f = pos - (double)i;
    return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

}  // namespace

extern "C" {

sdot_status sdot_server_create(sdot_server **out, int device, int n_slots, size_t memory_budget)
{
    if (!out || n_slots < 1 || n_slots > 64) return SDOT_EINVAL;
    *out = nullptr;
    sdot_server *s = new sdot_server();
    s->device = device;
    s->n_slots = n_slots;
    s->budget = memory_budget;
    for (int i = 0; i < n_slots; ++i) {
        sdot_options o{};
        o.device = device;
        o.precision = SDOT_PREC_HYBRID;
        sdot_ctx *c = nullptr;
        sdot_status st = sdot_create(&c, &o);
        if (st != SDOT_OK) {
            for (sdot_ctx *x : s->ctxs) sdot_destroy(x);
            delete s;
            return st;
        }
        s->ctxs.push_back(c);
    }
    for (int i = 0; i < n_slots; ++i) s->workers.emplace_back(worker, s, i);
    *out = s;
    return SDOT_OK;
}

void sdot_server_destroy(sdot_server *s)
{
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto &t : s->workers) t.join();
    for (sdot_ctx *c : s->ctxs) sdot_destroy(c);
    delete s;
}

const char *sdot_server_last_error(const sdot_server *s) { return s ? s->err.c_str() : "null server"; }

sdot_status sdot_server_submit(sdot_server *s, const sdot_request *q, int64_t *ticket)
{
    if (!s || !q || !ticket) return SDOT_EINVAL;
    if ((q->dim != 2 && q->dim != 3) || q->n_q <= 0 || q->n_t <= 0 || !q->x || !q->jxw || !q->density || !q->y ||
        !q->nu)
        return SDOT_EINVAL;
    if (q->n_cells < 0 || (q->n_cells > 0 && (!q->cell_offsets || !q->cell_centers))) return SDOT_EINVAL;
    if (q->n_cells == 0 && !untruncated(q->params)) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->err = "a request without cells must be untruncated (tau <= 0, pointwise threshold)";
        return SDOT_EINVAL;
    }
    Job j;
    j.dim = q->dim;
    j.nq = q->n_q;
    j.ncells = q->n_cells;
    j.nt = q->n_t;
    j.x.assign(q->x, q->x + q->n_q * q->dim);
    j.jxw.assign(q->jxw, q->jxw + q->n_q);
    j.density.assign(q->density, q->density + q->n_q);
    if (q->n_cells > 0) {
        j.offsets.assign(q->cell_offsets, q->cell_offsets + q->n_cells + 1);
        j.centers.assign(q->cell_centers, q->cell_centers + q->n_cells * q->dim);
    }
    j.y.assign(q->y, q->y + q->n_t * q->dim);
    j.nu.assign(q->nu, q->nu + q->n_t);
    if (q->psi0) j.psi.assign(q->psi0, q->psi0 + q->n_t);
    else j.psi.assign(q->n_t, 0.0);
    j.prm = q->params;
    j.method = q->method;
    j.precision = q->precision;
    j.hessian_method = q->hessian_method;
    j.eps_factor = q->epsilon_scaling_factor;
    j.eps_steps = q->epsilon_scaling_steps;
    j.inter_tol = q->intermediate_tolerance;
    const bool newton = q->method == SDOT_METHOD_NEWTON ||
                        (q->method == SDOT_METHOD_AUTO && untruncated(q->params) && q->n_t <= 46340);
    j.need = estimate_bytes(j, newton);
    j.t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->budget && j.need > s->budget) {
            s->err = "request needs " + std::to_string(j.need) + " device bytes, above the budget of " +
                     std::to_string(s->budget);
            return SDOT_EBUDGET;
        }
        const int64_t t = s->next_ticket++;
        s->jobs.emplace(t, std::move(j));
        s->queue.push_back(t);
        *ticket = t;
    }
    s->cv_work.notify_all();
    return SDOT_OK;
}

int sdot_server_poll(sdot_server *s, int64_t ticket)
{
    if (!s) return -1;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return -1;
    return it->second.state == Job::DONE ? 1 : 0;
}

sdot_status sdot_server_wait(sdot_server *s, int64_t ticket, double timeout_s, double *psi, sdot_result *res)
{
    if (!s) return SDOT_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) {
        s->err = "unknown ticket";
        return SDOT_EINVAL;
    }
    auto done = [&] { return it->second.state == Job::DONE; };
    if (timeout_s > 0) {
        if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done)) return SDOT_ETIMEOUT;
    } else {
        s->cv_done.wait(lk, done);
    }
    Job &j = it->second;
    if (psi) memcpy(psi, j.psi.data(), j.psi.size() * sizeof(double));
    if (res) *res = j.res;
    const sdot_status st = j.res.status;
    s->jobs.erase(it);
    return st;
}

sdot_status sdot_server_get_stats(sdot_server *s, sdot_server_stats *out)
{
    if (!s || !out) return SDOT_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    out->completed = s->completed;
    out->failed = s->failed;
    out->queued = (int64_t)s->queue.size();
    out->running = s->running;
    out->peak_running = s->peak_running;
    out->in_use_bytes = s->in_use;
    out->peak_bytes = s->peak_in_use;
    out->p50_ms = percentile(s->latencies, 0.50);
    out->p99_ms = percentile(s->latencies, 0.99);
    out->mean_ms = s->latencies.empty()
                       ? 0.0
                       : std::accumulate(s->latencies.begin(), s->latencies.end(), 0.0) / (double)s->latencies.size();
    return SDOT_OK;
}

sdot_status sdot_server_reset_stats(sdot_server *s)
{
    if (!s) return SDOT_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    s->latencies.clear();
    s->completed = 0;
    s->failed = 0;
    s->peak_in_use = s->in_use;
    s->peak_running = s->running;
    return SDOT_OK;
}

}  // extern "C"
