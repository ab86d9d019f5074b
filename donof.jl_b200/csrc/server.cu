// Native serving of GNOF energy jobs on one GPU (donof_server_*): continuous
// batching behind a thread-safe queue, for hosts that drive the library
// through the C ABI (a Julia process, a C++ service).
//
// A request carries host arrays (H, b, C, gamma) and the energy loop's
// parameters; it is admitted while its device footprint fits the memory budget
// and a worker is free -- first fit in arrival order, the head of the queue
// passed over at most max_bypass times, so a large job is not starved by small
// ones.  Each worker owns a library context (its own CUDA stream), uploads the
// job's b, runs donof_energy (for the mixed precision: the mixed form until
// its gradients are below ten times the thresholds or its energy stops moving
// by more than its rounding, then closing FP64 iterations), writes the
// orbitals and occupations to the request's output arrays and frees the job.
// Jobs of different workers overlap on the device; a small job's persistent
// kernels are limited to a share of the SMs so that several run side by side.
//
// The request's host arrays must stay valid until the job is done (poll/wait).
#include <math.h>
#include <string.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <algorithm>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "kernels.cuh"

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Device bytes a job holds while it runs (upper estimate: RI tensor, bf16
// split, transform scratch of both forms, orbital state).
size_t job_footprint(int nbf, int naux, int nbf5, bool mixed) {
    const double b = 8.0 * nbf * nbf * naux;
    const double nb = (nbf + 63) / 64;
    const double split = mixed ? 4.0 * 64 * nb * nbf * naux : 0.0;
    double scratch = 8.0 * ((double)nbf * nbf5 * naux + 2.0 * nbf5 * nbf5 * naux);
    if (mixed && (nbf > 256 || nbf5 > 64)) {
        const double ldm = (nbf + 7) / 8 * 8, ldq = (nbf5 + 7) / 8 * 8;
        scratch += 4.0 * (ldm * nbf5 * naux + (double)nbf5 * nbf5 * naux + ldq * nbf5 * naux + 148.0 * nbf * nbf5);
    }
    const double small = 8.0 * (4.0 * nbf * nbf + 16.0 * nbf * nbf5) + (32 << 20);
    return (size_t)(b + split + scratch + small);
}

// the reference's initial gamma (src/guess.jl:184-213)
void guess_gamma(const donof_occ_params& q, std::vector<double>& g) {
    const int ndoc = q.nbeta - q.no1, nc = q.ncwo;
    g.assign((size_t)ndoc * nc, 0.0);
    if (q.occ_method == 0) {
        const double v = log(std::max(0.001 / nc, 1e-16)) - log(0.999);
        for (double& x : g) x = v;
        return;
    }
    for (int i = 0; i < ndoc; ++i) g[i] = acos(sqrt(2.0 * 0.999 - 1.0));
    for (int i = 1; i <= ndoc; ++i)
        for (int j = 1; j < nc; ++j) g[ndoc + (ndoc - i) + ndoc * (j - 1)] = asin(sqrt(1.0 / (nc - j + 1)));
}

struct Job {
    unsigned long long ticket;
    donof_request req;
    double* C_out;
    double* n_out;
    size_t bytes;
    donof_result res;
    bool done = false;
    double t_submit = 0.0;
    std::atomic<int> cancel{0};  // set by donof_server_cancel; the energy loop reads it
};

void mark_cancelled(Job* j, double t) {
    j->res.status = DONOF_ERR_STATE;
    snprintf(j->res.error, sizeof(j->res.error), "cancelled");
    j->res.queue_s = t - j->t_submit;
    j->res.latency_s = t - j->t_submit;
    j->done = true;
}

}  // namespace

struct donof_server {
    int device = 0;
    int max_inflight = 1;
    int max_bypass = 4;
    int cta_share = 0;
    size_t budget = 0, used = 0;
    int inflight = 0;
    int waiters = 0;  // callers blocked in donof_server_wait
    int head_bypassed = 0;
    bool closing = false;
    unsigned long long next_ticket = 1;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Job*> queue;                 // waiting, in arrival order
    std::map<unsigned long long, Job*> jobs;  // every job not yet collected
    std::vector<std::thread> workers;

    // first fit in arrival order, bounded bypass of the head (mu held)
    Job* take() {
        if (inflight >= max_inflight) return nullptr;
        for (size_t i = 0; i < queue.size(); ++i) {
            Job* j = queue[i];
            if (used + j->bytes > budget) continue;
            if (i > 0 && head_bypassed >= max_bypass) return nullptr;  // the head waits for memory
            queue.erase(queue.begin() + (long)i);
            head_bypassed = (i > 0) ? head_bypassed + 1 : 0;
            used += j->bytes;
            ++inflight;
            return j;
        }
        return nullptr;
    }
};

namespace {

int run_job(donof_ctx* ctx, int cta_share, Job* j) {
    using donof::energy_run;
    const donof_request& r = j->req;
    donof_energy_params prm = r.params;
    const int nbf = r.nbf, nbf5 = prm.occ.nbf5;
    int prec = r.precision;
    if (prec == DONOF_PREC_AUTO)
        prec = ((double)nbf * nbf5 * r.naux >= DONOF_AUTO_MIXED_MIN_WORK) ? DONOF_PREC_MIXED : DONOF_PREC_FP64;
    const bool small = (double)nbf * nbf5 * r.naux < DONOF_AUTO_MIXED_MIN_WORK;
    DONOF_CHECK(donof_set_cta_limit(ctx, small ? cta_share : 0));
    donof_job* job = nullptr;
    DONOF_CHECK(donof_b_upload(ctx, r.b, nbf, r.naux, prec, &job));
    std::vector<double> gamma;
    if (r.gamma) gamma.assign(r.gamma, r.gamma + (size_t)(prm.occ.nbeta - prm.occ.no1) * prm.occ.ncwo);
    else guess_gamma(prm.occ, gamma);
    memcpy(j->C_out, r.C, sizeof(double) * (size_t)nbf * nbf);
    donof_energy_result er{};
    int s = DONOF_OK;
    if (prec == DONOF_PREC_MIXED) {
        // mixed phase: ten times the thresholds, or until E stops moving by more than its rounding
        donof_energy_params pm = prm;
        pm.threshgorb *= 10.0;
        pm.threshgocc *= 10.0;
        pm.order_subspaces = 0;
        pm.stop_rel_de = 1e-6;
        s = donof_job_set_precision(job, DONOF_PREC_MIXED);
        if (s == DONOF_OK)
            s = energy_run(job, &pm, r.H, j->C_out, gamma.data(), nullptr, nullptr, nullptr, &er, &j->cancel);
        prm.maxloop = pm.maxloop;
        prm.alpha = pm.alpha;
        if (s == DONOF_OK) s = donof_job_set_precision(job, DONOF_PREC_FP64);
    }
    if (s == DONOF_OK)
        s = energy_run(job, &prm, r.H, j->C_out, gamma.data(), j->n_out, nullptr, nullptr, &er, &j->cancel);
    donof_job_free(job);
    if (s != DONOF_OK) return s;
    j->res.E_elec = er.E_elec;
    j->res.E_tot = er.E_elec + r.E_nuc;
    j->res.iterations = er.iterations;
    j->res.converged = er.converged;
    j->res.precision = prec;
    return DONOF_OK;
}

void worker_main(donof_server* S) {
    donof_ctx* ctx = nullptr;
    const int cs = donof_create(S->device, &ctx);
    for (;;) {
        Job* j = nullptr;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_work.wait(lk, [&] { return S->closing || (j = S->take()) != nullptr; });
            if (!j) {
                if (ctx) donof_destroy(ctx);
                return;
            }
        }
        const double t0 = now_s();
        j->res.status = (cs == DONOF_OK) ? run_job(ctx, S->cta_share, j) : cs;
        if (j->res.status != DONOF_OK) {
            const char* msg = (cs == DONOF_OK) ? donof_last_error(ctx) : donof_last_error(nullptr);
            snprintf(j->res.error, sizeof(j->res.error), "%s", msg ? msg : "");
        }
        const double t1 = now_s();
        {
            std::lock_guard<std::mutex> lk(S->mu);
            j->res.queue_s = t0 - j->t_submit;
            j->res.latency_s = t1 - j->t_submit;
            j->done = true;
            S->used -= j->bytes;
            --S->inflight;
        }
        S->cv_done.notify_all();
        S->cv_work.notify_all();
    }
}

}  // namespace

extern "C" {

int donof_server_create(int device, size_t budget_bytes, int max_inflight, donof_server** out) {
    if (!out || max_inflight < 1) return DONOF_ERR_ARG;
    *out = nullptr;
    if (budget_bytes == 0) {
        size_t free_b = 0, total = 0;
        if (cudaSetDevice(device) != cudaSuccess || cudaMemGetInfo(&free_b, &total) != cudaSuccess) {
            donof::set_error(nullptr, "donof_server_create: device %d not available", device);
            return DONOF_ERR_CUDA;
        }
        budget_bytes = (size_t)(0.85 * (double)free_b);
    }
    donof_server* S = new (std::nothrow) donof_server();
    if (!S) return DONOF_ERR_OOM;
    S->device = device;
    S->budget = budget_bytes;
    S->max_inflight = max_inflight;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    // about two small jobs per SM, at least 16 CTAs; one job alone keeps every SM
    S->cta_share = (max_inflight <= 1) ? 0 : std::max(16, (2 * sms + max_inflight - 1) / max_inflight);
    for (int i = 0; i < max_inflight; ++i) S->workers.emplace_back(worker_main, S);
    *out = S;
    return DONOF_OK;
}

int donof_server_submit(donof_server* S, const donof_request* req, double* C_out, double* n_out,
                        unsigned long long* ticket) {
    if (!S || !req || !C_out || !ticket || !req->H || !req->b || !req->C) return DONOF_ERR_ARG;
    const donof_occ_params& q = req->params.occ;
    if (req->nbf <= 0 || req->naux <= 0 || q.nbf5 <= 0 || q.nbf5 > req->nbf || req->params.maxit < 1 ||
        req->params.maxloop < 1 ||
        (req->precision != DONOF_PREC_FP64 && req->precision != DONOF_PREC_MIXED &&
         req->precision != DONOF_PREC_AUTO)) {
        donof::set_error(nullptr, "donof_server_submit: invalid sizes, precision, maxit or maxloop");
        return DONOF_ERR_ARG;
    }
    Job* j = new (std::nothrow) Job();
    if (!j) return DONOF_ERR_OOM;
    j->req = *req;
    j->C_out = C_out;
    j->n_out = n_out;
    const bool mixed = req->precision == DONOF_PREC_MIXED ||
                       (req->precision == DONOF_PREC_AUTO &&
                        (double)req->nbf * q.nbf5 * req->naux >= DONOF_AUTO_MIXED_MIN_WORK);
    j->bytes = job_footprint(req->nbf, req->naux, q.nbf5, mixed);
    j->res = donof_result{};
    j->t_submit = now_s();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->closing) {
            delete j;
            return DONOF_ERR_STATE;
        }
        if (j->bytes > S->budget) {
            delete j;
            donof::set_error(nullptr, "donof_server_submit: the job needs %zu bytes, more than the budget", j->bytes);
            return DONOF_ERR_ARG;
        }
        j->ticket = S->next_ticket++;
        *ticket = j->ticket;
        S->queue.push_back(j);
        S->jobs[j->ticket] = j;
    }
    S->cv_work.notify_all();
    return DONOF_OK;
}

int donof_server_poll(donof_server* S, unsigned long long ticket, donof_result* res, int* done) {
    if (!S || !res || !done) return DONOF_ERR_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->jobs.find(ticket);
    if (it == S->jobs.end()) return DONOF_ERR_ARG;
    *done = it->second->done ? 1 : 0;
    if (*done) {
        *res = it->second->res;
        delete it->second;
        S->jobs.erase(it);
    }
    return DONOF_OK;
}

int donof_server_wait(donof_server* S, unsigned long long ticket, donof_result* res) {
    if (!S || !res) return DONOF_ERR_ARG;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->jobs.find(ticket);
    if (it == S->jobs.end()) return DONOF_ERR_ARG;
    Job* j = it->second;
    ++S->waiters;
    S->cv_done.wait(lk, [&] { return j->done; });
    *res = j->res;
    delete j;
    S->jobs.erase(ticket);
    --S->waiters;
    lk.unlock();
    S->cv_done.notify_all();  // donof_server_destroy waits for the waiters to leave
    return DONOF_OK;
}

int donof_server_cancel(donof_server* S, unsigned long long ticket) {
    if (!S) return DONOF_ERR_ARG;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        auto it = S->jobs.find(ticket);
        if (it == S->jobs.end()) return DONOF_ERR_ARG;
        Job* j = it->second;
        if (j->done) return DONOF_OK;
        auto q = std::find(S->queue.begin(), S->queue.end(), j);
        if (q == S->queue.end()) {  // in flight: the energy loop stops at its next outer iteration
            j->cancel.store(1, std::memory_order_relaxed);
            return DONOF_OK;
        }
        S->queue.erase(q);
        mark_cancelled(j, now_s());
    }
    S->cv_done.notify_all();
    S->cv_work.notify_all();  // the queue's head may have changed
    return DONOF_OK;
}

int donof_server_destroy(donof_server* S) {
    if (!S) return DONOF_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->closing = true;
        const double t = now_s();
        for (Job* j : S->queue) mark_cancelled(j, t);  // not started
        S->queue.clear();
    }
    S->cv_done.notify_all();  // waiters on queued jobs return their cancelled result
    S->cv_work.notify_all();
    for (std::thread& t : S->workers) t.join();  // jobs in flight finish (and notify)
    {
        std::unique_lock<std::mutex> lk(S->mu);
        S->cv_done.wait(lk, [&] { return S->waiters == 0; });
    }
    for (auto& kv : S->jobs) delete kv.second;
    delete S;
    return DONOF_OK;
}

}  // extern "C"
