// rc_serve.cu -- the request server: continuous batching of eigen-solves on one GPU.
//
// No reference counterpart: the reference solves one problem per call
// (RayleighChebyshevLMCuda::getMinEigenSystem, RayleighChebyshevLMCuda.h:794-819). Here:
//   * submit: a request (operator, rc_solve_params, start block, output buffers) joins a FIFO;
//   * admission: first-fit over the queue while a slot is free and the request's device
//     footprint (its working blocks plus the operator's storage, charged once per operator in
//     use) fits the HBM budget; a request that has waited longer than starvation_ms holds back
//     the requests behind it until it fits;
//   * slots: max_active worker threads, each with its own context (stream, scratch slots from
//     the server's stream-ordered memory pool). A worker runs the ordinary solver (rc_solver.cu)
//     for its request, so the request's subspace, bounds and Ritz state stay resident in the
//     slot until it finishes, and its scratch goes back to the pool afterwards;
//   * batching: every row-major filter application of a running solve is handed to the batcher
//     thread (serve_filter). The batcher waits until every running solve has posted one, or
//     batch_window_us after the first, then launches all posted applications as one batch
//     (rc_batch.cu: one launch per degree step for all of them, replayed from a captured CUDA
//     graph), and each solve's stream waits on the batch's event. Solves that are in their
//     Lanczos or Rayleigh-Ritz phase meanwhile keep running on their own streams, so the filter
//     sweeps of some solves overlap with the dense work of others.
// A solve's arithmetic does not depend on what else is in its batch (rc_batch.cu), so its
// result is the same alone and in the mix.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>
#include "rc_batch.h"
#include "rc_internal.h"

namespace rcb {
rc_status solve(rc_ctx* ctx, rc_op* op, const rc_solve_params& p, const void* v0, double* evals_out, void* evecs_out,
                double* resid_out, rc_solve_info* info);
int64_t rm_leading_dim(int dtype, int prec, int64_t s);
}  // namespace rcb

using rcb::BatchJob;

namespace rcserve {

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

int64_t round_2m(int64_t b) {
    const int64_t m = (int64_t)2 << 20;
    return ((b + m - 1) / m) * m;
}

struct Request {
    int64_t id = 0;
    rc_op* op = nullptr;
    rc_solve_params p{};
    const void* v0 = nullptr;
    double* evals = nullptr;
    void* evecs = nullptr;
    double* resid = nullptr;
    int64_t need = 0;
    std::atomic<int> state{RC_REQ_QUEUED};
    std::atomic<int> cancel{0};
    rc_status status = RC_OK;
    std::string err;
    double t_submit = 0, t_start = 0, t_end = 0;
    int64_t batches = 0;
    int64_t device_bytes = 0;
    rc_solve_info info{};
};

struct PendingJob {
    BatchJob job;
    cudaEvent_t ready = nullptr;
    double t_post = 0;
    bool launched = false;
    rc_status status = RC_OK;
    std::string err;
    cudaEvent_t done = nullptr;
};

struct Server;

struct Worker {
    Server* server = nullptr;
    rc_ctx* ctx = nullptr;
    cudaEvent_t ready = nullptr;
    Request* req = nullptr;
    std::thread th;
};

}  // namespace rcserve

// Per-worker link from a context to its server (rc_ctx::serve).
struct ServeHook {
    rcserve::Server* server;
    rcserve::Worker* worker;
};

namespace rcserve {

struct Server {
    rc_server_params P{};
    int device = 0;
    int sm_count = 148;
    int64_t budget = 0;
    std::mutex mu;
    std::condition_variable cv_work;   // workers: a request is ready
    std::condition_variable cv_batch;  // batcher: jobs posted or solves started/finished
    std::condition_variable cv_done;   // jobs launched, requests finished
    std::deque<Request*> queue;        // submitted, not admitted
    std::deque<Request*> ready;        // admitted, waiting for a worker
    std::map<int64_t, Request*> reqs;
    std::vector<PendingJob*> pending;
    int running = 0;
    int64_t next_id = 1;
    int64_t bytes_in_use = 0, bytes_peak = 0;
    std::map<rc_op*, std::pair<int, int64_t>> op_refs;  // admitted requests using the op, bytes charged
    bool stopping = false;
    std::vector<Worker*> workers;
    std::vector<ServeHook*> hooks;
    std::thread batcher;
    rcb::BatchRunner* runner = nullptr;
    cudaMemPool_t pool = nullptr;
    std::mutex op_mu;  // serialises building FP32 operator copies at submit
    std::string err;
    int64_t submitted = 0, completed = 0, failed = 0, cancelled = 0;
};

// Device bytes one solve of `op` with parameters p holds at its peak (the slots of rc_solver.cu,
// rc_dense.cu, rc_gemm.cu, rc_lanczos.cu and rc_filter.cu, each rounded up to 2 MiB).
int64_t solve_footprint(const rc_op* op, const rc_solve_params& p, int sm_count) {
    const int64_t n = op->n;
    const int64_t esz = op->dtype == RC_COMPLEX128 ? 16 : 8;
    const int64_t ss = std::max<int64_t>(1, std::min<int64_t>(p.subspace_increment + p.buffer_size, n));
    int64_t md = p.eig_count;
    if ((p.mode == 2 || p.mode == 3) && md <= 0) md = n;
    md = std::max<int64_t>(1, std::min<int64_t>(md, n));
    const int64_t sq = std::max(ss, md);
    int64_t t = 4 * round_2m(n * ss * esz) + round_2m(n * md * esz);
    for (int prec : {P64, P32}) {
        const int64_t rm = n * rcb::rm_leading_dim(op->dtype, prec, ss) * (int64_t)elem_bytes(op->dtype, prec);
        if (rm > n * ss * esz) t += 2 * round_2m(rm);
    }
    t += round_2m(8 * sq * sq * esz + sq * 16 + 512);                 // small Rayleigh-Ritz matrices
    t += round_2m((8 * (int64_t)sm_count + 2) * sq * sq * esz);       // Gram partial sums
    t += round_2m(((n + 63) / 64) * sq * 8);                         // residual partial sums
    t += round_2m(3 * n * esz + sq * sq * esz + 4096);                // Lanczos vectors / small QR
    t += round_2m(4 * sq * sq * esz + 1024) + round_2m(2 * (sq + 1) * (sq + 1) * esz + 4096);  // cholqr, Jacobi
    if (op->kind == 2) t += round_2m(n * ss * esz);                   // callback step scratch
    if (rcb::resid_supported(op, ss))                                 // row-major copy of the Ritz vectors
        t += round_2m(n * rcb::rm_leading_dim(op->dtype, P64, ss) * esz);
    if (p.precision == RC_PREC_MIXED && p.mixed_refine == 0 && rcb::rm_corr_supported(op, ss)) {
        // correction filter: the residual block (rc_corr_t / rc_corr2_t) and the coefficient table
        const int64_t ld32 = rcb::corr_leading_dim(op->dtype, ss);
        const int64_t dmax = p.poly_degree_max > 0 ? p.poly_degree_max : 200;
        t += round_2m(n * ld32 * (int64_t)rcb::corr_elem_bytes(op->dtype)) +
             round_2m((dmax + 1) * ld32 * 4 + ld32 * 8 + 512);
    }
    return t;
}

void try_admit(Server* S) {
    int idle = (int)S->workers.size() - S->running - (int)S->ready.size();
    const double now = now_ms();
    for (auto it = S->queue.begin(); it != S->queue.end() && idle > 0;) {
        Request* r = *it;
        auto& ref = S->op_refs[r->op];
        const int64_t op_charge = ref.first == 0 ? r->op->bytes : 0;
        if (S->bytes_in_use + r->need + op_charge <= S->budget) {
            S->bytes_in_use += r->need + op_charge;
            if (ref.first == 0) ref.second = op_charge;
            ref.first++;
            S->bytes_peak = std::max(S->bytes_peak, S->bytes_in_use);
            S->ready.push_back(r);
            it = S->queue.erase(it);
            --idle;
            S->cv_work.notify_one();
        } else {
            if (ref.first == 0) S->op_refs.erase(r->op);
            if (now - r->t_submit > S->P.starvation_ms) break;  // keep the room for it
            ++it;
        }
    }
}

void finish_request(Server* S, Request* r, rc_status st, const std::string& msg) {
    // caller holds S->mu; r was admitted
    S->bytes_in_use -= r->need;
    auto it = S->op_refs.find(r->op);
    if (it != S->op_refs.end() && --it->second.first == 0) {
        S->bytes_in_use -= it->second.second;
        S->op_refs.erase(it);
    }
    r->status = st;
    r->err = msg;
    r->t_end = now_ms();
    if (st == RC_OK) {
        r->state = RC_REQ_DONE;
        S->completed++;
    } else if (st == RC_ERR_CANCELLED) {
        r->state = RC_REQ_CANCELLED;
        S->cancelled++;
    } else {
        r->state = RC_REQ_FAILED;
        S->failed++;
    }
}

void worker_main(Worker* W) {
    Server* S = W->server;
    cudaSetDevice(S->device);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        S->cv_work.wait(lk, [&] { return S->stopping || !S->ready.empty(); });
        if (S->ready.empty()) break;  // stopping
        Request* r = S->ready.front();
        S->ready.pop_front();
        S->running++;
        r->state = RC_REQ_RUNNING;
        r->t_start = now_ms();
        W->req = r;
        lk.unlock();
        S->cv_batch.notify_all();

        rc_status st = RC_OK;
        std::string msg;
        if (r->cancel.load()) {
            st = RC_ERR_CANCELLED;
            msg = "request cancelled";
        } else {
            rc_ctx* c = W->ctx;
            c->cancel = &r->cancel;
            c->err.clear();
            r->info.struct_size = sizeof(rc_solve_info);
            st = rcb::solve(c, r->op, r->p, r->v0, r->evals, r->evecs, r->resid, &r->info);
            if (cudaStreamSynchronize(c->stream) != cudaSuccess && st == RC_OK) {
                st = RC_ERR_CUDA;
                c->err = "stream synchronize after the solve failed";
            }
            msg = st == RC_OK ? std::string() : c->err;
            int64_t held = 0;
            for (auto& b : c->slots) held += (int64_t)b.bytes;
            r->device_bytes = held;
            rc_release_slots(c);
            cudaStreamSynchronize(c->stream);
            c->cancel = nullptr;
        }

        lk.lock();
        W->req = nullptr;
        S->running--;
        finish_request(S, r, st, msg);
        try_admit(S);
        S->cv_done.notify_all();
        S->cv_batch.notify_all();
    }
}

void batcher_main(Server* S) {
    cudaSetDevice(S->device);
    cudaStream_t bs = rcb::batch_runner_stream(S->runner);
    const double window = S->P.batch_window_us * 1e-3;
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        S->cv_batch.wait(lk, [&] {
            return !S->pending.empty() || (S->stopping && S->running == 0 && S->ready.empty());
        });
        if (S->pending.empty()) break;
        const double deadline = S->pending.front()->t_post + window;
        for (;;) {
            if ((int)S->pending.size() >= S->running || (int)S->pending.size() >= rcb::kMaxBatchJobs) break;
            const double left = deadline - now_ms();
            if (left <= 0) break;
            S->cv_batch.wait_for(lk, std::chrono::duration<double, std::milli>(left));
        }
        const size_t take = std::min<size_t>(S->pending.size(), rcb::kMaxBatchJobs);
        std::vector<PendingJob*> batch(S->pending.begin(), S->pending.begin() + take);
        S->pending.erase(S->pending.begin(), S->pending.begin() + take);
        lk.unlock();

        std::vector<BatchJob> jobs;
        jobs.reserve(batch.size());
        rc_status st = RC_OK;
        std::string msg;
        for (PendingJob* pj : batch) {
            jobs.push_back(pj->job);
            if (cudaStreamWaitEvent(bs, pj->ready, 0) != cudaSuccess) {
                st = RC_ERR_CUDA;
                msg = "batcher: waiting for a solve's inputs failed";
            }
        }
        cudaEvent_t done = nullptr;
        if (st == RC_OK) st = rcb::batch_run(S->runner, jobs.data(), (int)jobs.size(), &done, &msg);

        lk.lock();
        for (PendingJob* pj : batch) {
            pj->status = st;
            pj->err = msg;
            pj->done = done;
            pj->launched = true;
        }
        S->cv_done.notify_all();
    }
}

Request* find_req(Server* S, int64_t id) {
    auto it = S->reqs.find(id);
    return it == S->reqs.end() ? nullptr : it->second;
}

}  // namespace rcserve

struct rc_server : rcserve::Server {};

using namespace rcserve;

namespace rcb {

// Post one described filter application to the batcher and wait until its batch is launched;
// the solve's stream then waits for the batch before it reads V.
static rc_status serve_post(rc_ctx* ctx, const BatchJob& job, bool* handled) {
    ServeHook* h = ctx->serve;
    PendingJob pj;
    pj.job = job;
    RC_CU(ctx, cudaEventRecord(h->worker->ready, ctx->stream));
    pj.ready = h->worker->ready;
    Server* S = h->server;
    {
        std::unique_lock<std::mutex> lk(S->mu);
        pj.t_post = now_ms();
        S->pending.push_back(&pj);
        S->cv_batch.notify_all();
        S->cv_done.wait(lk, [&] { return pj.launched; });
        if (h->worker->req) h->worker->req->batches++;
    }
    if (pj.status != RC_OK) return rc_fail(ctx, pj.status, pj.err);
    RC_CU(ctx, cudaStreamWaitEvent(ctx->stream, pj.done, 0));
    *handled = true;
    return RC_OK;
}

rc_status serve_filter(rc_ctx* ctx, rc_op* op, void* V, int64_t ld, int64_t s, int64_t degree, double a, double b,
                       int prec, void* bufA, void* bufB, size_t buf_bytes, bool* handled) {
    *handled = false;
    if (!ctx->serve) return RC_OK;
    BatchJob job;
    if (!batch_job_describe(ctx, op, V, ld, s, degree, a, b, prec, bufA, bufB, buf_bytes, &job)) return RC_OK;
    return serve_post(ctx, job, handled);
}

rc_status serve_filter_corr(rc_ctx* ctx, rc_op* op, double* V, int64_t ldv, int64_t s, int64_t degree, double a,
                            double b, const rc_corr_t* R, const float* sig, const double* coef, void* bufA,
                            void* bufB, bool* handled) {
    *handled = false;
    if (!ctx->serve) return RC_OK;
    BatchJob job;
    if (!batch_job_describe_corr(ctx, op, V, ldv, s, degree, a, b, R, sig, coef, bufA, bufB, &job)) return RC_OK;
    return serve_post(ctx, job, handled);
}

}  // namespace rcb

extern "C" {

void rc_server_params_default(rc_server_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->struct_size = sizeof(*p);
    p->device = 0;
    p->hbm_budget_bytes = 0;
    p->max_active = 16;
    p->batch_window_us = 200.0;
    p->use_graphs = 1;
    p->starvation_ms = 2000.0;
}

static void server_teardown(Server* S) {
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopping = true;
        for (Request* r : S->queue) {
            r->state = RC_REQ_CANCELLED;
            r->status = RC_ERR_CANCELLED;
            r->err = "server destroyed";
            S->cancelled++;
        }
        S->queue.clear();
        for (auto& kv : S->reqs) kv.second->cancel = 1;
    }
    S->cv_work.notify_all();
    S->cv_batch.notify_all();
    for (Worker* W : S->workers)
        if (W->th.joinable()) W->th.join();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        // admitted requests no worker picked up
        for (Request* r : S->ready) finish_request(S, r, RC_ERR_CANCELLED, "server destroyed");
        S->ready.clear();
    }
    S->cv_batch.notify_all();
    if (S->batcher.joinable()) S->batcher.join();
    cudaSetDevice(S->device);
    for (Worker* W : S->workers) {
        if (W->ctx) rc_ctx_destroy(W->ctx);
        if (W->ready) cudaEventDestroy(W->ready);
        delete W;
    }
    S->workers.clear();
    for (ServeHook* h : S->hooks) delete h;
    S->hooks.clear();
    rcb::batch_runner_destroy(S->runner);
    S->runner = nullptr;
    if (S->pool) cudaMemPoolDestroy(S->pool);
    for (auto& kv : S->reqs) delete kv.second;
    S->reqs.clear();
}

rc_status rc_server_create(const rc_server_params* params, rc_server** out) {
    if (!out) return RC_ERR_INVALID;
    *out = nullptr;
    rc_server_params P;
    rc_server_params_default(&P);
    if (params) {
        const size_t sz = params->struct_size ? std::min(params->struct_size, sizeof(P)) : sizeof(P);
        std::memcpy(&P, params, sz);
        P.struct_size = sizeof(P);
    }
    if (P.max_active < 1 || P.max_active > rcb::kMaxBatchJobs || P.batch_window_us < 0 || P.hbm_budget_bytes < 0)
        return RC_ERR_INVALID;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || P.device < 0 || P.device >= count) {
        cudaGetLastError();
        return RC_ERR_INVALID;
    }
    if (cudaSetDevice(P.device) != cudaSuccess) return RC_ERR_CUDA;
    rc_server* S = new (std::nothrow) rc_server();
    if (!S) return RC_ERR_NOMEM;
    S->P = P;
    S->device = P.device;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, P.device) == cudaSuccess) S->sm_count = prop.multiProcessorCount;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
        delete S;
        return RC_ERR_CUDA;
    }
    S->budget = P.hbm_budget_bytes > 0 ? P.hbm_budget_bytes : (int64_t)(0.9 * (double)fr);
    auto fail = [&](rc_status st) {
        server_teardown(S);
        delete S;
        return st;
    };
    cudaMemPoolProps pp;
    std::memset(&pp, 0, sizeof(pp));
    pp.allocType = cudaMemAllocationTypePinned;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = P.device;
    if (cudaMemPoolCreate(&S->pool, &pp) != cudaSuccess) {
        S->pool = nullptr;
        return fail(RC_ERR_CUDA);
    }
    uint64_t keep = UINT64_MAX;  // freed scratch stays in the pool for the next request
    cudaMemPoolSetAttribute(S->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    std::string err;
    if (rcb::batch_runner_create(P.device, S->sm_count, P.use_graphs != 0, &S->runner, &err) != RC_OK)
        return fail(RC_ERR_CUDA);
    for (int i = 0; i < P.max_active; ++i) {
        Worker* W = new Worker();
        W->server = S;
        S->workers.push_back(W);
        if (rc_ctx_create(P.device, &W->ctx) != RC_OK) return fail(RC_ERR_CUDA);
        if (cudaEventCreateWithFlags(&W->ready, cudaEventDisableTiming) != cudaSuccess) return fail(RC_ERR_CUDA);
        ServeHook* h = new ServeHook{S, W};
        S->hooks.push_back(h);
        W->ctx->serve = h;
        W->ctx->pool = S->pool;
    }
    for (Worker* W : S->workers) W->th = std::thread(worker_main, W);
    S->batcher = std::thread(batcher_main, S);
    *out = S;
    return RC_OK;
}

rc_status rc_server_destroy(rc_server* server) {
    if (!server) return RC_OK;
    server_teardown(server);
    delete server;
    return RC_OK;
}

const char* rc_server_last_error(const rc_server* server) { return server ? server->err.c_str() : "null server"; }

rc_status rc_serve_submit(rc_server* S, const rc_op* op_c, const rc_solve_params* params, const void* v0,
                          double* evals_out, void* evecs_out, double* residuals_out, int64_t* request_id) {
    if (!S || !op_c || !params || !request_id) return RC_ERR_INVALID;
    rc_op* op = const_cast<rc_op*>(op_c);
    *request_id = 0;
    if (!op->ctx || op->ctx->device != S->device) {
        std::lock_guard<std::mutex> lk(S->mu);
        S->err = "rc_serve_submit: operator lives on another device";
        return RC_ERR_INVALID;
    }
    rc_solve_params p;
    rc_solve_params_default(&p);
    const size_t sz = params->struct_size ? std::min(params->struct_size, sizeof(p)) : sizeof(p);
    std::memcpy(&p, params, sz);
    p.struct_size = sizeof(p);
    if (p.subspace_increment < 0 || p.buffer_size < 0 || p.subspace_increment + p.buffer_size < 1 ||
        ((p.mode == 0 || p.mode == 1) && p.eig_count < 1)) {
        std::lock_guard<std::mutex> lk(S->mu);
        S->err = "rc_serve_submit: bad eig_count / subspace sizes";
        return RC_ERR_INVALID;
    }
    if (p.precision == RC_PREC_MIXED && op->kind != 2) {
        // the mixed filter's FP32 operator copy is built once here, not by concurrent solves
        std::lock_guard<std::mutex> lk(S->op_mu);
        cudaSetDevice(S->device);
        const rc_status st = rcb::ensure_fp32(op->ctx, op);
        if (st != RC_OK || cudaStreamSynchronize(op->ctx->stream) != cudaSuccess) {
            std::lock_guard<std::mutex> lk2(S->mu);
            S->err = "rc_serve_submit: building the FP32 operator copy failed: " + op->ctx->err;
            return st != RC_OK ? st : RC_ERR_CUDA;
        }
    }
    Request* r = new (std::nothrow) Request();
    if (!r) return RC_ERR_NOMEM;
    r->op = op;
    r->p = p;
    r->v0 = v0;
    r->evals = evals_out;
    r->evecs = evecs_out;
    r->resid = residuals_out;
    r->need = solve_footprint(op, p, S->sm_count);
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stopping) {
        delete r;
        return RC_ERR_CANCELLED;
    }
    if (r->need + op->bytes > S->budget) {
        S->err = "rc_serve_submit: request needs " + std::to_string(r->need + op->bytes) +
                 " device bytes, above the budget of " + std::to_string(S->budget);
        delete r;
        return RC_ERR_NOMEM;
    }
    r->id = S->next_id++;
    r->t_submit = now_ms();
    S->reqs[r->id] = r;
    S->queue.push_back(r);
    S->submitted++;
    try_admit(S);
    *request_id = r->id;
    return RC_OK;
}

rc_status rc_serve_poll(rc_server* S, int64_t id, int* state) {
    if (!S || !state) return RC_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    Request* r = find_req(S, id);
    if (!r) return RC_ERR_INVALID;
    *state = r->state.load();
    return RC_OK;
}

rc_status rc_serve_wait(rc_server* S, int64_t id, double timeout_ms, int* state) {
    if (!S) return RC_ERR_INVALID;
    std::unique_lock<std::mutex> lk(S->mu);
    Request* r = find_req(S, id);
    if (!r) return RC_ERR_INVALID;
    auto finished = [&] { return r->state.load() >= RC_REQ_DONE; };
    if (timeout_ms < 0) {
        S->cv_done.wait(lk, finished);
    } else if (!S->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), finished)) {
        if (state) *state = r->state.load();
        return RC_ERR_NOT_READY;
    }
    if (state) *state = r->state.load();
    return RC_OK;
}

rc_status rc_serve_result(rc_server* S, int64_t id, rc_solve_info* info, rc_request_info* rinfo, char* errbuf,
                          size_t errbuf_len) {
    if (!S) return RC_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    Request* r = find_req(S, id);
    if (!r) return RC_ERR_INVALID;
    const int st = r->state.load();
    if (rinfo) {
        rc_request_info q;
        std::memset(&q, 0, sizeof(q));
        q.struct_size = sizeof(q);
        q.state = st;
        q.status = st >= RC_REQ_DONE ? r->status : RC_ERR_NOT_READY;
        q.queue_ms = r->t_start > 0 ? r->t_start - r->t_submit : 0.0;
        q.run_ms = r->t_end > 0 && r->t_start > 0 ? r->t_end - r->t_start : 0.0;
        q.latency_ms = r->t_end > 0 ? r->t_end - r->t_submit : 0.0;
        q.batches = r->batches;
        q.reserved_bytes = r->need;
        q.device_bytes = r->device_bytes;
        const size_t sz = rinfo->struct_size ? std::min(rinfo->struct_size, sizeof(q)) : sizeof(q);
        std::memcpy(rinfo, &q, sz);
    }
    if (st < RC_REQ_DONE) return RC_ERR_NOT_READY;
    if (info) {
        const size_t sz = info->struct_size ? std::min(info->struct_size, sizeof(rc_solve_info)) : sizeof(rc_solve_info);
        std::memcpy(info, &r->info, sz);
    }
    if (errbuf && errbuf_len > 0) {
        std::strncpy(errbuf, r->err.c_str(), errbuf_len - 1);
        errbuf[errbuf_len - 1] = '\0';
    }
    return r->status;
}

rc_status rc_serve_cancel(rc_server* S, int64_t id) {
    if (!S) return RC_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    Request* r = find_req(S, id);
    if (!r) return RC_ERR_INVALID;
    r->cancel = 1;
    auto it = std::find(S->queue.begin(), S->queue.end(), r);
    if (it != S->queue.end()) {
        S->queue.erase(it);
        r->state = RC_REQ_CANCELLED;
        r->status = RC_ERR_CANCELLED;
        r->err = "request cancelled";
        r->t_end = now_ms();
        S->cancelled++;
        S->cv_done.notify_all();
        try_admit(S);
    }
    return RC_OK;
}

rc_status rc_serve_release(rc_server* S, int64_t id) {
    if (!S) return RC_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return RC_ERR_INVALID;
    if (it->second->state.load() < RC_REQ_DONE) {
        S->err = "rc_serve_release: request still queued or running";
        return RC_ERR_NOT_READY;
    }
    delete it->second;
    S->reqs.erase(it);
    return RC_OK;
}

rc_status rc_server_stats_get(rc_server* S, rc_server_stats* out) {
    if (!S || !out) return RC_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    const rcb::BatchCounters c = rcb::batch_runner_counters(S->runner);
    rc_server_stats q;
    std::memset(&q, 0, sizeof(q));
    q.struct_size = sizeof(q);
    q.submitted = S->submitted;
    q.completed = S->completed;
    q.failed = S->failed;
    q.cancelled = S->cancelled;
    q.queued = (int64_t)S->queue.size();
    q.running = S->running + (int64_t)S->ready.size();
    q.batches = c.batches;
    q.batched_jobs = c.jobs;
    q.max_jobs_in_batch = c.max_jobs;
    q.graph_launches = c.graph_launches;
    q.graphs_built = c.graphs_built;
    q.kernel_launches = c.kernel_launches;
    q.bytes_in_use = S->bytes_in_use;
    q.bytes_peak = S->bytes_peak;
    q.budget = S->budget;
    const size_t sz = out->struct_size ? std::min(out->struct_size, sizeof(q)) : sizeof(q);
    std::memcpy(out, &q, sz);
    return RC_OK;
}

}  // extern "C"
