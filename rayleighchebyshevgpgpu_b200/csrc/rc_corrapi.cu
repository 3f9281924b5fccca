// rc_corrapi.cu -- kernel-level entry points of the correction filter (the MIXED refinement).
//
// The reference's filter (LanczosCpolyOperatorLMCuda::apply, LanczosCpolyOperatorLMCuda.h:194-265)
// applied to Ritz pairs (v_c, lam_c) and rewritten as x_k = c_k(lam_c) v_c + a e_k, where e_k
// carries the residual block R = A V - V diag(lam) as a source term (rc_filter_rm.cu). These entry
// points run exactly the solver's steps on a caller's block: R from the residual kernel
// (rc_resid.cu, stored as rc_corr_t, or rc_corr2_t for complex operators), the coefficient tables
// (corr_coefficients), the degree steps (rm_step_src_kernel, or batch_corr_step_kernel for several
// real blocks in one launch per step), and the FP64 combination coef v + a e_m/(m+1) in the
// column-major block.
#include <algorithm>
#include <string>
#include <vector>
#include "rc_batch.h"
#include "rc_common.cuh"
#include "rc_internal.h"

namespace {

constexpr size_t kAlign = 256;
inline size_t up(size_t b) { return (b + kAlign - 1) / kAlign * kAlign; }

// Device memory of one application: Ritz values, coefficient tables, R and the two recurrence blocks.
struct CorrLayout {
    size_t lam = 0, tab = 0, R = 0, A = 0, B = 0, total = 0;
};
CorrLayout corr_layout(int dtype, int64_t n, int64_t s, int64_t degree) {
    const int64_t ld = rcb::corr_leading_dim(dtype, s);
    const size_t blk = up((size_t)n * ld * rcb::corr_elem_bytes(dtype));
    CorrLayout L;
    L.lam = 0;
    L.tab = up((size_t)ld * sizeof(double));
    L.R = L.tab + up(rcb::corr_table_bytes(degree, ld));
    L.A = L.R + blk;
    L.B = L.A + blk;
    L.total = L.B + blk;
    return L;
}

rc_status check_job(rc_ctx* ctx, const rc_op* op, const void* V, int64_t ld, int64_t s, const double* lam,
                    int64_t degree) {
    if (!op || !V || !lam || s < 1 || degree < 1 || ld < op->n)
        return rc_fail(ctx, RC_ERR_INVALID, "correction filter: bad arguments");
    if (op->ctx != ctx) return rc_fail(ctx, RC_ERR_INVALID, "correction filter: operator of another context");
    if (!rcb::rm_corr_supported(op, s) || !rcb::resid_supported(op, s))
        return rc_fail(ctx, RC_ERR_UNSUPPORTED,
                       "correction filter: CSR or 5/7-point stencil operators (27-point: real only) with s <= 256 only");
    return RC_OK;
}

// R (row-major, the correction filter's storage) = A V - V diag(lam) for the column-major FP64 (c128)
// block V, through the row-major copy in slot S_YRM.
rc_status residual_block(rc_ctx* ctx, rc_op* op, const void* V, int64_t ldv, int64_t s, const double* lam_dev,
                         void* R) {
    const int64_t n = op->n;
    const int64_t ldrm = rcb::rm_leading_dim(op->dtype, P64, s);
    void* yrm = nullptr;
    RC_TRY(rc_slot(ctx, S_YRM, (size_t)n * ldrm * elem_bytes(op->dtype, P64), &yrm));
    RC_TRY(rcb::to_row_major(ctx, op->dtype, n, s, V, ldv, yrm, ldrm));
    return rcb::resid_block(ctx, op, yrm, ldrm, s, lam_dev, 0, nullptr, R, rcb::corr_leading_dim(op->dtype, s));
}

}  // namespace

extern "C" {

rc_status rc_filter_correction(rc_ctx* ctx, const rc_op* op_c, void* V, int64_t ld, int64_t s, const double* lam,
                               int64_t degree, double gamma1, double gamma2) {
    if (!ctx) return RC_ERR_INVALID;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return rc_fail(ctx, RC_ERR_CUDA, "cudaSetDevice failed");
    rc_op* op = const_cast<rc_op*>(op_c);
    RC_TRY(check_job(ctx, op, V, ld, s, lam, degree));
    RC_TRY(rcb::ensure_fp32(ctx, op));
    const CorrLayout L = corr_layout(op->dtype, op->n, s, degree);
    void* arena = nullptr;
    RC_TRY(rc_slot(ctx, S_BATCH, L.total, &arena));
    char* base = (char*)arena;
    double* lam_dev = (double*)(base + L.lam);
    void* R = base + L.R;
    RC_CU(ctx, cudaMemcpyAsync(lam_dev, lam, (size_t)s * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    RC_TRY(residual_block(ctx, op, V, ld, s, lam_dev, R));
    RC_TRY(rcb::rm_filter_corr(ctx, op, V, ld, s, degree, gamma2 * gamma1, gamma2, lam_dev, R, base + L.A,
                               base + L.B));
    // lam may be pageable host memory: the copy above has read it once the stream reaches it
    RC_CU(ctx, cudaStreamSynchronize(ctx->stream));
    return RC_OK;
}

rc_status rc_filter_correction_batch(rc_ctx* ctx, int njobs, const rc_correction_job* jobs, int* batched) {
    if (!ctx) return RC_ERR_INVALID;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return rc_fail(ctx, RC_ERR_CUDA, "cudaSetDevice failed");
    if (batched) *batched = 0;
    if (njobs < 1 || njobs > rcb::kMaxBatchJobs || !jobs)
        return rc_fail(ctx, RC_ERR_INVALID, "rc_filter_correction_batch: njobs must be in [1, 64]");
    std::vector<CorrLayout> lay(njobs);
    std::vector<size_t> at(njobs);
    size_t total = 0;
    for (int j = 0; j < njobs; ++j) {
        const rc_correction_job& J = jobs[j];
        if (J.struct_size != 0 && J.struct_size != sizeof(rc_correction_job))
            return rc_fail(ctx, RC_ERR_INVALID, "rc_filter_correction_batch: bad struct_size");
        rc_op* op = const_cast<rc_op*>(J.op);
        RC_TRY(check_job(ctx, op, J.V, J.ld, J.s, J.lam, J.degree));
        for (int i = 0; i < j; ++i)
            if (jobs[i].V == J.V) return rc_fail(ctx, RC_ERR_INVALID, "rc_filter_correction_batch: blocks alias");
        RC_TRY(rcb::ensure_fp32(ctx, op));
        lay[j] = corr_layout(op->dtype, op->n, J.s, J.degree);
        at[j] = total;
        total += lay[j].total;
    }
    void* arena = nullptr;
    RC_TRY(rc_slot(ctx, S_BATCH, total, &arena));
    char* base = (char*)arena;
    // residual blocks and coefficient tables of every job, in order on the context stream
    std::vector<rcb::BatchJob> bj;
    std::vector<int> single;
    for (int j = 0; j < njobs; ++j) {
        const rc_correction_job& J = jobs[j];
        rc_op* op = const_cast<rc_op*>(J.op);
        char* b = base + at[j];
        const int64_t ld = rcb::corr_leading_dim(op->dtype, J.s);
        double* lam_dev = (double*)(b + lay[j].lam);
        float* sig = (float*)(b + lay[j].tab);
        double* coef = (double*)(b + lay[j].tab + rcb::corr_table_coef_offset(J.degree, ld));
        void* R = b + lay[j].R;
        const double a = J.gamma2 * J.gamma1, bb = J.gamma2;
        RC_CU(ctx, cudaMemcpyAsync(lam_dev, J.lam, (size_t)J.s * sizeof(double), cudaMemcpyHostToDevice,
                                   ctx->stream));
        RC_TRY(residual_block(ctx, op, J.V, J.ld, J.s, lam_dev, R));
        RC_TRY(rcb::corr_coefficients(ctx, J.s, ld, J.degree, a, bb, lam_dev, sig, coef));
        rcb::BatchJob d;
        if (op->dtype == RC_REAL64 &&
            rcb::batch_job_describe_corr(ctx, op, (double*)J.V, J.ld, J.s, J.degree, a, bb, (const rc_corr_t*)R,
                                         sig, coef, b + lay[j].A, b + lay[j].B, &d))
            bj.push_back(d);
        else
            single.push_back(j);
    }
    // jobs the batched kernels do not take (complex operators, the 27-point stencil, 64-bit offsets) run as the
    // request server runs them: the single-solve kernels on the context stream
    for (int j : single) {
        const rc_correction_job& J = jobs[j];
        rc_op* op = const_cast<rc_op*>(J.op);
        char* b = base + at[j];
        RC_TRY(rcb::rm_filter_corr(ctx, op, J.V, J.ld, J.s, J.degree, J.gamma2 * J.gamma1, J.gamma2,
                                   (const double*)(b + lay[j].lam), b + lay[j].R, b + lay[j].A, b + lay[j].B));
    }
    if (!bj.empty()) {
        rcb::BatchRunner* runner = nullptr;
        std::string err;
        if (rcb::batch_runner_create(ctx->device, ctx->sm_count, false, &runner, &err) != RC_OK)
            return rc_fail(ctx, RC_ERR_CUDA, err);
        cudaEvent_t ready = nullptr;
        cudaEvent_t done = nullptr;
        rc_status st = RC_OK;
        if (cudaEventCreateWithFlags(&ready, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventRecord(ready, ctx->stream) != cudaSuccess ||
            cudaStreamWaitEvent(rcb::batch_runner_stream(runner), ready, 0) != cudaSuccess) {
            st = rc_fail(ctx, RC_ERR_CUDA, "rc_filter_correction_batch: stream ordering failed");
        } else if (rcb::batch_run(runner, bj.data(), (int)bj.size(), &done, &err) != RC_OK) {
            st = rc_fail(ctx, RC_ERR_CUDA, err);
        } else if (cudaStreamWaitEvent(ctx->stream, done, 0) != cudaSuccess) {
            st = rc_fail(ctx, RC_ERR_CUDA, "rc_filter_correction_batch: stream ordering failed");
        } else {
            ctx->launches += rcb::batch_runner_counters(runner).kernel_launches;
        }
        rcb::batch_runner_destroy(runner);  // waits for the batch
        if (ready) cudaEventDestroy(ready);
        if (st != RC_OK) return st;
    }
    RC_CU(ctx, cudaStreamSynchronize(ctx->stream));
    if (batched) *batched = (int)bj.size();
    return RC_OK;
}

}  // extern "C"
