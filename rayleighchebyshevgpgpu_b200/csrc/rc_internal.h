// rc_internal.h -- context/operator structs and kernel launchers shared by the library sources.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <atomic>
#include <string>
#include <vector>
#include "../../include/rc_b200.h"

// Storage/compute precision of a block: FP64 (double / c128) or FP32 (float / c64).
enum { P64 = 0, P32 = 1 };

// Storage of the correction filter's residual block R and recurrence blocks e_k: bfloat16
// (default) or FP32 (RC_CORR_BF16=0); the arithmetic is FP32 either way. e_k is of the size of the
// residual, so the 8-bit mantissa perturbs the filtered vectors by about 2^-9 of a residual-sized
// term, and the error keeps shrinking with the residual: on the 128^3 7-point and 256^3 27-point
// workloads the solves take the same inner iterations as with FP32 storage, with eigenvalues
// equal to a few units in the 15th digit.
#ifndef RC_CORR_BF16
#define RC_CORR_BF16 1
#endif
// Complex Hermitian operators store real and imaginary parts that way (rc_corr2_t).
#if RC_CORR_BF16
typedef __nv_bfloat16 rc_corr_t;
typedef __nv_bfloat162 rc_corr2_t;
#else
typedef float rc_corr_t;
typedef float2 rc_corr2_t;
#endif
// Widest block of the correction filter and of the residual-block kernel.
constexpr int64_t kCorrMaxCols = 256;

struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
};

struct rc_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    std::string err;
    int64_t launches = 0;
    int64_t op_bytes = 0;
    // grow-only scratch slots, indexed by the Slot enum
    std::vector<DevBuf> slots;
    // pinned host staging for small read-backs
    double* host_small = nullptr;
    size_t host_small_bytes = 0;
    int sm_count = 148;
    size_t smem_optin = 232448;
    // operators created on this context; rc_ctx_destroy releases the ones still alive
    std::vector<struct rc_op*> ops;
    // CSR step kernel: 0 auto (register-cached rows when every row has <= 8 entries),
    // 1 row loop, 2 register-cached rows. Read from RCB200_CSR_KERNEL at context creation.
    int csr_variant = 0;
    // Column-major operator steps and residual blocks (W = A V, R = A Y - Y diag(lam)): columns per
    // chunk (0 = all) and chunk order (0: chunk index slowest, one sweep down the rows per chunk;
    // 1: chunk index fastest). RCB200_CM_CPT, RCB200_CM_ORDER.
    int cm_cpt = 0;
    int cm_order = 0;
    // L2 prefetch distance (rows) of the row-major filter steps; 0 = off. RCB200_PF_ROWS.
    int64_t pf_rows = 0;
    // 16-byte slices per thread in the row-major filter steps: 0 = by storage precision (two
    // for FP32, one for FP64), else 1 or 2. RCB200_RM_SLICES.
    int rm_slices = 0;
    // consecutive row groups per CTA in the row-major filter steps: 0 = by operator kind and
    // storage precision, else 1..64. RCB200_RM_GROUPS.
    int rm_groups = 0;
    // 27-point steps with a warp's lanes on consecutive rows (rm_step27w_kernel) for narrow rows: 1,
    // or 0 (default: the per-thread runs, measured 1.7 % faster on the configuration-5 filter phase,
    // 3792-3803 ms against 3856-3864 ms), from RCB200_ROWS27W.
    int rows27w = 0;
    // Degree steps with their operands staged in shared memory (rc_staged.cuh) for
    // stencil-structured operators: 1, or 0 (default: the per-row gather kernels, measured faster
    // on the 128^3 workloads), from RCB200_STAGED.
    int staged = 0;
    // CTAs of the Jacobi eigensolve when its working copies live in global memory (0 = 32; 1 = the
    // one-CTA kernel), from RCB200_JACOBI_CTAS.
    int jacobi_ctas = 0;
    // Threads of the one-CTA Jacobi kernel (0 = 1024), from RCB200_JACOBI_THREADS; jacobi_sweeps is
    // the number of sweeps the last rc_small_eigh call ran.
    int jacobi_threads = 0;
    // Complex Hermitian Gram products (m <= 192) on the FP64 tensor pipe (gram_c): 1 (default), or 0
    // for the FP64 SIMT kernel, from RCB200_GRAM_C.
    int gram_c = 1;
    int64_t jacobi_sweeps = 0;
    // Rayleigh-Ritz of the correction filter's output on row-major blocks (the filtered block and
    // W = A V formed row-major, no transposes): 1 (default) or 0, from RCB200_RM_RR.
    int rm_rr = 1;
    // Correction-filter degree steps two per launch (rm_corr2_kernel): 1, or 0 (default: one step per
    // launch, measured faster on the 128^3 CSR workload and equal on the stencil form), from
    // RCB200_CORR_PAIR; pair_launches counts those launches.
    int corr_pair = 0;
    int64_t pair_launches = 0;
    int64_t staged_launches = 0;
    // staged step shape: rows per chunk (multiple of 4) and pipeline stages; 0 = the largest that
    // fit. RCB200_STAGED_ROWS, RCB200_STAGED_STAGES.
    int staged_rows = 0;
    int staged_stages = 0;
    // CUDA-event pairs around the degree-step loops of the row-major filter (no transposes),
    // recorded while step_timing is set; step_flush() waits for them and adds to step_ms.
    bool step_timing = false;
    std::vector<cudaEvent_t> step_events;
    size_t step_events_used = 0;
    double step_ms = 0.0;
    // Request-server hooks, null outside the server (rc_serve.cu): filter applications go to the
    // server's batcher, the solver checks the cancel flag once per inner iteration, and scratch
    // slots come from the server's stream-ordered memory pool and go back to it after a request.
    struct ServeHook* serve = nullptr;
    const std::atomic<int>* cancel = nullptr;
    cudaMemPool_t pool = nullptr;
};

enum Slot {
    S_V = 0, S_W, S_T1, S_T2, S_FOUND, S_PART, S_SMALL, S_LANCZOS, S_RPART, S_IO, S_CB, S_EIG, S_FA, S_FB,
    S_R32, S_CORR, S_YRM, S_BATCH, S_VFRM, S_WRM, S_PAIR, S_COUNT
};

struct rc_op {
    rc_ctx* ctx = nullptr;
    int dtype = RC_REAL64;
    int kind = 0;  // 0 CSR, 1 stencil, 2 callback
    int64_t n = 0;
    // CSR
    int64_t nnz = 0;
    int64_t max_row_nnz = 0;
    int64_t band = 0;  // max over entries of (column - row): distance to the farthest later neighbour
    // distinct column offsets (column - row) of all entries, ascending, when there are at most
    // kMaxOffsets of them (a stencil-structured matrix); n_offsets = -1 otherwise
    static constexpr int kMaxOffsets = 32;
    int n_offsets = -1;
    int64_t offsets[kMaxOffsets] = {};
    int32_t* rowptr = nullptr;
    int32_t* colind = nullptr;
    void* vals64 = nullptr;
    void* vals32 = nullptr;  // built lazily for the mixed-precision filter
    // stencil
    int skind = 7;
    int64_t nx = 1, ny = 1, nz = 1;
    double* diag64 = nullptr;
    float* diag32 = nullptr;
    double offdiag = 0.0;
    double flux = 0.0;
    // complex stencils: the Peierls phase exp(i 2 pi flux x) for x = 0..nx-1, as double2 and
    // float2, so the kernels look it up instead of evaluating sincos per row
    void* phase64 = nullptr;
    void* phase32 = nullptr;
    // callback
    rc_block_apply_fn fn = nullptr;
    void* user = nullptr;
    int64_t bytes = 0;
};

// Set the context error and return the status.
rc_status rc_fail(rc_ctx* ctx, rc_status st, const std::string& msg);
#define RC_CU(ctx, call)                                                                       \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return rc_fail((ctx), RC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)
#define RC_TRY(call)                   \
    do {                               \
        rc_status s_ = (call);         \
        if (s_ != RC_OK) return s_;    \
    } while (0)

// Allow `kernel` the device's largest dynamic shared memory. The attribute is process-wide state
// of the function: every caller sets the same value, so concurrent solves (request-server
// workers) never shrink it under one another's launches.
template <class K>
cudaError_t allow_max_smem(const rc_ctx* ctx, K kernel) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(ctx->smem_optin - fa.sharedSizeBytes));
}

// Scratch slot of at least `bytes` (contents not preserved on growth).
rc_status rc_slot(rc_ctx* ctx, int slot, size_t bytes, void** out);
// Free every scratch slot (stream-ordered when the context has a memory pool).
void rc_release_slots(rc_ctx* ctx);
rc_status rc_host_small(rc_ctx* ctx, size_t bytes, double** out);
inline size_t elem_bytes(int dtype, int prec) {
    return (dtype == RC_COMPLEX128 ? 2 : 1) * (prec == P64 ? 8 : 4);
}

namespace rcb {

// ---- operator steps: y = scale*(alpha*(A x) + beta*x + gamma*z) -----------------------
// x, z, y are n x s column-major; z may be null; y may alias z (not x).
struct StepArgs {
    const void* x = nullptr; int xp = P64; int64_t ldx = 0;
    const void* z = nullptr; int zp = P64; int64_t ldz = 0;
    void* y = nullptr; int yp = P64; int64_t ldy = 0;
    int64_t s = 0;
    double alpha[2] = {1, 0}, beta[2] = {0, 0}, gamma[2] = {0, 0};
    double scale = 1.0;
    int cp = P64;  // compute precision (P32: float/c64 accumulation with FP32 matrix values)
};
rc_status op_step(rc_ctx* ctx, rc_op* op, const StepArgs& a);

// Filter X <- P_m(A')X (in place on V, FP64/c128 in and out) with the step
// x_k = a*A*x_{k-1} + b*x_{k-1} - x_{k-2} (a = gamma2*gamma1, b = gamma2). tmp: one n x s FP64
// block of scratch (holds two FP32 blocks in MIXED).
rc_status filter_apply(rc_ctx* ctx, rc_op* op, void* V, int64_t ld, int64_t s, int64_t degree,
                       int64_t rep, double a, double b, int prec, void* tmp1, void* tmp2, size_t tmp_bytes,
                       int64_t* steps_done);
// Inside the request server: hand a row-major filter application to the server's batcher and
// make ctx->stream wait for its batch. *handled = false when the application needs the
// single-solve path (rc_serve.cu).
rc_status serve_filter(rc_ctx* ctx, rc_op* op, void* V, int64_t ld, int64_t s, int64_t degree, double a, double b,
                       int prec, void* bufA, void* bufB, size_t buf_bytes, bool* handled);
// The same for a correction-filter application (rm_filter_corr, after corr_coef_kernel).
rc_status serve_filter_corr(rc_ctx* ctx, rc_op* op, double* V, int64_t ldv, int64_t s, int64_t degree, double a,
                            double b, const rc_corr_t* R, const float* sig, const double* coef, void* bufA,
                            void* bufB, bool* handled);
// Correction filter (rc_filter_rm.cu), the MIXED precision refinement: V (FP64 / c128 column-major,
// leading dimension ldv) holds Ritz vectors with Ritz values lam_dev (device) and R (row-major
// rc_corr_t, or rc_corr2_t for complex operators, leading dimension corr_leading_dim(dtype, s))
// their residual block A V - V diag(lam); V <- P_m(A')V with bfloat16 (or FP32) storage of the
// (small) deviation from the scalar recurrence. bufA and bufB: two row-major blocks of the same
// size as R.
bool rm_corr_supported(const rc_op* op, int64_t s);
// With Vf (real operators, not under the request server): the result goes to the row-major FP64 block
// Vf (leading dimension ldf, even) instead of V, formed from Yrm, the row-major copy of V (leading
// dimension ldy), and V is left unchanged.
rc_status rm_filter_corr(rc_ctx* ctx, rc_op* op, void* V, int64_t ldv, int64_t s, int64_t degree, double a,
                         double b, const double* lam_dev, const void* R, void* bufA, void* bufB,
                         const double* Yrm = nullptr, int64_t ldy = 0, double* Vf = nullptr, int64_t ldf = 0);
int64_t rm_leading_dim(int dtype, int prec, int64_t s);
// Leading dimension (elements) and element bytes of the correction filter's row-major blocks.
inline int64_t corr_leading_dim(int dtype, int64_t s) { return rm_leading_dim(dtype, P32, s); }
inline size_t corr_elem_bytes(int dtype) { return dtype == RC_COMPLEX128 ? sizeof(rc_corr2_t) : sizeof(rc_corr_t); }
// One degree step y = alpha A x + beta x + gamma z on row-major blocks (leading dimension ld, a
// multiple of 32 bytes of elements), storage and arithmetic by prec (RC_PREC_FP64 / RC_PREC_MIXED);
// alpha, beta, gamma are (re, im) pairs, z may be null. The filter's own step kernels.
rc_status rm_step(rc_ctx* ctx, rc_op* op, const void* x, const void* z, void* y, int64_t ld, int64_t s,
                  const double* alpha, const double* beta, const double* gamma, int prec);
// Tables of a correction-filter application of degree m over rows of leading dimension ld: the
// source coefficients sig[k*ld + c] = c_{k-1}(lam_c) (FP32, k = 2..m) and the weights
// coef[c] = c_m(lam_c)/(m+1) (FP64) of the Ritz vectors in the result, written by
// corr_coefficients from the device Ritz values lam_dev (one launch on ctx->stream).
inline size_t corr_table_coef_offset(int64_t degree, int64_t ld) {
    return (((size_t)(degree + 1) * ld * sizeof(float) + 255) / 256) * 256;
}
inline size_t corr_table_bytes(int64_t degree, int64_t ld) {
    return corr_table_coef_offset(degree, ld) + (size_t)ld * sizeof(double) + 256;
}
rc_status corr_coefficients(rc_ctx* ctx, int64_t s, int64_t ld, int64_t degree, double a, double b,
                            const double* lam_dev, float* sig, double* coef);
// Row-major FP64 (c128 for RC_COMPLEX128) copy Yrm (leading dimension ld) of the column-major n x s
// block V.
rc_status to_row_major(rc_ctx* ctx, int dtype, int64_t n, int64_t s, const void* V, int64_t ldv, void* Yrm,
                       int64_t ld);
// The reverse: column-major V (leading dimension ldv) from the row-major Yrm (leading dimension ld).
rc_status to_col_major(rc_ctx* ctx, int dtype, int64_t n, int64_t s, const void* Yrm, int64_t ld, void* V,
                       int64_t ldv);
// Build the FP32 (c64) copy of an operator's values/diagonal used by the MIXED filter.
rc_status ensure_fp32(rc_ctx* ctx, rc_op* op);
// Degree-step timing (ctx->step_timing): record an event on the context stream; step_flush
// waits for the recorded pairs and adds their elapsed time to ctx->step_ms.
void step_mark(rc_ctx* ctx);
void step_flush(rc_ctx* ctx);

// ---- dense FP64 kernels (T = double or double2) ------------------------------------
// C (m x nc, ld m) = X^H Y where X is n x m, Y is n x nc. upper: only i<=j computed then mirrored
// (requires m == nc and a Hermitian result). part: scratch for per-chunk partial sums.
rc_status gram(rc_ctx* ctx, int dtype, int64_t n, int64_t m, int64_t nc, const void* X, int64_t ldx,
               const void* Y, int64_t ldy, void* C, bool upper);
// Y (n x nc) = beta*Y + alpha * X (n x k) * T (k x nc, ld ldt). Y must not alias X.
// Optional dual: X2 * T (stored in Y2 unless Y2 is null) and residual norms
// ||(X2 T)_c - lam_c Y_c|| for c < res_count.
struct XtArgs {
    int64_t n = 0, k = 0, nc = 0;
    const void* X = nullptr; int64_t ldx = 0;
    const void* T = nullptr; int64_t ldt = 0;
    void* Y = nullptr; int64_t ldy = 0;
    double alpha = 1.0;
    double beta = 0.0;
    const void* X2 = nullptr; int64_t ldx2 = 0;
    void* Y2 = nullptr; int64_t ldy2 = 0;
    const double* lam = nullptr; int64_t res_count = 0;
    double* res = nullptr;  // device output, res_count residual norms
    // optional: the residual block X2 T - Y diag(lam) (all nc columns) in row-major FP32 with
    // leading dimension ldr (real blocks with k, nc <= 96 only)
    float* R32 = nullptr; int64_t ldr = 0;
    // optional: a row-major FP64 copy of Y (plain products, real blocks with k, nc <= 96)
    double* Yrm = nullptr; int64_t ldyr = 0;
};
rc_status xt(rc_ctx* ctx, int dtype, const XtArgs& a);

// FP64 real fast paths (s <= 96), rc_gemm.cu. gram2: C0 = X^T Y0 (and C1 = X^T Y1 when Y1),
// symmetric results. xt2: Y = X T, plus residual norms of W T against lam when W is given, and
// the residual block W T - Y diag(lam) in row-major FP32 when R32 is given.
bool gram2_supported(int dtype, int64_t m);
// Complex Hermitian Gram C = X^H Y (m x m, m <= 192, column-major, upper formed and mirrored) on the
// FP64 tensor pipe.
bool gram_c_supported(int dtype, int64_t m);
rc_status gram_c(rc_ctx* ctx, int64_t n, int64_t m, const double2* X, int64_t ldx, const double2* Y, int64_t ldy,
                 double2* C);
rc_status gram2(rc_ctx* ctx, int64_t n, int64_t m, const double* X, int64_t ldx, const double* Y0, int64_t ldy0,
                double* C0, const double* Y1, int64_t ldy1, double* C1, bool rm = false);
bool xt2_supported(int dtype, int64_t k, int64_t nc);
// Y = X T with X row-major (leading dimension ldx): Y column-major and, with Yrm, row-major.
rc_status xt2_rm(rc_ctx* ctx, int64_t n, int64_t k, int64_t nc, const double* X, int64_t ldx, const double* T,
                 int64_t ldt, double* Y, int64_t ldy, double* Yrm, int64_t ldyr);
rc_status xt2(rc_ctx* ctx, int64_t n, int64_t k, int64_t nc, const double* X, int64_t ldx, const double* T,
              int64_t ldt, double* Y, int64_t ldy, const double* W, int64_t ldw, const double* lam, int64_t res_count,
              double* res, float* R32 = nullptr, int64_t ldr = 0, double* Yrm = nullptr, int64_t ldyr = 0);

// Residual block of Ritz vectors on native operators (rc_resid.cu; real, or complex CSR and 5/7-point
// stencils; s <= kCorrMaxCols): R = A Y - Y diag(lam) from the row-major FP64 (c128) copy Yrm of Y
// (leading dimension rm_leading_dim(dtype, P64, s)), its column norms ||R_c|| for c < res_count into
// res (device), and with R the row-major copy of R in the correction filter's storage (rc_corr_t or
// rc_corr2_t, leading dimension corr_leading_dim(dtype, s)). One pass over Yrm.
bool resid_supported(const rc_op* op, int64_t s);
rc_status resid_block(rc_ctx* ctx, const rc_op* op, const void* Yrm, int64_t ld, int64_t s, const double* lam,
                      int64_t res_count, double* res, void* R, int64_t ldr);

// Cholesky factor of Gram G (s x s) with diagonal scaling, shift on breakdown;
// writes Tout = D^-1 R^-1 (upper). flags (device int[4]): [0] shifted, [1] failed, [2] zero column.
// pivout (device, optional): smallest pivot of the scaled Cholesky (1 = orthonormal columns).
rc_status chol_factor(rc_ctx* ctx, int dtype, int64_t s, int64_t nrows, const void* G, void* Tout,
                      int* flags, double* pivout);
// Hermitian eigensolve (parallel Jacobi, one CTA). A (s x s) is read only; evals ascending.
rc_status small_eigh(rc_ctx* ctx, int dtype, int64_t s, void* A, void* Q, double* evals, int* info);
// Same with caller-provided work memory (small_eigh_work_bytes(...) bytes, 0 when the working
// copies fit in shared memory; 256-byte aligned).
size_t small_eigh_work_bytes(rc_ctx* ctx, int dtype, int64_t s);
rc_status small_eigh_work(rc_ctx* ctx, int dtype, int64_t s, void* A, void* Q, double* evals, int* info, void* work);
// C = op(A) B for s x s matrices (op = conjugate transpose when transA), and C <- (C + C^H)/2.
rc_status small_gemm(rc_ctx* ctx, int dtype, int64_t s, const void* A, bool transA, const void* B, void* C);
rc_status hermitize(rc_ctx* ctx, int dtype, int64_t s, void* C);

// Elementwise helpers.
rc_status fill_random(rc_ctx* ctx, int dtype, void* X, int64_t ld, int64_t n, int64_t c0, int64_t c1,
                      uint64_t seed);
rc_status copy_cols(rc_ctx* ctx, int dtype, const void* X, int64_t ldx, void* Y, int64_t ldy, int64_t n,
                    int64_t s);
// y = a*x + b*y (real coefficients), n x s blocks.
rc_status axpby(rc_ctx* ctx, int dtype, double a, const void* X, int64_t ldx, double b, void* Y,
                int64_t ldy, int64_t n, int64_t s);

// ---- Lanczos -------------------------------------------------------------------------
struct LanczosResult {
    double lmin = 0, lmax = 0;
    int64_t iters = 0;
};
rc_status lanczos_bounds(rc_ctx* ctx, rc_op* op, const void* v0_host, uint64_t seed, double tol, int which,
                         int64_t max_iter, LanczosResult* res);

// ---- cholqr over a block (uses ctx slots S_PART, S_SMALL) ---------------------------
rc_status cholqr(rc_ctx* ctx, int dtype, void* V, int64_t ld, int64_t n, int64_t s, void* tmp, bool* swapped,
                 int* passes);

}  // namespace rcb
