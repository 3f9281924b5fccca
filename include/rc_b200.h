/*
 * rc_b200.h -- C ABI of the B200-native Rayleigh-Chebyshev eigensolver.
 *
 * Every entry point returns an rc_status (0 = success) and never terminates the process;
 * the reference instead calls exit() from its error macros (cudaErrchk.h:8-51).
 * The last error message of a context is available from rc_ctx_last_error().
 *
 * Dense blocks ("n x s blocks") are column-major with a leading dimension ld >= n, the
 * layout of AmatrixClassLMCuda<T>::mData / mData_d (AmatrixClassLMCuda.h:333-341).
 * Scalars of a complex problem are interleaved (re, im) pairs of double, the layout of
 * std::complex<double>. Unless a call says otherwise, block pointers are DEVICE pointers
 * on the context's device, owned by the caller.
 *
 * All work is issued on the context's stream (rc_ctx_set_stream), in order.
 */
#ifndef RC_B200_H_
#define RC_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RC_B200_ABI_VERSION 1

typedef int rc_status;
enum {
    RC_OK = 0,
    RC_ERR_INVALID = 1,        /* bad argument (null pointer, size, dtype, ...) */
    RC_ERR_CUDA = 2,           /* a CUDA runtime call failed */
    RC_ERR_NOMEM = 3,          /* device allocation failed or HBM budget exceeded */
    RC_ERR_NOT_HERMITIAN = 4,  /* operator failed the Hermitian check (LanczosMaxMinFinder.h:350-356) */
    RC_ERR_BREAKDOWN = 5,      /* orthonormalisation could not build a basis (RayleighChebyshevLMCuda.h:1110-1113) */
    RC_ERR_TIMEOUT = 6,        /* a bounded device wait gave up */
    RC_ERR_CANCELLED = 7,      /* a served request was cancelled */
    RC_ERR_UNSUPPORTED = 8,    /* valid request this build does not implement */
    RC_ERR_CALLBACK = 9,       /* a user callback returned non-zero */
    RC_ERR_NOT_READY = 10      /* served request still running */
};

/* Problem scalar type: RayleighChebyshevLMCuda's Dtype (RayleighChebyshevLMCuda.h:220). */
enum { RC_REAL64 = 0, RC_COMPLEX128 = 1 };

/* Arithmetic of the Chebyshev filter. FP64: everything in double (c128).
 * MIXED: filter recurrence stored and accumulated in float (c64), orthonormalisation,
 * Rayleigh-Ritz, residuals and the stop test in double, then closing FP64 filter sweeps
 * until the requested residual tolerance is met. (No reference counterpart.) */
enum { RC_PREC_FP64 = 0, RC_PREC_MIXED = 1 };

/* RC_Types::StopCondition (RC_Types.h:33-38). DEFAULT behaves as COMBINATION. */
enum { RC_STOP_DEFAULT = 0, RC_STOP_COMBINATION = 1, RC_STOP_EIGENVALUE_ONLY = 2, RC_STOP_RESIDUAL_ONLY = 3 };

/* Stencil kinds for rc_op_stencil_create. */
enum { RC_STENCIL_5PT_2D = 5, RC_STENCIL_7PT_3D = 7, RC_STENCIL_27PT_3D = 27 };

typedef struct rc_ctx rc_ctx;
typedef struct rc_op rc_op;

/* ------------------------------------------------------------------------------------
 * Context: device, stream, workspace arena, error string, launch counter.
 * Replaces the handle/workspace members of RayleighChebyshevLMCuda
 * (RayleighChebyshevLMCuda.h:2444-2471) and their set-up (:904-911).
 * ------------------------------------------------------------------------------------ */
rc_status rc_ctx_create(int device, rc_ctx** out);
/* Releases the context and every operator still alive on it (their handles become invalid). */
rc_status rc_ctx_destroy(rc_ctx* ctx);
const char* rc_ctx_last_error(const rc_ctx* ctx);
/* stream: a cudaStream_t, or NULL for the context's own non-blocking stream (the legacy default
 * stream cannot be selected: events recorded there do not order against the context's work). */
rc_status rc_ctx_set_stream(rc_ctx* ctx, void* stream);
rc_status rc_ctx_synchronize(rc_ctx* ctx);
/* Number of kernels this library launched through ctx since creation (or last reset). */
rc_status rc_ctx_launch_count(rc_ctx* ctx, int64_t* launches, int reset);
/* A named counter of ctx since creation: "launches" (as rc_ctx_launch_count), "staged_launches"
 * (degree steps that ran with their operands staged in shared memory by asynchronous copies),
 * "pair_launches" (launches that ran two correction-filter degree steps in one pass),
 * "jacobi_sweeps" (Jacobi sweeps of the last rc_small_eigh call). */
rc_status rc_ctx_counter(rc_ctx* ctx, const char* name, int64_t* value);
/* Device bytes currently held by ctx (workspaces + operators created on it). */
rc_status rc_ctx_device_bytes(rc_ctx* ctx, int64_t* bytes);
int rc_abi_version(void);

/* ------------------------------------------------------------------------------------
 * Operators. The reference leaves the operator to the user (Otype, contract at
 * RayleighChebyshevLMCuda.h:70-94 and LanczosMaxMinFinder.h:10-28) and calls its device
 * block apply out = alpha*A*in + beta*out (LanczosCpolyOperatorLMCuda.h:236,245;
 * RayleighChebyshevLMCuda.h:2135,2235). Native operators below let the fused filter
 * see the matrix structure; the callback operator keeps any foreign Otype usable.
 * ------------------------------------------------------------------------------------ */

/* CSR matrix (Hermitian). rowptr: n+1 int32, colind: nnz int32, vals: nnz scalars of dtype.
 * Arrays are HOST pointers and are copied to the device; the operator keeps an FP64 (c128)
 * copy and builds an FP32 (c64) copy the first time a mixed-precision filter needs it. */
rc_status rc_op_csr_create(rc_ctx* ctx, int dtype, int64_t n, int64_t nnz, const int32_t* rowptr,
                           const int32_t* colind, const void* vals, rc_op** out);

/* Matrix-free stencil with Dirichlet boundaries on an nx*ny*nz grid (nz = 1 for 5-point),
 * row index i = x + nx*(y + ny*z):
 *   (A v)_i = diag[i]*v_i + offdiag * sum_{neighbours j} phase(i,j) * v_j
 * diag: n HOST doubles (copied). For RC_COMPLEX128, bonds along y carry the Peierls
 * phase exp(+i*2*pi*flux*x) on the entry (x,y+1,z)<-(x,y,z) and its conjugate on the
 * reverse entry (Landau gauge, uniform flux along z); flux is ignored for RC_REAL64. */
rc_status rc_op_stencil_create(rc_ctx* ctx, int dtype, int kind, int64_t nx, int64_t ny, int64_t nz,
                               const double* diag, double offdiag, double flux, rc_op** out);

/* Foreign operator. fn must compute out = alpha*A*in + beta*out on DEVICE column-major
 * n x s blocks with leading dimension ld, in the scalar type of dtype, ordered on
 * `stream` (a cudaStream_t). alpha/beta point to (re, im) pairs (im = 0 for real).
 * Return 0 on success. */
typedef int (*rc_block_apply_fn)(void* user, const void* in, void* out, int64_t n, int64_t s,
                                 int64_t ld, const double* alpha, const double* beta, void* stream);
rc_status rc_op_callback_create(rc_ctx* ctx, int dtype, int64_t n, rc_block_apply_fn fn, void* user,
                                rc_op** out);
rc_status rc_op_destroy(rc_op* op);
rc_status rc_op_dim(const rc_op* op, int64_t* n, int* dtype);

/* ------------------------------------------------------------------------------------
 * Filter-polynomial design (host arithmetic, no context or GPU needed).
 * ------------------------------------------------------------------------------------ */

/* XStar and UpperXStar of the degree-m Lanczos "C" polynomial (LanczosCpoly::getXStar /
 * getUpperXStar, LanczosCpoly.h:285-305). */
rc_status rc_cpoly_xstar(int64_t m, double* xstar, double* upper_xstar);
/* LanczosCpoly::getStarDegreeAndSpectralRadius (LanczosCpoly.h:498-555). */
rc_status rc_cpoly_star_degree(double shift, double lambda_bound, double lambda_star, int64_t degree_max,
                               int64_t* star_degree, double* star_bound);
/* Recurrence coefficients of LanczosCpolyOperatorLMCuda::apply (LanczosCpolyOperatorLMCuda.h:206-209)
 * for degree m, bound lambda_max and shift: gamma1 = -2/(rhoB - 2 shift), gamma2 = 2 - 4 shift/rhoB
 * with rhoB = (lambda_max + shift)/UpperXStar(m). */
rc_status rc_cpoly_gammas(int64_t m, double lambda_max, double shift, double* gamma1, double* gamma2);
/* P_m(x) (LanczosCpoly::evaluatePm, LanczosCpoly.h:234-270). */
double rc_cpoly_pm(int64_t m, double x);

/* ------------------------------------------------------------------------------------
 * Kernel-level entry points (device blocks, FP64/c128).
 * ------------------------------------------------------------------------------------ */

/* Y = alpha*A*X + beta*Y on n x s blocks. Replaces the user SpMM Op->apply(in,out,a,b)
 * (LanczosCpolyOperatorLMCuda.h:245; RayleighChebyshevLMCuda.h:2135,2235). */
rc_status rc_spmm(rc_ctx* ctx, const rc_op* op, const void* X, int64_t ldx, void* Y, int64_t ldy,
                  int64_t s, const double* alpha, const double* beta);

/* In-place X <- P_m(A')X, the Lanczos "C" polynomial filter with recurrence coefficients
 * gamma1, gamma2 (LanczosCpolyOperatorLMCuda.h:194-265; coefficients at :206-209):
 *   x1 = gamma2*(gamma1*A*x0 + x0),  x_k = gamma2*(gamma1*A*x_{k-1} + x_{k-1}) - x_{k-2},
 *   X  = x_m/(m+1), repeated `repetition` times.
 * precision: RC_PREC_FP64 or RC_PREC_MIXED (float/c64 recurrence, double in and out). */
rc_status rc_filter(rc_ctx* ctx, const rc_op* op, void* X, int64_t ld, int64_t s, int64_t degree,
                    int64_t repetition, double gamma1, double gamma2, int precision);

/* Leading dimension of the filter's row-major blocks for s columns: s rounded up to 32 bytes of
 * elements of dtype in the storage precision (double/c128 for RC_PREC_FP64, float/c64 for
 * RC_PREC_MIXED). 0 for bad arguments. */
int64_t rc_rm_leading_dim(int dtype, int precision, int64_t s);

/* One degree step of the filter on ROW-MAJOR device blocks (row i holds its s columns
 * contiguously; leading dimension ld >= s, a multiple of 32 bytes of elements):
 *   y = alpha*A*x + beta*x + gamma*z
 * the step of LanczosCpolyOperatorLMCuda::apply (LanczosCpolyOperatorLMCuda.h:241-257: the user
 * SpMM out = alpha*A*in + beta*out, then the substract kernel) fused into one pass. Storage and
 * arithmetic: double/c128 (RC_PREC_FP64) or float/c64 (RC_PREC_MIXED). z may be NULL (no gamma
 * term); y may alias z but not x. alpha, beta, gamma: (re, im) pairs. CSR and stencil operators.
 * The kernels are the filter's own, so each row is computed exactly as rc_filter computes it:
 * a row-sharded filter runs this step on each rank's extended block (own rows plus the halo rows
 * its rows couple to, filled by an exchange between steps) and matches the unsharded filter bit
 * for bit. No reference counterpart as a separate call. */
rc_status rc_filter_step_rm(rc_ctx* ctx, const rc_op* op, const void* x, const void* z, void* y, int64_t ld,
                            int64_t s, const double* alpha, const double* beta, const double* gamma, int precision);

/* The filter above in correction form, the MIXED-precision refinement step of rc_solve (no
 * reference counterpart; it computes LanczosCpolyOperatorLMCuda::apply, LanczosCpolyOperatorLMCuda.h:194-265,
 * on Ritz pairs). V (n x s, DEVICE, FP64, or c128 for complex Hermitian operators) holds Ritz
 * vectors v_c with Ritz values lam[c] (HOST, s doubles). With a = gamma2*gamma1, b = gamma2, the scalar recurrence c_0 = 1, c_1 = a lam + b,
 * c_k = (a lam + b) c_{k-1} - c_{k-2}, and the residual block R = A V - V diag(lam):
 *   e_1 = R,  e_k = a*A*e_{k-1} + b*e_{k-1} - e_{k-2} + c_{k-1} R,
 *   V <- (c_m V + a e_m)/(m+1)     (= x_m/(m+1) of rc_filter in exact arithmetic),
 * with R and every e_k stored in bfloat16 (complex: real and imaginary part each a bfloat16) and
 * FP32 (c64) arithmetic; the last combination is FP64. CSR or 5/7-point stencil operators, real or
 * complex, and real 27-point stencils; 1 <= s <= 256, degree >= 1. Returns after the work is
 * complete. */
rc_status rc_filter_correction(rc_ctx* ctx, const rc_op* op, void* V, int64_t ld, int64_t s, const double* lam,
                               int64_t degree, double gamma1, double gamma2);

/* One correction-filter application of rc_filter_correction_batch. */
typedef struct rc_correction_job {
    size_t struct_size;            /* sizeof(rc_correction_job), or 0 */
    const rc_op* op;
    void* V;                       /* DEVICE n x s FP64 (c128) block, leading dimension ld; distinct per job */
    int64_t ld;
    int64_t s;
    const double* lam;             /* HOST, s Ritz values */
    int64_t degree;
    double gamma1, gamma2;
} rc_correction_job;

/* Several rc_filter_correction applications (up to 64, each with its own operator, block, degree
 * and coefficients) whose degree steps run as one batched launch per step: the request server's
 * batched correction-filter kernels, with each block's arithmetic equal to rc_filter_correction's.
 * Jobs those kernels do not take (complex operators, 27-point stencils, blocks with 64-bit element
 * offsets) run through the single-block kernels in the same call. batched (optional out): the
 * number of jobs that ran in the batched launches. No reference counterpart. */
rc_status rc_filter_correction_batch(rc_ctx* ctx, int njobs, const rc_correction_job* jobs, int* batched);

/* Spectral bounds by single-vector Lanczos with Sturm multisection of the tridiagonal
 * every 5 steps (LanczosMaxMinFinder.h:248-544, Dstebz_C.h:112). v0: optional start
 * vector (HOST, n scalars; NULL = internal uniform[-1,1] draw from `seed`).
 * which: 0 = stop on both extremes, 1 = max only (getInitialRCspectralEstimates,
 * RayleighChebyshevLMCuda.h:710), 2 = min only. */
rc_status rc_lanczos_bounds(rc_ctx* ctx, const rc_op* op, const void* v0, uint64_t seed, double tol,
                            int which, int64_t max_iter, double* lmin, double* lmax, int64_t* iters);

/* Orthonormalise the columns of V (n x s) in place: CholeskyQR2 with diagonal scaling,
 * escalating to shifted CholeskyQR3 when the Gram matrix is numerically singular.
 * Replaces orthogonalize() = cusolverDn geqrf+orgqr (RayleighChebyshevLMCuda.h:1979-2107).
 * passes (optional out): number of Cholesky passes used. */
rc_status rc_cholqr(rc_ctx* ctx, int dtype, void* V, int64_t ld, int64_t n, int64_t s, int* passes);

/* Rayleigh-Ritz on orthonormal V (n x s): W = A*V, H = V^H W, H = Q diag(evals) Q^H
 * (ascending), then V <- V*Q, W <- W*Q (= A*V) and residuals r_j = ||W_j - evals_j V_j||
 * for j < res_count. Replaces formVtAV + computeVtVeigensystem +
 * createEigenVectorsAndResiduals (RayleighChebyshevLMCuda.h:2115-2285, :570-642).
 * evals, residuals: HOST outputs (s and res_count doubles); Q: optional HOST s*s output. */
rc_status rc_rayleigh_ritz(rc_ctx* ctx, const rc_op* op, void* V, void* W, int64_t ld, int64_t s,
                           int64_t res_count, double* evals, double* residuals, void* Q);

/* Eigen-decomposition of a small Hermitian matrix on the GPU (one-CTA parallel Jacobi),
 * ascending eigenvalues, eigenvectors in the columns of Q. H, Q, evals: HOST arrays.
 * Replaces DSYEV/ZHPEVX (RayleighChebyshevLMCuda.h:614,618) and JacobiDiagonalizer. */
rc_status rc_small_eigh(rc_ctx* ctx, int dtype, int64_t s, const void* H, double* evals, void* Q);

/* rc_small_eigh for callers that must not allocate device memory: code running under a fixed
 * device-memory budget negotiated at start-up, where a cudaMalloc can fail or take memory another
 * tenant of the GPU counts on, and callbacks invoked from another library's allocator or from an
 * operator apply(), where allocating would re-enter that library. Same arguments and results, but
 * the device staging and work memory come from one fixed array of this library (about 1.3 MiB, held
 * on every GPU that loads the library until the process exits), and no cudaMalloc/cudaFree is
 * called. s must be at most 128 (RC_ERR_INVALID otherwise). The first call on a device (and the
 * first after its CUDA context is re-created) looks up the array's device address, which may load
 * the library's module on the device: make that first call before any stream capture. All calls
 * share the array: calls whose GPU work overlaps (several host threads, or several contexts on one
 * device) race on it and must be serialised by the caller. The call copies H in and the results
 * out through host memory and returns when they are on the host.
 * This entry point has no counterpart in the reference. */
rc_status rc_small_eigh_noalloc(rc_ctx* ctx, int dtype, int64_t s, const void* H, double* evals, void* Q);

/* ------------------------------------------------------------------------------------
 * Whole solve: RayleighChebyshevLMCuda::getMinEigenSystem / getMinIntervalEigenSystem
 * (RayleighChebyshevLMCuda.h:775,794,827,876; base routine :896-1973).
 * ------------------------------------------------------------------------------------ */

/* Fill a HOST column-major n x s block with random start values (the VRandomizeOpType
 * contract randomize(Atype&), RayleighChebyshevLMCuda.h:1046,1178). */
typedef void (*rc_randomize_fn)(void* user, void* host_block, int64_t n, int64_t s);

typedef struct rc_solve_params {
    size_t struct_size;            /* sizeof(rc_solve_params) */
    int64_t eig_count;             /* eigCount / maxEigensystemDim */
    double tol;                    /* subspaceTol (clamped to >= 1e-11, :934-937) */
    int64_t subspace_increment;    /* subspaceIncrementSize */
    int64_t buffer_size;           /* bufferSize */
    int stop_condition;            /* RC_STOP_* (default COMBINATION) */
    int precision;                 /* RC_PREC_* */
    int64_t poly_degree_max;       /* minIntervalPolyDegreeMax (default 200) */
    int64_t filter_repetition;     /* filterRepetitionCount (default 1) */
    int64_t max_inner_loop;        /* maxInnerLoopCount (default 10000) */
    double max_min_tol;            /* Lanczos tolerance maxMinTol (default 1e-6) */
    int64_t lanczos_max_iter;      /* setMaxSpectralBoundsIter (default 10000) */
    int mode;                      /* 0 getMinEigenSystem(k,tol,...), 1 getMinEigenSystem with bounds,
                                      2 getMinIntervalEigenSystem(lambdaMax,...),
                                      3 getMinIntervalEigenSystem(minEst,lambdaMax,maxBound,...) */
    double min_eig_est;            /* modes 1,3 */
    double max_eig_bound;          /* modes 1,3 */
    double lambda_max;             /* modes 2,3: interval upper limit */
    int host_buffers;              /* 1: v0 / evecs_out are HOST pointers */
    int non_random_start;          /* setNonRandomStartFlag: use v0 columns as the start block */
    int64_t v0_cols;               /* number of columns provided in v0 (<= subspace size) */
    uint64_t seed;                 /* internal random draws when randomize_fn is NULL */
    rc_randomize_fn randomize_fn;  /* optional host randomizer for start/refresh blocks */
    void* randomize_user;
    const void* lanczos_v0;        /* optional HOST start vector for the bounds (n scalars) */
    double mixed_switch_tol;       /* MIXED: relative residual at which the plain FP32 filter gives way to
                                      the correction filter (or, where that is unsupported or
                                      mixed_refine = 1, to the FP64 filter). Default 0: the correction
                                      filter from the first Rayleigh-Ritz step, the FP64 filter at 1e-6 */
    int verbose;                   /* print per-iteration lines like verboseFlag */
    int phase_timing;              /* record CUDA-event time per phase (TIMING_ buckets) */
    int orth_mode;                 /* 0: Rayleigh-Ritz on the filtered block with the Cholesky factor of its
                                      scaled Gram matrix folded in, CholeskyQR2 when that matrix is
                                      ill-conditioned; 1: always CholeskyQR2 then Rayleigh-Ritz */
    int mixed_refine;              /* MIXED, after the switch tolerance: 0 (default) the correction filter
                                      (the recurrence applied to the residual block A V - V diag(lam) of
                                      the Ritz vectors, stored in bfloat16 with FP32 / c64 arithmetic,
                                      whose rounding error shrinks with the residual; CSR and 5/7-point
                                      stencil operators, real or complex, and real 27-point stencils,
                                      subspace <= 256; FP64 filter otherwise or when it stalls); 1 the
                                      FP64 filter */
} rc_solve_params;

typedef struct rc_solve_info {
    size_t struct_size;
    int64_t found;                 /* return value of getMinEigenSystem */
    int64_t inner_iterations;      /* total inner iterations (applyCountCumulative) */
    int64_t outer_passes;
    int64_t degree_steps;          /* filter degree-steps applied (all precisions) */
    int64_t fp64_degree_steps;     /* of which in FP64 */
    int64_t mixed_iterations;      /* inner iterations with the FP32 filter */
    int64_t lanczos_iterations;
    int64_t cholqr_passes;
    double min_eig_est;            /* spectral bounds used */
    double max_eig_est;
    double max_residual;           /* finalData["maxResidual"] (relative) */
    double max_eig_diff;           /* finalData["maxEigValueDifference"] */
    double max_rel_gap;            /* finalData["maxRelEigValueGap"] */
    int64_t count_ortho;           /* countData["ortho"] */
    int64_t count_opapply;         /* countData["OpApply"] */
    int64_t count_eigenvalue;      /* countData["eigenvalue"] */
    double time_total_ms;          /* timeValue buckets (phase_timing = 1) */
    double time_lanczos_ms;
    double time_filter_ms;
    double time_ortho_ms;
    double time_eigenvalue_ms;
    int64_t kernel_launches;
    double guard_value;            /* getGuardEigenvalue */
    int64_t fused_rr;              /* inner iterations whose Rayleigh-Ritz ran on the filtered block */
    int64_t fused_rr_fallbacks;    /* of those, rejected for conditioning and redone after CholeskyQR2 */
    double time_filter_steps_ms;   /* part of time_filter_ms spent in the fused degree-step launches
                                      themselves (row-major filter, transposes excluded; phase_timing = 1) */
    int64_t correction_iterations; /* MIXED: inner iterations that ran the correction filter */
    int64_t correction_degree_steps; /* of degree_steps, those of the correction filter */
    int64_t correction_element_bytes; /* bytes per stored element of the correction filter's residual
                                         and recurrence blocks: 2 (bfloat16) or 4 (FP32) for real
                                         operators, twice that for complex ones */
} rc_solve_info;

void rc_solve_params_default(rc_solve_params* p);

/* evals_out: HOST, eig_count doubles. evecs_out: column-major n x eig_count block (HOST or
 * DEVICE per host_buffers), leading dimension n. residuals_out: optional HOST eig_count
 * doubles (getEigVectorResiduals). v0: optional start block (see non_random_start). */
rc_status rc_solve(rc_ctx* ctx, const rc_op* op, const rc_solve_params* params, const void* v0,
                   double* evals_out, void* evecs_out, double* residuals_out, rc_solve_info* info);

/* ------------------------------------------------------------------------------------
 * Request server (no reference counterpart; the reference solves one problem per call,
 * RayleighChebyshevLMCuda::getMinEigenSystem, RayleighChebyshevLMCuda.h:794).
 *
 * A server owns one GPU's worth of solve slots. Each admitted request runs the same solver as
 * rc_solve, with its subspace, spectral bounds and Ritz state resident in that slot until it
 * finishes. Requests are admitted first-fit while a slot is free and the request's device
 * footprint fits the HBM budget (working blocks n*(4*(incr+buffer) + eig_count) scalars, the
 * small Rayleigh-Ritz buffers, and the operator's storage, charged once per operator in use).
 * Filter applications of the running solves that are ready at the same time are packed into
 * one batched launch per degree step (replayed from a captured CUDA graph), so the filter
 * sweeps of concurrent solves overlap on the device; each solve's arithmetic is the same as
 * when it runs alone or through rc_solve.
 * ------------------------------------------------------------------------------------ */
typedef struct rc_server rc_server;

typedef struct rc_server_params {
    size_t struct_size;            /* sizeof(rc_server_params) */
    int device;
    int64_t hbm_budget_bytes;      /* 0: 90 % of the device memory free at creation */
    int max_active;                /* solves resident at once, 1..64 (default 16) */
    double batch_window_us;        /* longest wait for more solves to join a filter batch (default 200) */
    int use_graphs;                /* 1 (default): batches replay captured CUDA graphs; 0: direct launches */
    double starvation_ms;          /* admission passes over a queued request for at most this long,
                                      then holds back later ones until it fits (default 2000) */
} rc_server_params;

enum { RC_REQ_QUEUED = 0, RC_REQ_RUNNING = 1, RC_REQ_DONE = 2, RC_REQ_FAILED = 3, RC_REQ_CANCELLED = 4 };

typedef struct rc_request_info {
    size_t struct_size;
    int state;                     /* RC_REQ_* */
    rc_status status;              /* the solve's status once finished */
    double queue_ms;               /* submit -> admitted to a slot */
    double run_ms;                 /* admitted -> finished */
    double latency_ms;             /* submit -> finished */
    int64_t batches;               /* batched filter launches the request joined */
    int64_t reserved_bytes;        /* device bytes charged to the budget (operator excluded) */
    int64_t device_bytes;          /* scratch the solve actually held at its peak */
} rc_request_info;

typedef struct rc_server_stats {
    size_t struct_size;
    int64_t submitted, completed, failed, cancelled, queued, running;
    int64_t batches;               /* batched filter launches */
    int64_t batched_jobs;          /* filter applications in them */
    int64_t max_jobs_in_batch;
    int64_t graph_launches, graphs_built;
    int64_t kernel_launches;       /* kernels of the batched filter */
    int64_t bytes_in_use, bytes_peak, budget;
} rc_server_stats;

void rc_server_params_default(rc_server_params* p);
rc_status rc_server_create(const rc_server_params* params, rc_server** out);
/* Cancels queued and running requests, waits for the running ones to stop, frees everything. */
rc_status rc_server_destroy(rc_server* server);
const char* rc_server_last_error(const rc_server* server);
/* Queue a solve of op (created on a context of the server's device; it must outlive the
 * request) with rc_solve's parameters and arguments. The output buffers are written when the
 * request finishes and must stay valid until then. RC_ERR_NOMEM when the request alone
 * exceeds the budget. */
rc_status rc_serve_submit(rc_server* server, const rc_op* op, const rc_solve_params* params, const void* v0,
                          double* evals_out, void* evecs_out, double* residuals_out, int64_t* request_id);
rc_status rc_serve_poll(rc_server* server, int64_t request_id, int* state);
/* Wait up to timeout_ms (< 0: no limit) for the request to finish; RC_ERR_NOT_READY on timeout. */
rc_status rc_serve_wait(rc_server* server, int64_t request_id, double timeout_ms, int* state);
/* The finished request's solve info, timings and error text (errbuf may be NULL). Returns the
 * request's own status, or RC_ERR_NOT_READY while it is queued or running. */
rc_status rc_serve_result(rc_server* server, int64_t request_id, rc_solve_info* info, rc_request_info* rinfo,
                          char* errbuf, size_t errbuf_len);
/* A queued request is dropped at once; a running one stops at its next inner iteration
 * (status RC_ERR_CANCELLED). */
rc_status rc_serve_cancel(rc_server* server, int64_t request_id);
/* Forget a finished request (its id becomes invalid). */
rc_status rc_serve_release(rc_server* server, int64_t request_id);
rc_status rc_server_stats_get(rc_server* server, rc_server_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* RC_B200_H_ */
