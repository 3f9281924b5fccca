// rc_solver.cu -- the Rayleigh-Chebyshev driver on one GPU.
//
// Restates RayleighChebyshevLMCuda::getMinIntervalEigenSystem_Base (RayleighChebyshevLMCuda.h:896-1973)
// with the block work on the device and the scalar control on the host:
//   outer loop (:1162-1818): orthonormalise the working block, run the inner loop, capture the
//     converged pairs below lambdaMax, shift minEigValue past them, refresh the stale columns;
//   inner loop (:1221-1607): choose the filter degree (LanczosCpoly), filter, deflate against
//     found vectors, CholeskyQR, Rayleigh-Ritz with fused residuals, stop test.
// Deliberate differences (the converged eigenpairs are the same):
//   * deflation against found vectors follows the CPU LM path (OrthogonalizeAtoB,
//     RayleighChebyshevLM.h:1241, :1844-1917) as two block Gram-Schmidt sweeps; the GPU
//     reference omits it (RayleighChebyshevLMCuda.h:1330-1334) and is only correct for one pass;
//   * Householder QR is replaced by CholeskyQR2 (shifted CholeskyQR3 when ill-conditioned);
//   * A*(V*Q) is taken as (A*V)*Q, which removes the second SpMM per iteration (:2235);
//   * Ritz vectors V*Q are not renormalised (V and Q are orthonormal);
//   * after an outer pass only the stale tail columns are refreshed (the CPU LM refreshes the
//     buffer range, RayleighChebyshevLM.h:1086-1092; the GPU reference the whole block, :1176-1179);
//   * MIXED precision: the first filter application runs in FP32 / c64 (there is no residual
//     block yet), then the correction filter (bfloat16 storage, FP32 / c64 arithmetic) on the
//     residual block of the Ritz vectors (rc_filter_rm.cu), which converges like the FP64 filter.
//     Operators without it (callback operators, blocks wider than kCorrMaxCols) run the FP32/c64 filter until the residuals reach mixed_switch_tol (1e-6) or
//     stall (never stopping in that phase), then the FP64 filter; a set mixed_switch_tol also
//     delays the correction filter to that residual. The FP64 filter also takes over when the
//     correction filter stalls.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>
#include "rc_common.cuh"
#include "rc_cpoly.h"
#include "rc_internal.h"

namespace rcb {

static constexpr double kSmallTol = 1.0e-11;  // RAYLEIGH_CHEBYSHEV_SMALL_TOL_ (:210)

// getRelErrorFactor (RayleighChebyshevLMCuda.h:325-338)
static double rel_err_factor(double val, double tol) {
    if (std::fabs(val) * tol > kSmallTol) return std::fabs(val);
    return kSmallTol / tol;
}

enum Phase { PH_TOTAL = 0, PH_LANCZOS, PH_FILTER, PH_ORTHO, PH_EIG, PH_N };

class Solver {
public:
    Solver(rc_ctx* ctx, rc_op* op, const rc_solve_params& p) : ctx_(ctx), op_(op), P_(p) {
        dtype_ = op->dtype;
        esz_ = dtype_ == RC_COMPLEX128 ? 16 : 8;
        n_ = op->n;
    }
    ~Solver() {
        for (auto& e : pool_) cudaEventDestroy(e);
    }
    rc_status run(const void* v0, double* evals_out, void* evecs_out, double* resid_out, rc_solve_info* info);

private:
    rc_status base(double minEigValue, double lambdaMax, double maxEigValue, int64_t maxEigensystemDim,
                   bool intervalStop, bool hardIntervalStop, const void* v0);
    rc_status alloc(int64_t ss, int64_t maxDim);
    rc_status randomize_cols(void* X, int64_t c0, int64_t c1);
    rc_status deflate(void* X, int64_t s);
    rc_status ortho(int64_t s);
    rc_status rr(void*& X, void*& AX, int64_t s, int64_t res_count, bool read_back, void* R32 = nullptr);
    rc_status rr_fused(int64_t s, int64_t res_count, bool* ok, void* R32 = nullptr);
    rc_status r32_block(int64_t s, void** out);
    rc_status ritz_and_residuals(XtArgs a, int64_t s, int64_t res_count, void* R32);
    rc_status lanczos(int which, double tol, double* lmin, double* lmax);
    void tic(int ph);
    void toc(int ph);
    void flush();

    rc_ctx* ctx_;
    rc_op* op_;
    rc_solve_params P_;
    int dtype_;
    size_t esz_;
    int64_t n_;
    CPoly cpoly_;

    void *V_ = nullptr, *W_ = nullptr, *T1_ = nullptr, *T2_ = nullptr, *E_ = nullptr;
    void *H_ = nullptr, *Q_ = nullptr, *C_ = nullptr;
    void *G_ = nullptr, *Tt_ = nullptr, *M1_ = nullptr, *Cc_ = nullptr;  // fused Rayleigh-Ritz
    double* dlam_ = nullptr;
    double* dres_ = nullptr;
    int* dinfo_ = nullptr;
    int* dflags_ = nullptr;
    double* dpiv_ = nullptr;
    int64_t fused_ok_ = 0, fused_fallback_ = 0;
    double* hbuf_ = nullptr;
    int64_t ss_cap_ = 0;
    // MIXED correction filter: the residual block of the current Ritz vectors (row-major, in the
    // correction filter's storage: rc_corr_t, or rc_corr2_t for complex operators),
    // valid while haveR_ (written by the last Rayleigh-Ritz step, consumed by the next filter)
    bool haveR_ = false;
    bool rWritten_ = false;  // set by ritz_and_residuals when it wrote the residual block
    // the correction filter left the filtered block row-major in the S_VFRM slot (V_ still holds the
    // Ritz vectors it started from); rr_fused then works on row-major blocks
    bool vfRm_ = false;
    bool rm_rr_ok(int64_t s, int64_t reps) const;
    int64_t corr_iters_ = 0, corr_steps_ = 0;

    std::vector<double> eigValues_, eigVecResiduals_, VtAVeigValue_, subspaceResiduals_;
    int64_t foundSize_ = 0;
    double guardValue_ = 0.0;
    uint64_t rng_counter_ = 0;

    int64_t count_ortho_ = 0, count_opapply_ = 0, count_eigenvalue_ = 0;
    double fd_maxResidual_ = 0.0, fd_maxEigDiff_ = 0.0, fd_maxGap_ = 0.0;
    int64_t inner_total_ = 0, outer_passes_ = 0, degree_steps_ = 0, fp64_steps_ = 0, mixed_iters_ = 0;
    int64_t cholqr_passes_ = 0, lanczos_iters_ = 0;
    double minEst_ = 0.0, maxEst_ = 0.0;

    double t_[PH_N] = {0, 0, 0, 0, 0};
    double step_ms0_ = 0.0;
    std::vector<cudaEvent_t> pool_;
    size_t pool_used_ = 0;
    struct Pending { int ph; cudaEvent_t a, b; };
    std::vector<Pending> pending_;
    cudaEvent_t open_[PH_N] = {nullptr, nullptr, nullptr, nullptr, nullptr};
};

// ---- phase timing with CUDA events on the solver stream (TIMING_ buckets, :2342-2381) ----
void Solver::tic(int ph) {
    if (!P_.phase_timing) return;
    if (pool_used_ == pool_.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        pool_.push_back(e);
    }
    open_[ph] = pool_[pool_used_++];
    cudaEventRecord(open_[ph], ctx_->stream);
}
void Solver::toc(int ph) {
    if (!P_.phase_timing || !open_[ph]) return;
    if (pool_used_ == pool_.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        pool_.push_back(e);
    }
    cudaEvent_t e = pool_[pool_used_++];
    cudaEventRecord(e, ctx_->stream);
    pending_.push_back({ph, open_[ph], e});
    open_[ph] = nullptr;
}
void Solver::flush() {
    if (!P_.phase_timing) return;
    step_flush(ctx_);
    for (auto& p : pending_) {
        float ms = 0.f;
        cudaEventSynchronize(p.b);
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) t_[p.ph] += ms;
    }
    pending_.clear();
    bool any_open = false;
    for (auto& o : open_) any_open = any_open || o != nullptr;
    if (!any_open) pool_used_ = 0;
}

rc_status Solver::alloc(int64_t ss, int64_t maxDim) {
    const size_t blk = (size_t)n_ * ss * esz_;
    RC_TRY(rc_slot(ctx_, S_V, blk, &V_));
    RC_TRY(rc_slot(ctx_, S_W, blk, &W_));
    RC_TRY(rc_slot(ctx_, S_T1, blk, &T1_));
    RC_TRY(rc_slot(ctx_, S_T2, blk, &T2_));
    const int64_t md = std::max<int64_t>(maxDim, 1);
    RC_TRY(rc_slot(ctx_, S_FOUND, (size_t)n_ * md * esz_, &E_));
    const int64_t sq = std::max<int64_t>(ss, md);
    const size_t mat = (size_t)sq * sq * esz_;
    void* sm = nullptr;
    RC_TRY(rc_slot(ctx_, S_IO, 8 * mat + (size_t)sq * 16 + 512, &sm));
    H_ = sm;
    Q_ = (char*)sm + mat;
    C_ = (char*)sm + 2 * mat;
    G_ = (char*)sm + 4 * mat;
    Tt_ = (char*)sm + 5 * mat;
    M1_ = (char*)sm + 6 * mat;
    Cc_ = (char*)sm + 7 * mat;
    dlam_ = (double*)((char*)sm + 8 * mat);
    dres_ = dlam_ + sq;
    dpiv_ = dres_ + sq;
    dinfo_ = (int*)(dpiv_ + 2);
    dflags_ = dinfo_ + 4;
    RC_TRY(rc_host_small(ctx_, (size_t)sq * 16 + 64, &hbuf_));
    ss_cap_ = ss;
    return RC_OK;
}

rc_status Solver::randomize_cols(void* X, int64_t c0, int64_t c1) {
    if (c1 <= c0) return RC_OK;
    if (P_.randomize_fn) {
        std::vector<unsigned char> host((size_t)n_ * (c1 - c0) * esz_);
        P_.randomize_fn(P_.randomize_user, host.data(), n_, c1 - c0);
        RC_CU(ctx_, cudaMemcpyAsync((char*)X + (size_t)c0 * n_ * esz_, host.data(), host.size(),
                                    cudaMemcpyHostToDevice, ctx_->stream));
        RC_CU(ctx_, cudaStreamSynchronize(ctx_->stream));
        return RC_OK;
    }
    return fill_random(ctx_, dtype_, X, n_, n_, c0, c1, P_.seed * 0x9E3779B97F4A7C15ull + (++rng_counter_));
}

// X <- X - E (E^H X), applied twice (block form of OrthogonalizeAtoB, RayleighChebyshevLM.h:1844-1917).
rc_status Solver::deflate(void* X, int64_t s) {
    if (foundSize_ <= 0) return RC_OK;
    for (int sweep = 0; sweep < 2; ++sweep) {
        RC_TRY(gram(ctx_, dtype_, n_, foundSize_, s, E_, n_, X, n_, C_, false));
        XtArgs a;
        a.n = n_; a.k = foundSize_; a.nc = s;
        a.X = E_; a.ldx = n_;
        a.T = C_; a.ldt = foundSize_;
        a.Y = X; a.ldy = n_;
        a.alpha = -1.0; a.beta = 1.0;
        RC_TRY(xt(ctx_, dtype_, a));
    }
    return RC_OK;
}

// Orthonormalise V (n x s) after deflation; V_ may be swapped with T1_.
rc_status Solver::ortho(int64_t s) {
    RC_TRY(deflate(V_, s));
    bool swapped = false;
    int passes = 0;
    RC_TRY(cholqr(ctx_, dtype_, V_, n_, n_, s, T1_, &swapped, &passes));
    if (swapped) std::swap(V_, T1_);
    cholqr_passes_ += passes;
    return RC_OK;
}

// Rayleigh-Ritz on orthonormal X (n x s): AX = A X, H = X^H AX, H = Q L Q^H,
// X <- X Q, AX <- AX Q, residuals of the first res_count columns; results read to the host.
// Ritz vectors Y = X Q (a.Y) and the residuals of their first res_count columns (dres_), plus
// the correction filter's residual block when R32 is given. Native operators (real, or complex CSR
// and 5/7-point stencils) with s <= kCorrMaxCols: Y by the GEMM and a row-major FP64 (c128) copy of
// it (written by the real GEMM itself for s <= 96, else by a layout change), then
// R = A Y - Y diag(lam) in one pass over that copy (rc_resid.cu): a sparse product costs less than
// the second dense product W Q. Otherwise (callback operators, wider blocks): the dual GEMM (A X) Q
// with the residual norms reduced on the fly.
rc_status Solver::ritz_and_residuals(XtArgs a, int64_t s, int64_t res_count, void* R32) {
    rWritten_ = false;
    if (resid_supported(op_, s)) {
        const int64_t ldrm = rm_leading_dim(dtype_, P64, s);
        void* yrm = nullptr;
        RC_TRY(rc_slot(ctx_, S_YRM, (size_t)n_ * ldrm * esz_, &yrm));
        a.X2 = nullptr;
        a.Y2 = nullptr;
        a.lam = nullptr;
        a.res_count = 0;
        if (dtype_ == RC_REAL64 && xt2_supported(dtype_, a.k, a.nc)) {
            a.Yrm = (double*)yrm;
            a.ldyr = ldrm;
            RC_TRY(xt(ctx_, dtype_, a));
        } else {
            RC_TRY(xt(ctx_, dtype_, a));
            RC_TRY(to_row_major(ctx_, dtype_, n_, s, a.Y, a.ldy, yrm, ldrm));
        }
        RC_TRY(resid_block(ctx_, op_, yrm, ldrm, s, dlam_, res_count, dres_, R32,
                           R32 ? corr_leading_dim(dtype_, s) : 0));
        rWritten_ = R32 != nullptr;
        return RC_OK;
    }
    a.Y2 = nullptr;  // only the residual norms of (A X) Q are needed
    a.lam = dlam_;
    a.res_count = res_count;
    a.res = dres_;
    return xt(ctx_, dtype_, a);
}

// The row-major Rayleigh-Ritz step after a correction filter: real native operators with blocks the
// DMMA kernels take (s <= 96), one filter application per iteration, no found vectors to deflate
// against (the deflation works on column-major blocks), outside the request server.
bool Solver::rm_rr_ok(int64_t s, int64_t reps) const {
    return ctx_->rm_rr && dtype_ == RC_REAL64 && !ctx_->serve && P_.orth_mode == 0 && reps == 1 && foundSize_ == 0 &&
           gram2_supported(dtype_, s) && xt2_supported(dtype_, s, s) && resid_supported(op_, s);
}

rc_status Solver::r32_block(int64_t s, void** out) {
    return rc_slot(ctx_, S_R32, (size_t)n_ * corr_leading_dim(dtype_, s) * corr_elem_bytes(dtype_), out);
}

rc_status Solver::rr(void*& X, void*& AX, int64_t s, int64_t res_count, bool read_back, void* R32) {
    StepArgs st;
    st.s = s;
    st.x = X; st.xp = P64; st.ldx = n_;
    st.y = AX; st.yp = P64; st.ldy = n_;
    st.cp = P64;
    RC_TRY(op_step(ctx_, op_, st));
    RC_TRY(gram(ctx_, dtype_, n_, s, s, X, n_, AX, n_, H_, true));
    RC_TRY(small_eigh(ctx_, dtype_, s, H_, Q_, dlam_, dinfo_));
    XtArgs a;
    a.n = n_; a.k = s; a.nc = s;
    a.X = X; a.ldx = n_;
    a.T = Q_; a.ldt = s;
    a.Y = T1_; a.ldy = n_;
    a.X2 = AX; a.ldx2 = n_;
    RC_TRY(ritz_and_residuals(a, s, res_count, R32));
    std::swap(X, T1_);
    if (read_back) {
        RC_CU(ctx_, cudaMemcpyAsync(hbuf_, dlam_, s * sizeof(double), cudaMemcpyDeviceToHost, ctx_->stream));
        if (res_count > 0)
            RC_CU(ctx_, cudaMemcpyAsync(hbuf_ + s, dres_, res_count * sizeof(double), cudaMemcpyDeviceToHost,
                                        ctx_->stream));
        RC_CU(ctx_, cudaStreamSynchronize(ctx_->stream));
        VtAVeigValue_.assign(hbuf_, hbuf_ + s);
        subspaceResiduals_.assign(hbuf_ + s, hbuf_ + s + res_count);
    }
    return RC_OK;
}

// Rayleigh-Ritz directly on the filtered (not orthonormalised) block V_f = V_:
//   W = A V_f, G = V_f^H V_f, H = V_f^H W, G = D R^H R D (scaled Cholesky), T = D^-1 R^-1,
//   C = T^H H T, C = Y L Y^H (Jacobi), Q = T Y, V <- V_f Q, W <- W Q (+ residuals).
// V_f Q has orthonormal columns (Q^H G Q = I) and spans span(V_f), so this is the Rayleigh-Ritz
// step of the reference on the orthonormalised block with the CholeskyQR folded into the small
// problem. Accepted only when the scaled Gram matrix is well conditioned (smallest Cholesky pivot
// >= 1e-3, no shift needed); otherwise *ok = false, V_ still holds V_f and the caller
// orthonormalises and repeats the Rayleigh-Ritz step.
rc_status Solver::rr_fused(int64_t s, int64_t res_count, bool* ok, void* R32) {
    const bool rm = vfRm_;
    vfRm_ = false;
    const int64_t ldrm = rm_leading_dim(RC_REAL64, P64, s);
    void *vf = nullptr, *wrm = nullptr;
    if (rm) {
        // row-major: V_f from the correction filter, W = A V_f by the filter's FP64 step kernel
        RC_TRY(rc_slot(ctx_, S_VFRM, (size_t)n_ * ldrm * sizeof(double), &vf));
        RC_TRY(rc_slot(ctx_, S_WRM, (size_t)n_ * ldrm * sizeof(double), &wrm));
        const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
        RC_TRY(rm_step(ctx_, op_, vf, nullptr, wrm, ldrm, s, one, zero, zero, RC_PREC_FP64));
        RC_TRY(gram2(ctx_, n_, s, (const double*)vf, ldrm, (const double*)vf, ldrm, (double*)G_, (const double*)wrm,
                     ldrm, (double*)H_, true));
    } else {
        StepArgs st;
        st.s = s;
        st.x = V_; st.xp = P64; st.ldx = n_;
        st.y = W_; st.yp = P64; st.ldy = n_;
        st.cp = P64;
        RC_TRY(op_step(ctx_, op_, st));
        if (gram2_supported(dtype_, s)) {
            RC_TRY(gram2(ctx_, n_, s, (const double*)V_, n_, (const double*)V_, n_, (double*)G_, (const double*)W_,
                         n_, (double*)H_));
        } else {
            RC_TRY(gram(ctx_, dtype_, n_, s, s, V_, n_, V_, n_, G_, true));
            RC_TRY(gram(ctx_, dtype_, n_, s, s, V_, n_, W_, n_, H_, true));
        }
    }
    RC_CU(ctx_, cudaMemsetAsync(dflags_, 0, 4 * sizeof(int), ctx_->stream));
    RC_TRY(chol_factor(ctx_, dtype_, s, n_, G_, Tt_, dflags_, dpiv_));
    RC_TRY(small_gemm(ctx_, dtype_, s, H_, false, Tt_, M1_));   // H T
    RC_TRY(small_gemm(ctx_, dtype_, s, Tt_, true, M1_, Cc_));   // T^H H T
    RC_TRY(hermitize(ctx_, dtype_, s, Cc_));
    RC_TRY(small_eigh(ctx_, dtype_, s, Cc_, M1_, dlam_, dinfo_));  // Y into M1
    RC_TRY(small_gemm(ctx_, dtype_, s, Tt_, false, M1_, Q_));  // Q = T Y
    if (rm) {
        // Ritz vectors V_f Q, column-major into T1_ and row-major beside them, then the residuals
        void* yrm = nullptr;
        RC_TRY(rc_slot(ctx_, S_YRM, (size_t)n_ * ldrm * sizeof(double), &yrm));
        RC_TRY(xt2_rm(ctx_, n_, s, s, (const double*)vf, ldrm, (const double*)Q_, s, (double*)T1_, n_, (double*)yrm,
                      ldrm));
        RC_TRY(resid_block(ctx_, op_, yrm, ldrm, s, dlam_, res_count, dres_, R32,
                           R32 ? corr_leading_dim(dtype_, s) : 0));
        rWritten_ = R32 != nullptr;
    } else {
        XtArgs a;
        a.n = n_; a.k = s; a.nc = s;
        a.X = V_; a.ldx = n_;
        a.T = Q_; a.ldt = s;
        a.Y = T1_; a.ldy = n_;
        a.X2 = W_; a.ldx2 = n_;
        RC_TRY(ritz_and_residuals(a, s, res_count, R32));
    }
    RC_CU(ctx_, cudaMemcpyAsync(hbuf_, dlam_, s * sizeof(double), cudaMemcpyDeviceToHost, ctx_->stream));
    if (res_count > 0)
        RC_CU(ctx_, cudaMemcpyAsync(hbuf_ + s, dres_, res_count * sizeof(double), cudaMemcpyDeviceToHost,
                                    ctx_->stream));
    RC_CU(ctx_, cudaMemcpyAsync(hbuf_ + s + res_count, dpiv_, sizeof(double), cudaMemcpyDeviceToHost, ctx_->stream));
    RC_CU(ctx_, cudaMemcpyAsync(hbuf_ + s + res_count + 1, dflags_, 4 * sizeof(int), cudaMemcpyDeviceToHost,
                                ctx_->stream));
    RC_CU(ctx_, cudaStreamSynchronize(ctx_->stream));
    const double piv = hbuf_[s + res_count];
    const int* fl = (const int*)(hbuf_ + s + res_count + 1);
    *ok = !(fl[0] || fl[1] || fl[2]) && piv >= 1e-3 && std::isfinite(piv);
    if (!*ok) {
        ++fused_fallback_;
        rWritten_ = false;
        // the caller orthonormalises V_f: bring it to V_ when it was formed row-major
        if (rm) RC_TRY(to_col_major(ctx_, dtype_, n_, s, vf, ldrm, V_, n_));
        return RC_OK;
    }
    ++fused_ok_;
    std::swap(V_, T1_);
    VtAVeigValue_.assign(hbuf_, hbuf_ + s);
    subspaceResiduals_.assign(hbuf_ + s, hbuf_ + s + res_count);
    return RC_OK;
}

rc_status Solver::lanczos(int which, double tol, double* lmin, double* lmax) {
    LanczosResult lr;
    tic(PH_LANCZOS);
    RC_TRY(lanczos_bounds(ctx_, op_, P_.lanczos_v0, P_.seed ^ 0x5bd1e995ull, tol, which,
                          P_.lanczos_max_iter > 0 ? P_.lanczos_max_iter : 10000, &lr));
    toc(PH_LANCZOS);
    flush();
    *lmin = lr.lmin;
    *lmax = lr.lmax;
    lanczos_iters_ += lr.iters;
    minEst_ = lr.lmin;
    maxEst_ = lr.lmax;
    return RC_OK;
}

rc_status Solver::base(double minEigValue, double lambdaMax, double maxEigValue, int64_t maxEigensystemDim,
                       bool intervalStopConditionFlag, bool hardIntervalStopFlag, const void* v0) {
    double subspaceTol = P_.tol;
    if (subspaceTol < kSmallTol) subspaceTol = kSmallTol;  // :934-937
    int64_t subspaceIncrementSize = P_.subspace_increment;
    int64_t bufferSize = P_.buffer_size;
    int64_t subspaceSize = subspaceIncrementSize + bufferSize;
    const int64_t vectorDimension = n_;
    if (subspaceSize > vectorDimension) {  // :973-988
        if (subspaceIncrementSize < vectorDimension) {
            bufferSize = vectorDimension - subspaceIncrementSize;
            subspaceSize = vectorDimension;
        } else {
            subspaceSize = vectorDimension;
            subspaceIncrementSize = vectorDimension;
            bufferSize = 0;
        }
        maxEigensystemDim = vectorDimension;
    }
    if (subspaceSize < 1) return rc_fail(ctx_, RC_ERR_INVALID, "subspace size must be positive");
    std::vector<double> oldEigs(subspaceSize, 0.0), eigDiffs(subspaceSize, 1.0), oldEigDiffs(subspaceSize, 1.0);
    RC_TRY(alloc(subspaceSize, maxEigensystemDim));
    eigValues_.clear();
    eigVecResiduals_.clear();
    foundSize_ = 0;

    // start block (:1040-1070): given columns first, random fill for the rest
    int64_t given = 0;
    if (P_.non_random_start && v0) {
        given = std::min<int64_t>(P_.v0_cols > 0 ? P_.v0_cols : subspaceSize, subspaceSize);
        RC_CU(ctx_, cudaMemcpyAsync(V_, v0, (size_t)n_ * given * esz_,
                                    P_.host_buffers ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                                    ctx_->stream));
    }
    RC_TRY(randomize_cols(V_, given, subspaceSize));

    // Quick return when the subspace spans the whole space (:1084-1125)
    if (vectorDimension == subspaceSize) {
        tic(PH_ORTHO);
        RC_TRY(ortho(subspaceSize));
        toc(PH_ORTHO);
        tic(PH_EIG);
        RC_TRY(rr(V_, W_, subspaceSize, subspaceSize, true));
        toc(PH_EIG);
        flush();
        RC_TRY(copy_cols(ctx_, dtype_, V_, n_, E_, n_, n_, subspaceSize));
        eigValues_ = VtAVeigValue_;
        eigVecResiduals_ = subspaceResiduals_;
        foundSize_ = subspaceSize;
        return RC_OK;
    }

    const int64_t maxInnerLoopCount = P_.max_inner_loop > 0 ? P_.max_inner_loop : 10000;
    const int64_t polyDegreeMax = P_.poly_degree_max > 0 ? P_.poly_degree_max : 200;
    const int64_t filterRepetitionCount = P_.filter_repetition > 0 ? P_.filter_repetition : 1;
    const int stopCondition = (P_.stop_condition == RC_STOP_DEFAULT) ? RC_STOP_COMBINATION : P_.stop_condition;
    const bool mixed = P_.precision == RC_PREC_MIXED && op_->kind != 2;
    // relative residual at which the plain FP32 filter gives way: by default at the first
    // Rayleigh-Ritz step to the correction filter (a bfloat16 correction step moves fewer bytes than
    // a plain FP32 step and converges like the FP64 filter), else at 1e-6 to the FP64 filter
    const double switchTolSet = P_.mixed_switch_tol > 0 ? P_.mixed_switch_tol : 0.0;
    // MIXED phases: 0 plain FP32 filter, 1 correction filter, 2 FP64 filter
    enum { PH_PLAIN32 = 0, PH_CORR32 = 1, PH_FP64 = 2 };

    bool completedBasisFlag = false;
    int exitFlag = 0;
    int64_t applyCountCumulative = 0;
    long starDegree = 0;
    double starBound = 0.0;
    int64_t lastFoundCount = 0;
    std::vector<double> residualHistory;

    while (exitFlag == 0) {
        ++outer_passes_;
        for (int64_t k = bufferSize; k < subspaceSize; ++k) oldEigs[k] = oldEigs[bufferSize];  // :1169-1172
        if (applyCountCumulative > 0) RC_TRY(randomize_cols(V_, subspaceSize - lastFoundCount, subspaceSize));
        haveR_ = false;
        const bool corrOk = mixed && P_.mixed_refine == 0 && rm_corr_supported(op_, subspaceSize);
        const double switchTol = switchTolSet > 0 ? switchTolSet : (corrOk ? HUGE_VAL : 1e-6);

        tic(PH_ORTHO);
        RC_TRY(ortho(subspaceSize));  // the reference orthogonalizes twice here (:1195-1196)
        toc(PH_ORTHO);
        count_ortho_ += 2;

        double lambdaStar = maxEigValue;
        double eigDiffRatio = 1.0;
        int64_t innerLoopCount = 0;
        long starDegreeSave = 0;
        double starBoundSave = 0.0;
        double stopCheckValue = subspaceTol + 1.0e10;
        int64_t applyCount = 0;
        residualHistory.clear();
        double maxGap = 0.0, maxResidual = 0.0, maxEigDiff = 0.0;
        int64_t oscillationCount = 0;
        int64_t residualCheckCount = 0;
        // mixed-precision phase state
        int phase = mixed ? PH_PLAIN32 : PH_FP64;
        double bestFp32Residual = 1e300;
        int stallCount = 0;
        size_t corrStart = 0;  // residualHistory index where the correction phase began

        while ((stopCheckValue > subspaceTol) && (innerLoopCount < maxInnerLoopCount)) {
            if (ctx_->cancel && ctx_->cancel->load(std::memory_order_relaxed))
                return rc_fail(ctx_, RC_ERR_CANCELLED, "request cancelled");
            // ---- filter parameters (:1233-1296)
            const double shift = -minEigValue;
            starDegreeSave = starDegree;
            starBoundSave = starBound;
            starDegree = 0;
            double relErrFactor = rel_err_factor(minEigValue, subspaceTol);
            const double eMin = std::fabs(minEigValue - lambdaStar) / relErrFactor;
            relErrFactor = rel_err_factor(maxEigValue, subspaceTol);
            const double eMax = std::fabs(maxEigValue - lambdaStar) / relErrFactor;
            if ((eMin < subspaceTol) && (eMax < subspaceTol)) {  // identity
                starDegree = 1;
                starBound = maxEigValue;
            } else if ((!(maxEigDiff > subspaceTol)) && (innerLoopCount > 3) && (eigDiffRatio < .2)) {
                starDegree = starDegreeSave;  // multiplicity > subspace dimension
                starBound = starBoundSave;
            }
            if (starDegree == 0)
                cpoly_.star_degree_and_bound(shift, maxEigValue, lambdaStar, (long)polyDegreeMax, starDegree, starBound);
            if (starDegree < starDegreeSave) {  // monotone degree within a subspace (:1298-1303)
                starDegree = starDegreeSave;
                starBound = starBoundSave;
            }
            // ---- filter (:1305-1319)
            double fa = 0.0, fb = 0.0;
            cpoly_.coefficients(starDegree, starBound, shift, fa, fb);
            const int prec = phase == PH_FP64 ? RC_PREC_FP64 : RC_PREC_MIXED;
            tic(PH_FILTER);
            if (!completedBasisFlag) {
                int64_t steps = 0;
                if (phase == PH_CORR32 && haveR_) {
                    // the correction filter: V_ holds the Ritz vectors, dlam_ their values and the
                    // R32 slot their residual block; its two work blocks (FP32 or bfloat16) fit in T1_
                    void* R32 = nullptr;
                    RC_TRY(r32_block(subspaceSize, &R32));
                    const size_t rmb =
                        (size_t)n_ * corr_leading_dim(dtype_, subspaceSize) * corr_elem_bytes(dtype_);
                    const size_t blk = (size_t)n_ * subspaceSize * esz_;
                    void* bufA = T1_;
                    void* bufB = (char*)T1_ + ((rmb + 255) / 256) * 256;
                    if (((rmb + 255) / 256) * 256 + rmb > blk) bufB = T2_;
                    if (rmb > blk) {  // narrow blocks: the row padding makes an FP32 block larger
                        RC_TRY(rc_slot(ctx_, S_FA, rmb, &bufA));
                        RC_TRY(rc_slot(ctx_, S_FB, rmb, &bufB));
                    }
                    for (int64_t r = 0; r < filterRepetitionCount; ++r) {
                        if (r > 0) {  // a repeated application has no residual block: plain FP32
                            int64_t st2 = 0;
                            RC_TRY(filter_apply(ctx_, op_, V_, n_, subspaceSize, starDegree, 1, fa, fb,
                                                RC_PREC_MIXED, T1_, T2_, (size_t)n_ * subspaceSize * esz_, &st2));
                            steps += st2;
                            continue;
                        }
                        if (rm_rr_ok(subspaceSize, filterRepetitionCount)) {
                            // the filtered block row-major, from the row-major copy of the Ritz
                            // vectors that the last Rayleigh-Ritz step wrote beside V_
                            const int64_t ldrm = rm_leading_dim(RC_REAL64, P64, subspaceSize);
                            void* yrm = nullptr;
                            void* vf = nullptr;
                            RC_TRY(rc_slot(ctx_, S_YRM, (size_t)n_ * ldrm * sizeof(double), &yrm));
                            RC_TRY(rc_slot(ctx_, S_VFRM, (size_t)n_ * ldrm * sizeof(double), &vf));
                            RC_TRY(rm_filter_corr(ctx_, op_, V_, n_, subspaceSize, starDegree, fa, fb, dlam_, R32,
                                                  bufA, bufB, (const double*)yrm, ldrm, (double*)vf, ldrm));
                            vfRm_ = true;
                        } else {
                            RC_TRY(rm_filter_corr(ctx_, op_, V_, n_, subspaceSize, starDegree, fa, fb, dlam_, R32,
                                                  bufA, bufB));
                        }
                        steps += starDegree;
                        corr_steps_ += starDegree;
                    }
                    ++corr_iters_;
                } else {
                    // filter_apply takes (g1, g2) with a = g2*g1, b = g2
                    RC_TRY(filter_apply(ctx_, op_, V_, n_, subspaceSize, starDegree, filterRepetitionCount, fa,
                                        fb, prec, T1_, T2_, (size_t)n_ * subspaceSize * esz_, &steps));
                }
                degree_steps_ += steps;
                if (phase == PH_FP64) fp64_steps_ += steps;
            }
            haveR_ = false;
            toc(PH_FILTER);
            if (phase != PH_FP64) ++mixed_iters_;
            applyCount += 1;
            count_opapply_ += starDegree * subspaceSize;

            // ---- orthonormalise (:1321-1338) and Rayleigh-Ritz + residuals (:1344-1401):
            // fused on the filtered block when it is well conditioned, else CholeskyQR2 then RR.
            if (foundSize_ + subspaceSize < vectorDimension) residualCheckCount = subspaceIncrementSize;
            else residualCheckCount = subspaceSize;
            bool fused = false;
            // the residual block for the next correction filter, once the residuals approach the
            // switch tolerance
            void* R32 = nullptr;
            const double prevResidual = residualHistory.empty() ? 1e300 : residualHistory.back();
            if (corrOk && phase != PH_FP64 && (phase == PH_CORR32 || prevResidual < 1e3 * switchTol))
                RC_TRY(r32_block(subspaceSize, &R32));
            if (P_.orth_mode == 0) {
                tic(PH_EIG);
                RC_TRY(deflate(V_, subspaceSize));
                RC_TRY(rr_fused(subspaceSize, residualCheckCount, &fused, R32));
                toc(PH_EIG);
            }
            if (!fused) {
                tic(PH_ORTHO);
                RC_TRY(ortho(subspaceSize));
                toc(PH_ORTHO);
                tic(PH_EIG);
                RC_TRY(rr(V_, W_, subspaceSize, residualCheckCount, true, R32));
                toc(PH_EIG);
            }
            haveR_ = R32 != nullptr && rWritten_;
            flush();
            count_ortho_ += 1;
            count_opapply_ += subspaceSize + residualCheckCount;
            count_eigenvalue_ += 1;
            for (double r : subspaceResiduals_)
                if (!std::isfinite(r))
                    return rc_fail(ctx_, RC_ERR_BREAKDOWN, "non-finite residual (NaN or Inf in the operator?)");

            maxResidual = 0.0;
            for (size_t k = 0; k < subspaceResiduals_.size(); ++k) {
                relErrFactor = rel_err_factor(VtAVeigValue_[k], subspaceTol);
                maxResidual = std::max(maxResidual, subspaceResiduals_[k] / relErrFactor);
            }
            residualHistory.push_back(maxResidual);

            // ---- eigenvalue convergence (:1436-1497)
            const int64_t eigSubspaceCheckSize =
                std::min<int64_t>(intervalStopConditionFlag ? subspaceIncrementSize + 1 : subspaceIncrementSize,
                                  subspaceSize);
            for (int64_t i = 0; i < eigSubspaceCheckSize; ++i) oldEigDiffs[i] = eigDiffs[i];
            maxEigDiff = 0.0;
            for (int64_t i = 0; i < eigSubspaceCheckSize; ++i) {
                double eigDiff = std::fabs(VtAVeigValue_[i] - oldEigs[i]);
                relErrFactor = rel_err_factor(oldEigs[i], subspaceTol);
                eigDiff = eigDiff / relErrFactor;
                eigDiffs[i] = eigDiff;
                maxEigDiff = eigDiff > maxEigDiff ? eigDiff : maxEigDiff;
            }
            for (int64_t i = 0; i < subspaceSize; ++i) oldEigs[i] = VtAVeigValue_[i];
            int64_t diffCount = 0;
            eigDiffRatio = 0.0;
            if (maxEigDiff > subspaceTol) {
                for (int64_t i = 0; i < eigSubspaceCheckSize; ++i) {
                    if (std::fabs(oldEigDiffs[i]) > subspaceTol / 10.0) {
                        eigDiffRatio += std::fabs(eigDiffs[i] / oldEigDiffs[i]);
                        diffCount++;
                    }
                }
                eigDiffRatio = diffCount > 0 ? eigDiffRatio / (double)diffCount : 1.0;
            }
            const double spectralRange = std::fabs(lambdaMax - minEigValue);
            maxGap = 0.0;
            for (int64_t i = 1; i < eigSubspaceCheckSize; ++i)
                maxGap = std::max(maxGap, std::fabs(VtAVeigValue_[i] - VtAVeigValue_[i - 1]) / spectralRange);

            if (P_.verbose)
                printf("[rc] iter %ld  degree %ld  max rel residual %.4e  max eig change %.4e  change ratio %.3f  "
                       "max gap %.4e %s\n",
                       (long)innerLoopCount, (long)starDegree, maxResidual, maxEigDiff, eigDiffRatio, maxGap,
                       phase == PH_PLAIN32 ? "[fp32 filter]" : (phase == PH_CORR32 ? "[bf16 correction]" : ""));

            // ---- stop test (:1520-1545)
            if (stopCondition == RC_STOP_RESIDUAL_ONLY) {
                stopCheckValue = maxResidual;
            } else if (stopCondition == RC_STOP_EIGENVALUE_ONLY) {
                stopCheckValue = maxEigDiff;
            } else {
                stopCheckValue = maxEigDiff;
                if (maxResidual > std::sqrt(subspaceTol)) stopCheckValue = maxResidual;
            }
            if (subspaceIncrementSize == 0) stopCheckValue = 0.0;
            // oscillation stop for RESIDUAL_ONLY (:1551-1592)
            if ((stopCondition == RC_STOP_RESIDUAL_ONLY) && (maxResidual < std::sqrt(subspaceTol)) &&
                phase != PH_PLAIN32) {
                const int64_t rIndex = (int64_t)residualHistory.size() - 1;
                if (rIndex > 3) {
                    const double a = (residualHistory[rIndex - 3] - 2.0 * residualHistory[rIndex - 2] +
                                      residualHistory[rIndex - 1]) / std::fabs(maxResidual);
                    const double b = (residualHistory[rIndex - 2] - 2.0 * residualHistory[rIndex - 1] +
                                      residualHistory[rIndex]) / std::fabs(maxResidual);
                    if (a * b < 0.0) {
                        oscillationCount += 1;
                        if (oscillationCount > 5) stopCheckValue = 0.0;
                    }
                }
            }
            // ---- mixed precision: leave the plain FP32 phase once the residual has reached the
            // switch tolerance, has stalled, or the stop test would pass (never stop there); leave
            // the correction phase for FP64 when it stops converging (no 0.7x reduction over eight
            // iterations).
            if (phase == PH_PLAIN32) {
                bool sw = maxResidual <= switchTol || stopCheckValue <= subspaceTol;
                if (maxResidual < 0.5 * bestFp32Residual) {
                    bestFp32Residual = maxResidual;
                    stallCount = 0;
                } else if (maxResidual < 1e-4 && ++stallCount >= 2) {
                    sw = true;  // FP32 rounding floor reached
                }
                if (sw) {
                    phase = corrOk ? PH_CORR32 : PH_FP64;
                    corrStart = residualHistory.size();
                    if (stopCheckValue <= subspaceTol) stopCheckValue = subspaceTol + 1.0;
                }
            } else if (phase == PH_CORR32) {
                const size_t h = residualHistory.size();
                if (h >= corrStart + 9 && maxResidual > 0.7 * residualHistory[h - 9]) phase = PH_FP64;
            }
            // ---- update the filter interval (:1602-1605)
            lambdaStar = VtAVeigValue_[subspaceSize - 1];
            minEigValue = (minEigValue < VtAVeigValue_[0]) ? minEigValue : VtAVeigValue_[0];
            innerLoopCount++;
        }
        inner_total_ += innerLoopCount;
        fd_maxResidual_ = std::max(maxResidual, fd_maxResidual_);
        fd_maxEigDiff_ = std::max(maxEigDiff, fd_maxEigDiff_);
        fd_maxGap_ = std::max(maxGap, fd_maxGap_);
        applyCountCumulative += applyCount;

        // ---- capture found eigenpairs (:1643-1702)
        int64_t foundCount = 0;
        const int64_t checkIndexCount =
            (foundSize_ + subspaceSize < vectorDimension) ? subspaceIncrementSize : subspaceSize;
        for (int64_t i = 0; i < checkIndexCount; ++i) {
            const double vtvEig = VtAVeigValue_[i];
            const double rf = rel_err_factor(lambdaMax, subspaceTol);
            if ((vtvEig - lambdaMax) / rf < subspaceTol) foundCount++;
        }
        if ((foundCount + foundSize_) >= maxEigensystemDim) {
            foundCount = maxEigensystemDim - foundSize_;
            exitFlag = 1;
        }
        if ((foundCount + foundSize_) >= vectorDimension) {
            foundCount = vectorDimension - foundSize_;
            exitFlag = 1;
        }
        if (foundCount > 0) {
            RC_TRY(copy_cols(ctx_, dtype_, V_, n_, (char*)E_ + (size_t)foundSize_ * n_ * esz_, n_, n_, foundCount));
            for (int64_t i = 0; i < foundCount; ++i) {
                eigValues_.push_back(VtAVeigValue_[i]);
                eigVecResiduals_.push_back(i < (int64_t)subspaceResiduals_.size() ? subspaceResiduals_[i] : 0.0);
            }
            foundSize_ += foundCount;
            if (P_.verbose)
                printf("[rc] found %ld eigenpairs, largest %.15e (bound %.15e)\n", (long)foundSize_,
                       eigValues_[foundSize_ - 1], lambdaMax);
        }
        haveR_ = false;
        // shuffle the unconverged vectors to the head of the block (:1707-1716)
        if (!exitFlag && foundCount > 0) {
            RC_TRY(copy_cols(ctx_, dtype_, (char*)V_ + (size_t)foundCount * n_ * esz_, n_, T1_, n_, n_,
                             subspaceSize - foundCount));
            std::swap(V_, T1_);
        }
        lastFoundCount = foundCount;
        // guard eigenvalue (:1720-1766)
        double vtvEig = bufferSize > 0 ? VtAVeigValue_[subspaceSize - bufferSize] : lambdaMax;
        guardValue_ = vtvEig;
        const double rf = rel_err_factor(lambdaMax, subspaceTol);
        const double vtvEigCheck = (vtvEig - lambdaMax) / rf;
        if (hardIntervalStopFlag) {
            if (guardValue_ > lambdaMax) exitFlag = 1;
        } else {
            if (vtvEigCheck >= 10.0 * subspaceTol) exitFlag = 1;
        }
        if (foundSize_ > 0) minEigValue = eigValues_[foundSize_ - 1];  // :1772
        starDegree = 1;
        starBound = maxEigValue;
        // subspace reduction when the block would exceed the space (:1784-1816)
        if (!exitFlag && (foundSize_ + subspaceSize) >= vectorDimension) {
            if (foundSize_ + subspaceIncrementSize >= vectorDimension) {
                bufferSize = 0;
                subspaceIncrementSize = vectorDimension - foundSize_;
                subspaceSize = subspaceIncrementSize;
                completedBasisFlag = true;
                RC_TRY(randomize_cols(V_, 0, subspaceSize));
                lastFoundCount = 0;
            } else {
                bufferSize = vectorDimension - (foundSize_ + subspaceIncrementSize);
                subspaceSize = subspaceIncrementSize + bufferSize;
            }
            oldEigs.assign(subspaceSize, 0.0);
            eigDiffs.assign(subspaceSize, 1.0);
            oldEigDiffs.assign(subspaceSize, 1.0);
        }
        if (!exitFlag && foundCount == 0 && applyCount >= maxInnerLoopCount) {
            // no progress possible within the iteration cap
            exitFlag = 1;
        }
    }

    // ---- non-monotone correction (:1835-1882): Rayleigh-Ritz over the found vectors
    bool nonMonotone = false;
    for (int64_t i = 0; i + 1 < foundSize_; ++i)
        if (eigValues_[i] > eigValues_[i + 1]) nonMonotone = true;
    if (nonMonotone) {
        tic(PH_EIG);
        // the found block must fit the working buffers: use W_/T1_/T2_ sized n x subspace >= found?
        if (foundSize_ > ss_cap_) RC_TRY(alloc(foundSize_, maxEigensystemDim));
        RC_TRY(copy_cols(ctx_, dtype_, E_, n_, V_, n_, n_, foundSize_));
        RC_TRY(rr(V_, W_, foundSize_, foundSize_, true));
        toc(PH_EIG);
        flush();
        RC_TRY(copy_cols(ctx_, dtype_, V_, n_, E_, n_, n_, foundSize_));
        eigValues_ = VtAVeigValue_;
        eigVecResiduals_ = subspaceResiduals_;
        count_opapply_ += 2 * foundSize_;
        count_eigenvalue_ += 1;
    }
    // ---- interval trim (:1890-1910)
    if (intervalStopConditionFlag) {
        const double rf = rel_err_factor(lambdaMax, subspaceTol);
        int64_t finalFoundCount = 0;
        for (double ev : eigValues_)
            if ((ev - lambdaMax) / rf < subspaceTol) finalFoundCount++;
        if (finalFoundCount < (int64_t)eigValues_.size()) {
            eigValues_.resize(finalFoundCount);
            eigVecResiduals_.resize(finalFoundCount);
            foundSize_ = finalFoundCount;
        }
    }
    return RC_OK;
}

// Entry points of RayleighChebyshevLMCuda: getMinEigenSystem (:775, :794) and
// getMinIntervalEigenSystem (:827, :876), selected by params.mode.
rc_status Solver::run(const void* v0, double* evals_out, void* evecs_out, double* resid_out, rc_solve_info* info) {
    if (P_.eig_count < 1 && (P_.mode == 0 || P_.mode == 1))
        return rc_fail(ctx_, RC_ERR_INVALID, "eig_count must be >= 1");
    if (P_.subspace_increment < 0 || P_.buffer_size < 0 || P_.subspace_increment + P_.buffer_size < 1)
        return rc_fail(ctx_, RC_ERR_INVALID, "subspace_increment + buffer_size must be >= 1");
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (P_.phase_timing) {
        cudaEventCreate(&t0);
        cudaEventCreate(&t1);
        cudaEventRecord(t0, ctx_->stream);
    }
    const int64_t launches0 = ctx_->launches;
    // degree-step timing for this solve only, switched off on every return path
    struct StepTimingScope {
        rc_ctx* c;
        ~StepTimingScope() {
            c->step_timing = false;
            c->step_events_used = 0;
        }
    } step_scope{ctx_};
    ctx_->step_timing = P_.phase_timing != 0;
    ctx_->step_events_used = 0;
    step_ms0_ = ctx_->step_ms;
    const double maxMinTol = P_.max_min_tol > 0 ? P_.max_min_tol : 1.0e-6;
    rc_status st = RC_OK;
    int64_t maxDim = P_.eig_count;
    double minEig = 0.0, maxEig = 0.0;
    switch (P_.mode) {
        case 0: {  // getMinEigenSystem(eigCount, tol, incr, buffer, ...) (:794-819)
            st = lanczos(1, maxMinTol, &minEig, &maxEig);
            if (st != RC_OK) break;
            if (std::fabs(maxEig - minEig) > 1.0e-12) maxEig += 0.001 * std::fabs(maxEig - minEig);
            st = base(minEig, maxEig, maxEig, maxDim, false, true, v0);
            break;
        }
        case 1: {  // getMinEigenSystem(eigCount, minEst, maxBound, ...) (:775-790)
            minEst_ = P_.min_eig_est;
            maxEst_ = P_.max_eig_bound;
            st = base(P_.min_eig_est, P_.max_eig_bound, P_.max_eig_bound, maxDim, false, true, v0);
            break;
        }
        case 2: {  // getMinIntervalEigenSystem(lambdaMax, ...) (:827-868)
            st = lanczos(0, maxMinTol, &minEig, &maxEig);
            if (st != RC_OK) break;
            if (P_.lambda_max < minEig) {
                eigValues_.clear();
                foundSize_ = 0;
                break;
            }
            if (std::fabs(maxEig - minEig) > 1.0e-12) maxEig += 0.001 * std::fabs(maxEig - minEig);
            st = base(minEig, P_.lambda_max, maxEig, maxDim > 0 ? maxDim : n_, true, false, v0);
            break;
        }
        case 3: {  // getMinIntervalEigenSystem(minEst, lambdaMax, maxBound, ...) (:876-886)
            minEst_ = P_.min_eig_est;
            maxEst_ = P_.max_eig_bound;
            st = base(P_.min_eig_est, P_.lambda_max, P_.max_eig_bound, maxDim > 0 ? maxDim : n_, true, false, v0);
            break;
        }
        default:
            st = rc_fail(ctx_, RC_ERR_INVALID, "unknown solve mode");
    }
    if (st != RC_OK) return st;
    // outputs: eigenvalues, eigenvectors (n x found, column-major), residuals
    const int64_t found = foundSize_;
    if (evals_out)
        for (int64_t i = 0; i < found; ++i) evals_out[i] = eigValues_[i];
    if (resid_out)
        for (int64_t i = 0; i < found; ++i) resid_out[i] = i < (int64_t)eigVecResiduals_.size() ? eigVecResiduals_[i] : 0.0;
    if (evecs_out && found > 0) {
        RC_CU(ctx_, cudaMemcpyAsync(evecs_out, E_, (size_t)n_ * found * esz_,
                                    P_.host_buffers ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, ctx_->stream));
    }
    if (P_.phase_timing) cudaEventRecord(t1, ctx_->stream);
    RC_CU(ctx_, cudaStreamSynchronize(ctx_->stream));
    flush();
    if (P_.phase_timing) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t0, t1);
        t_[PH_TOTAL] = ms;
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
    }
    if (info) {
        const size_t sz = info->struct_size ? info->struct_size : sizeof(rc_solve_info);
        rc_solve_info r;
        std::memset(&r, 0, sizeof(r));
        r.struct_size = sizeof(rc_solve_info);
        r.found = found;
        r.inner_iterations = inner_total_;
        r.outer_passes = outer_passes_;
        r.degree_steps = degree_steps_;
        r.fp64_degree_steps = fp64_steps_;
        r.mixed_iterations = mixed_iters_;
        r.lanczos_iterations = lanczos_iters_;
        r.cholqr_passes = cholqr_passes_;
        r.min_eig_est = minEst_;
        r.max_eig_est = maxEst_;
        r.max_residual = fd_maxResidual_;
        r.max_eig_diff = fd_maxEigDiff_;
        r.max_rel_gap = fd_maxGap_;
        r.count_ortho = count_ortho_;
        r.count_opapply = count_opapply_;
        r.count_eigenvalue = count_eigenvalue_;
        r.time_total_ms = t_[PH_TOTAL];
        r.time_lanczos_ms = t_[PH_LANCZOS];
        r.time_filter_ms = t_[PH_FILTER];
        r.time_ortho_ms = t_[PH_ORTHO];
        r.time_eigenvalue_ms = t_[PH_EIG];
        r.kernel_launches = ctx_->launches - launches0;
        r.guard_value = guardValue_;
        r.fused_rr = fused_ok_ + fused_fallback_;
        r.fused_rr_fallbacks = fused_fallback_;
        r.time_filter_steps_ms = ctx_->step_ms - step_ms0_;
        r.correction_iterations = corr_iters_;
        r.correction_degree_steps = corr_steps_;
        r.correction_element_bytes = (int64_t)corr_elem_bytes(dtype_);
        std::memcpy(info, &r, std::min(sz, sizeof(r)));
    }
    return RC_OK;
}

rc_status solve(rc_ctx* ctx, rc_op* op, const rc_solve_params& p, const void* v0, double* evals_out, void* evecs_out,
                double* resid_out, rc_solve_info* info) {
    Solver s(ctx, op, p);
    return s.run(v0, evals_out, evecs_out, resid_out, info);
}

}  // namespace rcb
