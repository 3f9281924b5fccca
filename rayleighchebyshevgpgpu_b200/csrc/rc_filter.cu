// rc_filter.cu -- fused operator step and the Lanczos "C" polynomial filter.
//
// One kernel launch is one degree-step of the three-term recurrence of
// LanczosCpolyOperatorLMCuda::apply (LanczosCpolyOperatorLMCuda.h:194-265):
//
//     x_k = gamma2*(gamma1*A*x_{k-1} + x_{k-1}) - x_{k-2}
//
// which the reference issues as a device memcpy, a user SpMM (out = a*A*in + b*out) and a
// `substract` kernel per step (:243-247) plus a final `scale` kernel (:259), about 7 block
// passes per step. Here the step is one pass over the n x s block: each thread owns one
// row, keeps that row's matrix entries in L1/registers, and for every column chunk gathers
// the neighbour rows of x_{k-1}, adds beta*x_{k-1} and gamma*x_{k-2} and writes x_k over
// x_{k-2} (in place), scaling by 1/(m+1) on the last step. HBM traffic per step is
// read x_{k-1} + read x_{k-2} + write x_k + the matrix (CSR) or the diagonal (stencil).
//
// Column-major blocks (ld >= n) keep the reference's AmatrixClassLMCuda layout, so warps
// read 32 consecutive rows of one column: every gather of a banded/stencil matrix is a
// coalesced 128-byte (FP32) or 256-byte (FP64) segment.
#include <cstdio>
#include <string>
#include <type_traits>
#include "rc_common.cuh"
#include "rc_internal.h"

namespace rcb {

template <class T> struct Cpx { using type = T; };
// storage scalar for (precision, complex?)
template <int P, bool C> struct Stor;
template <> struct Stor<P64, false> { using type = double; };
template <> struct Stor<P32, false> { using type = float; };
template <> struct Stor<P64, true> { using type = double2; };
template <> struct Stor<P32, true> { using type = float2; };

constexpr int kStepThreads = 256;
// Resident CTAs per SM the register budget of the real FP64 register-cached CSR step must allow: 4 (64
// registers). W = A V on 128^3 x 96 FP64 takes 1.17 ms at 4, 1.64 ms at 3 and 1.45 ms unbounded.
// The other scalar types (wider column chunks, complex) would spill at 64 and stay unbounded.
#ifndef RC_CM_MIN_BLOCKS
#define RC_CM_MIN_BLOCKS 4
#endif
template <class TC>
constexpr int cm_min_blocks() {
    return std::is_same<TC, double>::value ? RC_CM_MIN_BLOCKS : 1;
}

// ---------------------------------------------------------------------------------------
// CSR step
// ---------------------------------------------------------------------------------------
template <class TA, class TX, class TZ, class TY, class TC, int CB>
__global__ void __launch_bounds__(kStepThreads)
csr_step_kernel(int64_t n, int64_t s, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ colind,
                const TA* __restrict__ vals, const TX* __restrict__ x, int64_t ldx, const TZ* z, int64_t ldz,
                TY* y, int64_t ldy, TC alpha, TC beta, TC gamma, real_t<TC> scale) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k0 = __ldg(rowptr + i), k1 = __ldg(rowptr + i + 1);
    for (int64_t c0 = 0; c0 < s; c0 += CB) {
        const int nb = (int)((s - c0) < CB ? (s - c0) : CB);
        TC acc[CB];
#pragma unroll
        for (int cc = 0; cc < CB; ++cc) acc[cc] = s_zero(TC());
        const TX* xc = x + c0 * ldx;
        for (int k = k0; k < k1; ++k) {
            const int64_t j = __ldg(colind + k);
            const TC a = s_cvt<TC>(vals[k]);
            if (nb == CB) {
#pragma unroll
                for (int cc = 0; cc < CB; ++cc) acc[cc] = s_fma(a, s_cvt<TC>(xc[j + cc * ldx]), acc[cc]);
            } else {
#pragma unroll
                for (int cc = 0; cc < CB; ++cc)
                    if (cc < nb) acc[cc] = s_fma(a, s_cvt<TC>(xc[j + cc * ldx]), acc[cc]);
            }
        }
#pragma unroll
        for (int cc = 0; cc < CB; ++cc) {
            if (cc < nb) {
                const int64_t c = c0 + cc;
                TC v = s_mul(alpha, acc[cc]);
                v = s_fma(beta, s_cvt<TC>(x[i + c * ldx]), v);
                if (z) v = s_fma(gamma, s_cvt<TC>(z[i + c * ldz]), v);
                y[i + c * ldy] = s_cvt<TY>(s_rscale(scale, v));
            }
        }
    }
}

// Rows with at most MAXR entries: the row's (column, value) pairs are loaded once into
// registers (padded with (i, 0)), so the MAXR x CB gathers of a column chunk are independent
// loads the hardware keeps in flight together.
template <class TA, class TX, class TZ, class TY, class TC, int CB, int MAXR>
__global__ void __launch_bounds__(kStepThreads, cm_min_blocks<TC>())
csr_step_reg_kernel(int64_t n, int64_t s, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ colind,
                    const TA* __restrict__ vals, const TX* __restrict__ x, int64_t ldx, const TZ* z, int64_t ldz,
                    TY* y, int64_t ldy, TC alpha, TC beta, TC gamma, real_t<TC> scale) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k0 = __ldg(rowptr + i), k1 = __ldg(rowptr + i + 1);
    const int cnt = k1 - k0;
    int js[MAXR];
    TC as[MAXR];
#pragma unroll
    for (int r = 0; r < MAXR; ++r) {
        const bool ok = r < cnt;
        js[r] = ok ? __ldg(colind + k0 + r) : (int)i;
        as[r] = ok ? s_cvt<TC>(vals[k0 + r]) : s_zero(TC());
    }
    for (int64_t c0 = 0; c0 < s; c0 += CB) {
        const int nb = (int)((s - c0) < CB ? (s - c0) : CB);
        TC acc[CB];
#pragma unroll
        for (int cc = 0; cc < CB; ++cc) acc[cc] = s_zero(TC());
        const TX* xc = x + c0 * ldx;
        if (nb == CB) {
#pragma unroll
            for (int r = 0; r < MAXR; ++r)
#pragma unroll
                for (int cc = 0; cc < CB; ++cc) acc[cc] = s_fma(as[r], s_cvt<TC>(xc[js[r] + cc * ldx]), acc[cc]);
        } else {
#pragma unroll
            for (int r = 0; r < MAXR; ++r)
#pragma unroll
                for (int cc = 0; cc < CB; ++cc)
                    if (cc < nb) acc[cc] = s_fma(as[r], s_cvt<TC>(xc[js[r] + cc * ldx]), acc[cc]);
        }
#pragma unroll
        for (int cc = 0; cc < CB; ++cc) {
            if (cc < nb) {
                const int64_t c = c0 + cc;
                TC v = s_mul(alpha, acc[cc]);
                v = s_fma(beta, s_cvt<TC>(x[i + c * ldx]), v);
                if (z) v = s_fma(gamma, s_cvt<TC>(z[i + c * ldz]), v);
                y[i + c * ldy] = s_cvt<TY>(s_rscale(scale, v));
            }
        }
    }
}

// ---------------------------------------------------------------------------------------
// Stencil step (matrix-free, Dirichlet boundaries)
//   (A v)_i = diag[i]*v_i + offdiag * sum_j phase(i,j) v_j
// KIND 5: 2D 5-point (nz = 1); 7: 3D 7-point; 27: 3D 27-point (real only).
// Complex y-bonds carry exp(+i*theta*x) on (x,y+1)<-(x,y) and the conjugate on the reverse.
// ---------------------------------------------------------------------------------------
template <class TX> struct PhaseOf { using type = TX; };

template <class TC> __device__ __forceinline__ TC phase_val(double theta_x, bool conj_);
template <> __device__ __forceinline__ double phase_val<double>(double, bool) { return 1.0; }
template <> __device__ __forceinline__ float phase_val<float>(double, bool) { return 1.0f; }
template <> __device__ __forceinline__ double2 phase_val<double2>(double t, bool cj) {
    double sn, cs;
    sincos(t, &sn, &cs);
    return make_double2(cs, cj ? -sn : sn);
}
template <> __device__ __forceinline__ float2 phase_val<float2>(double t, bool cj) {
    double sn, cs;
    sincos(t, &sn, &cs);
    return make_float2((float)cs, (float)(cj ? -sn : sn));
}

template <class TD, class TX, class TZ, class TY, class TC, int KIND, int CB>
__global__ void __launch_bounds__(kStepThreads)
stencil_step_kernel(int64_t nx, int64_t ny, int64_t nz, RowDiv dnx, RowDiv dny, int64_t s,
                    const TD* __restrict__ diag, real_t<TC> offd, double theta, const TX* __restrict__ x, int64_t ldx,
                    const TZ* z, int64_t ldz, TY* y, int64_t ldy, TC alpha, TC beta, TC gamma, real_t<TC> scale) {
    const int64_t n = nx * ny * nz;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t t = dnx.div(i);
    const int64_t ix = i - t * nx;
    const int64_t iz = dny.div(t);
    const int64_t iy = t - iz * ny;
    const int64_t sy = nx, sz = nx * ny;
    const real_t<TC> d = (real_t<TC>)diag[i];
    constexpr bool kCplx = IsComplex<TC>::value;
    TC ph = s_zero(TC()), phc = s_zero(TC());
    if (kCplx) {
        ph = phase_val<TC>(theta * (double)ix, false);   // entry (x,y)<-(x,y-1)
        phc = phase_val<TC>(theta * (double)ix, true);   // entry (x,y)<-(x,y+1)
    }
    // neighbour validity
    const bool xm = ix > 0, xp = ix + 1 < nx, ym = iy > 0, yp = iy + 1 < ny, zm = iz > 0, zp = iz + 1 < nz;
    for (int64_t c0 = 0; c0 < s; c0 += CB) {
        const int nb = (int)((s - c0) < CB ? (s - c0) : CB);
#pragma unroll
        for (int cc = 0; cc < CB; ++cc) {
            if (cc >= nb) break;
            const int64_t c = c0 + cc;
            const TX* xc = x + c * ldx + i;
            const TC xi = s_cvt<TC>(xc[0]);
            TC nsum = s_zero(TC());
            if (KIND == 27) {
#pragma unroll
                for (int dz = -1; dz <= 1; ++dz) {
                    const bool vz = dz < 0 ? zm : (dz > 0 ? zp : true);
#pragma unroll
                    for (int dy = -1; dy <= 1; ++dy) {
                        const bool vy = dy < 0 ? ym : (dy > 0 ? yp : true);
#pragma unroll
                        for (int dx = -1; dx <= 1; ++dx) {
                            if (dx == 0 && dy == 0 && dz == 0) continue;
                            const bool vx = dx < 0 ? xm : (dx > 0 ? xp : true);
                            if (vx && vy && vz) nsum = s_add(nsum, s_cvt<TC>(xc[dx + dy * sy + dz * sz]));
                        }
                    }
                }
            } else {
                if (xm) nsum = s_add(nsum, s_cvt<TC>(xc[-1]));
                if (xp) nsum = s_add(nsum, s_cvt<TC>(xc[1]));
                if (kCplx) {
                    if (ym) nsum = s_fma(ph, s_cvt<TC>(xc[-sy]), nsum);
                    if (yp) nsum = s_fma(phc, s_cvt<TC>(xc[sy]), nsum);
                } else {
                    if (ym) nsum = s_add(nsum, s_cvt<TC>(xc[-sy]));
                    if (yp) nsum = s_add(nsum, s_cvt<TC>(xc[sy]));
                }
                if (KIND == 7) {
                    if (zm) nsum = s_add(nsum, s_cvt<TC>(xc[-sz]));
                    if (zp) nsum = s_add(nsum, s_cvt<TC>(xc[sz]));
                }
            }
            TC ax = s_add(s_rscale(d, xi), s_rscale(offd, nsum));
            TC v = s_mul(alpha, ax);
            v = s_fma(beta, xi, v);
            if (z) v = s_fma(gamma, s_cvt<TC>(z[i + c * ldz]), v);
            y[i + c * ldy] = s_cvt<TY>(s_rscale(scale, v));
        }
    }
}

// ---------------------------------------------------------------------------------------
// Dispatch
// ---------------------------------------------------------------------------------------
template <bool CPLX, int CP, int XP, int ZP, int YP>
static rc_status launch_step_t(rc_ctx* ctx, rc_op* op, const StepArgs& a) {
    using TC = typename Stor<CP, CPLX>::type;
    using TX = typename Stor<XP, CPLX>::type;
    using TZ = typename Stor<ZP, CPLX>::type;
    using TY = typename Stor<YP, CPLX>::type;
    using R = real_t<TC>;
    const TC alpha = s_from<TC>(a.alpha[0], a.alpha[1]);
    const TC beta = s_from<TC>(a.beta[0], a.beta[1]);
    const TC gamma = s_from<TC>(a.gamma[0], a.gamma[1]);
    const R scale = (R)a.scale;
    const int64_t n = op->n;
    const unsigned grid = (unsigned)((n + kStepThreads - 1) / kStepThreads);
    const TX* x = (const TX*)a.x;
    const TZ* z = (const TZ*)a.z;
    TY* y = (TY*)a.y;
    constexpr int CB = CPLX ? 4 : 8;
    // register-cached rows: fewer columns per chunk for the wider scalars keeps registers in check
    constexpr int CBR = sizeof(TC) >= 16 ? 2 : (sizeof(TC) == 8 ? 4 : 8);
    if (op->kind == 0) {
        using TA = typename Stor<CP, CPLX>::type;
        const TA* vals = (const TA*)(CP == P64 ? op->vals64 : op->vals32);
        const bool reg = ctx->csr_variant == 0 ? op->max_row_nnz <= 8 : (ctx->csr_variant == 2 && op->max_row_nnz <= 8);
        if (reg)
            csr_step_reg_kernel<TA, TX, TZ, TY, TC, CBR, 8><<<grid, kStepThreads, 0, ctx->stream>>>(
                n, a.s, op->rowptr, op->colind, vals, x, a.ldx, z, a.ldz, y, a.ldy, alpha, beta, gamma, scale);
        else
            csr_step_kernel<TA, TX, TZ, TY, TC, CB><<<grid, kStepThreads, 0, ctx->stream>>>(
                n, a.s, op->rowptr, op->colind, vals, x, a.ldx, z, a.ldz, y, a.ldy, alpha, beta, gamma, scale);
    } else {
        const double theta = 2.0 * 3.14159265358979323846 * op->flux;
        const R offd = (R)op->offdiag;
        const RowDiv dnx(op->nx), dny(op->ny);
        if (CP == P64) {
            const double* dg = op->diag64;
            if (op->skind == 27)
                stencil_step_kernel<double, TX, TZ, TY, TC, 27, CB><<<grid, kStepThreads, 0, ctx->stream>>>(
                    op->nx, op->ny, op->nz, dnx, dny, a.s, dg, offd, theta, x, a.ldx, z, a.ldz, y, a.ldy, alpha, beta,
                    gamma, scale);
            else if (op->skind == 7)
                stencil_step_kernel<double, TX, TZ, TY, TC, 7, CB><<<grid, kStepThreads, 0, ctx->stream>>>(
                    op->nx, op->ny, op->nz, dnx, dny, a.s, dg, offd, theta, x, a.ldx, z, a.ldz, y, a.ldy, alpha, beta,
                    gamma, scale);
            else
                stencil_step_kernel<double, TX, TZ, TY, TC, 5, CB><<<grid, kStepThreads, 0, ctx->stream>>>(
                    op->nx, op->ny, op->nz, dnx, dny, a.s, dg, offd, theta, x, a.ldx, z, a.ldz, y, a.ldy, alpha, beta,
                    gamma, scale);
        } else {
            const float* dg = op->diag32;
            if (op->skind == 27)
                stencil_step_kernel<float, TX, TZ, TY, TC, 27, CB><<<grid, kStepThreads, 0, ctx->stream>>>(
                    op->nx, op->ny, op->nz, dnx, dny, a.s, dg, offd, theta, x, a.ldx, z, a.ldz, y, a.ldy, alpha, beta,
                    gamma, scale);
            else if (op->skind == 7)
                stencil_step_kernel<float, TX, TZ, TY, TC, 7, CB><<<grid, kStepThreads, 0, ctx->stream>>>(
                    op->nx, op->ny, op->nz, dnx, dny, a.s, dg, offd, theta, x, a.ldx, z, a.ldz, y, a.ldy, alpha, beta,
                    gamma, scale);
            else
                stencil_step_kernel<float, TX, TZ, TY, TC, 5, CB><<<grid, kStepThreads, 0, ctx->stream>>>(
                    op->nx, op->ny, op->nz, dnx, dny, a.s, dg, offd, theta, x, a.ldx, z, a.ldz, y, a.ldy, alpha, beta,
                    gamma, scale);
        }
    }
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    return RC_OK;
}

template <bool CPLX, int CP>
static rc_status launch_step_c(rc_ctx* ctx, rc_op* op, const StepArgs& a) {
    const int code = a.xp * 4 + a.zp * 2 + a.yp;
    switch (code) {
        case 0: return launch_step_t<CPLX, CP, P64, P64, P64>(ctx, op, a);
        case 1: return launch_step_t<CPLX, CP, P64, P64, P32>(ctx, op, a);
        case 2: return launch_step_t<CPLX, CP, P64, P32, P64>(ctx, op, a);
        case 3: return launch_step_t<CPLX, CP, P64, P32, P32>(ctx, op, a);
        case 4: return launch_step_t<CPLX, CP, P32, P64, P64>(ctx, op, a);
        case 5: return launch_step_t<CPLX, CP, P32, P64, P32>(ctx, op, a);
        case 6: return launch_step_t<CPLX, CP, P32, P32, P64>(ctx, op, a);
        default: return launch_step_t<CPLX, CP, P32, P32, P32>(ctx, op, a);
    }
}

void step_mark(rc_ctx* ctx) {
    if (!ctx->step_timing) return;
    if (ctx->step_events_used == ctx->step_events.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return;
        ctx->step_events.push_back(e);
    }
    cudaEventRecord(ctx->step_events[ctx->step_events_used++], ctx->stream);
}

void step_flush(rc_ctx* ctx) {
    // events come in (begin, end) pairs, one pair per degree-step loop
    for (size_t i = 0; i + 1 < ctx->step_events_used; i += 2) {
        float ms = 0.f;
        cudaEventSynchronize(ctx->step_events[i + 1]);
        if (cudaEventElapsedTime(&ms, ctx->step_events[i], ctx->step_events[i + 1]) == cudaSuccess)
            ctx->step_ms += ms;
    }
    ctx->step_events_used = 0;
}

// Build the FP32 copy of the operator's values on first use.
__global__ void cvt_f64_f32_kernel(const double* __restrict__ a, float* __restrict__ b, int64_t count) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

rc_status ensure_fp32(rc_ctx* ctx, rc_op* op) {
    if (op->kind == 0 && op->vals32 == nullptr) {
        const int64_t cnt = op->nnz * (op->dtype == RC_COMPLEX128 ? 2 : 1);
        void* p = nullptr;
        if (cudaMalloc(&p, (size_t)cnt * 4 + 64) != cudaSuccess)  // tail padding as the other operator arrays
            return rc_fail(ctx, RC_ERR_NOMEM, "cudaMalloc failed for FP32 operator values");
        cvt_f64_f32_kernel<<<4 * kB200Sms, 256, 0, ctx->stream>>>((const double*)op->vals64, (float*)p, cnt);
        ctx->launches++;
        RC_CU(ctx, cudaGetLastError());
        op->vals32 = p;
        op->bytes += cnt * 4;
        ctx->op_bytes += cnt * 4;
    }
    if (op->kind == 1 && op->diag32 == nullptr) {
        void* p = nullptr;
        if (cudaMalloc(&p, (size_t)op->n * 4 + 64) != cudaSuccess)
            return rc_fail(ctx, RC_ERR_NOMEM, "cudaMalloc failed for FP32 stencil diagonal");
        cvt_f64_f32_kernel<<<4 * kB200Sms, 256, 0, ctx->stream>>>(op->diag64, (float*)p, op->n);
        ctx->launches++;
        RC_CU(ctx, cudaGetLastError());
        op->diag32 = (float*)p;
        op->bytes += op->n * 4;
        ctx->op_bytes += op->n * 4;
    }
    return RC_OK;
}

// Elementwise y = scale*(beta*x + gamma*z) used to complete a callback step.
template <class T>
__global__ void combine_kernel(int64_t n, int64_t s, const T* Ax, int64_t lda, T alpha, const T* x, int64_t ldx,
                               T beta, const T* z, int64_t ldz, T gamma, T* y, int64_t ldy, double scale) {
    const int64_t total = n * s;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e % n, c = e / n;
        T v = s_mul(alpha, Ax[i + c * lda]);
        v = s_fma(beta, x[i + c * ldx], v);
        if (z) v = s_fma(gamma, z[i + c * ldz], v);
        y[i + c * ldy] = s_rscale(scale, v);
    }
}

rc_status op_step(rc_ctx* ctx, rc_op* op, const StepArgs& a) {
    if (a.s <= 0) return RC_OK;
    const bool cplx = op->dtype == RC_COMPLEX128;
    if (op->kind == 2) {
        // Foreign operator: FP64 only; Ax = A*x via the callback into scratch, then combine.
        if (a.xp != P64 || a.yp != P64 || (a.z && a.zp != P64))
            return rc_fail(ctx, RC_ERR_UNSUPPORTED, "callback operators run the FP64 filter only");
        void* tmp = nullptr;
        RC_TRY(rc_slot(ctx, S_CB, (size_t)op->n * a.s * elem_bytes(op->dtype, P64), &tmp));
        const double one[2] = {1, 0}, zero[2] = {0, 0};
        if (op->fn(op->user, a.x, tmp, op->n, a.s, op->n, one, zero, (void*)ctx->stream) != 0)
            return rc_fail(ctx, RC_ERR_CALLBACK, "operator callback returned an error");
        const unsigned g = 4 * kB200Sms;
        if (cplx)
            combine_kernel<double2><<<g, 256, 0, ctx->stream>>>(
                op->n, a.s, (const double2*)tmp, op->n, make_double2(a.alpha[0], a.alpha[1]), (const double2*)a.x,
                a.ldx, make_double2(a.beta[0], a.beta[1]), (const double2*)a.z, a.ldz,
                make_double2(a.gamma[0], a.gamma[1]), (double2*)a.y, a.ldy, a.scale);
        else
            combine_kernel<double><<<g, 256, 0, ctx->stream>>>(op->n, a.s, (const double*)tmp, op->n, a.alpha[0],
                                                               (const double*)a.x, a.ldx, a.beta[0],
                                                               (const double*)a.z, a.ldz, a.gamma[0],
                                                               (double*)a.y, a.ldy, a.scale);
        ctx->launches++;
        RC_CU(ctx, cudaGetLastError());
        return RC_OK;
    }
    if (a.cp == P32) RC_TRY(ensure_fp32(ctx, op));
    if (op->kind == 1 && op->skind == 27 && cplx)
        return rc_fail(ctx, RC_ERR_UNSUPPORTED, "27-point stencil is real only");
    if (cplx) return a.cp == P64 ? launch_step_c<true, P64>(ctx, op, a) : launch_step_c<true, P32>(ctx, op, a);
    return a.cp == P64 ? launch_step_c<false, P64>(ctx, op, a) : launch_step_c<false, P32>(ctx, op, a);
}

// ---------------------------------------------------------------------------------------
// Filter driver: the recurrence of LanczosCpolyOperatorLMCuda::apply with the result left in V.
// Native operators with degree >= 2 run the row-major pipeline of rc_filter_rm.cu in the
// two scratch blocks (tmp1, tmp2 of tmp_bytes each, or context slots when too small).
// Foreign (callback) operators and degree 1 use the column-major steps below:
//  FP64:  buffers V (x0) and one temporary; x_k overwrites x_{k-2}.
//  MIXED: x_1..x_{m-1} in two FP32 blocks carved from `tmp1`; x_0 read from V (FP64), x_m
//         written to V (FP64) with the 1/(m+1) scale.
// ---------------------------------------------------------------------------------------
rc_status rm_filter(rc_ctx* ctx, rc_op* op, void* V, int64_t ldv, int64_t s, int64_t degree, double a, double b,
                    int prec, void* bufA, void* bufB);
int64_t rm_leading_dim(int dtype, int prec, int64_t s);

rc_status filter_apply(rc_ctx* ctx, rc_op* op, void* V, int64_t ld, int64_t s, int64_t degree, int64_t rep,
                       double a, double b, int prec, void* tmp1, void* tmp2, size_t tmp_bytes,
                       int64_t* steps_done) {
    if (degree < 1 || rep < 1 || s < 1) return RC_OK;
    if (op->kind != 2 && degree >= 2) {
        const int p = prec == RC_PREC_MIXED ? P32 : P64;
        const size_t need = (size_t)op->n * rm_leading_dim(op->dtype, p, s) * elem_bytes(op->dtype, p);
        void* bufA = tmp1;
        void* bufB = tmp2;
        if (!bufA || tmp_bytes < need) RC_TRY(rc_slot(ctx, S_FA, need, &bufA));
        if (!bufB || tmp_bytes < need) RC_TRY(rc_slot(ctx, S_FB, need, &bufB));
        if (p == P32) RC_TRY(ensure_fp32(ctx, op));
        for (int64_t r = 0; r < rep; ++r) {
            bool handled = false;
            if (ctx->serve) RC_TRY(serve_filter(ctx, op, V, ld, s, degree, a, b, prec, bufA, bufB, need, &handled));
            if (!handled) RC_TRY(rm_filter(ctx, op, V, ld, s, degree, a, b, prec, bufA, bufB));
        }
        if (steps_done) *steps_done += degree * rep;
        return RC_OK;
    }
    void* tmp = tmp1;
    if (!tmp || tmp_bytes < (size_t)op->n * s * elem_bytes(op->dtype, P64))
        RC_TRY(rc_slot(ctx, S_FA, (size_t)op->n * s * elem_bytes(op->dtype, P64), &tmp));
    const int64_t n = op->n;
    const bool cplx = op->dtype == RC_COMPLEX128;
    if (op->kind == 2) prec = RC_PREC_FP64;
    const double scale_last = 1.0 / (double)(degree + 1);
    int64_t steps = 0;
    for (int64_t r = 0; r < rep; ++r) {
        if (prec == RC_PREC_FP64) {
            void* bufs[2] = {V, tmp};  // x_k lives in bufs[k % 2]
            // x1 = g2*(g1*A x0 + x0) -> tmp
            StepArgs st;
            st.s = s;
            st.x = V; st.xp = P64; st.ldx = ld;
            st.y = tmp; st.yp = P64; st.ldy = n;
            st.alpha[0] = a; st.beta[0] = b;
            st.scale = degree == 1 ? scale_last : 1.0;
            st.cp = P64;
            RC_TRY(op_step(ctx, op, st));
            ++steps;
            for (int64_t k = 2; k <= degree; ++k) {
                StepArgs sk;
                sk.s = s;
                sk.x = bufs[(k - 1) % 2]; sk.xp = P64; sk.ldx = ((k - 1) % 2 == 0) ? ld : n;
                sk.z = bufs[k % 2]; sk.zp = P64; sk.ldz = (k % 2 == 0) ? ld : n;
                sk.y = bufs[k % 2]; sk.yp = P64; sk.ldy = sk.ldz;
                sk.alpha[0] = a; sk.beta[0] = b; sk.gamma[0] = -1.0;
                sk.scale = k == degree ? scale_last : 1.0;
                sk.cp = P64;
                RC_TRY(op_step(ctx, op, sk));
                ++steps;
            }
            if (degree % 2 == 1) {  // result in tmp: copy back into V
                RC_TRY(copy_cols(ctx, op->dtype, tmp, n, V, ld, n, s));
            }
        } else {
            const size_t half = (size_t)n * s * elem_bytes(op->dtype, P32);
            void* p32[2] = {tmp, (char*)tmp + half};  // x_k (1 <= k < m) lives in p32[(k-1) % 2]
            if (degree == 1) {
                // x1 needs neighbours of x0 = V, so it cannot overwrite V: FP64 result into tmp then copy.
                StepArgs st;
                st.s = s;
                st.x = V; st.xp = P64; st.ldx = ld;
                st.y = tmp; st.yp = P64; st.ldy = n;
                st.alpha[0] = a; st.beta[0] = b; st.scale = scale_last; st.cp = P32;
                RC_TRY(op_step(ctx, op, st));
                RC_TRY(copy_cols(ctx, op->dtype, tmp, n, V, ld, n, s));
                ++steps;
                continue;
            }
            {
                StepArgs st;
                st.s = s;
                st.x = V; st.xp = P64; st.ldx = ld;
                st.y = p32[0]; st.yp = P32; st.ldy = n;
                st.alpha[0] = a; st.beta[0] = b; st.cp = P32;
                RC_TRY(op_step(ctx, op, st));
                ++steps;
            }
            for (int64_t k = 2; k <= degree; ++k) {
                StepArgs sk;
                sk.s = s;
                sk.x = p32[(k - 2) % 2]; sk.xp = P32; sk.ldx = n;  // x_{k-1}
                if (k == 2) {
                    sk.z = V; sk.zp = P64; sk.ldz = ld;  // x_0
                } else {
                    sk.z = p32[(k - 3) % 2]; sk.zp = P32; sk.ldz = n;  // x_{k-2}
                }
                if (k == degree) {
                    sk.y = V; sk.yp = P64; sk.ldy = ld;
                    sk.scale = scale_last;
                } else {
                    sk.y = p32[(k - 1) % 2]; sk.yp = P32; sk.ldy = n;  // == x_{k-2}'s slot for k>=3
                }
                sk.alpha[0] = a; sk.beta[0] = b; sk.gamma[0] = -1.0;
                sk.cp = P32;
                RC_TRY(op_step(ctx, op, sk));
                ++steps;
            }
        }
    }
    (void)cplx;
    if (steps_done) *steps_done += steps;
    return RC_OK;
}

}  // namespace rcb
