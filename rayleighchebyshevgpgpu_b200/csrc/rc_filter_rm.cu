// rc_filter_rm.cu -- the Chebyshev filter with row-major intermediates.
//
// The recurrence of LanczosCpolyOperatorLMCuda::apply (LanczosCpolyOperatorLMCuda.h:194-265)
//   x1 = a*A*x0 + b*x0,   x_k = a*A*x_{k-1} + b*x_{k-1} - x_{k-2},   X = x_m/(m+1)
// with a = gamma2*gamma1 and b = gamma2. The caller's block X (x0 in, x_m out) stays
// column-major (the AmatrixClassLMCuda layout). The intermediates x1..x_{m-1} live in two
// row-major scratch blocks (row i = the s values x(i, 0..s-1), leading dimension ld), so a
// neighbour row is one contiguous run and each thread of the middle steps owns a 16-byte slice
// of a row: every gather is a coalesced 128-bit load, and the matrix entries of a row are
// broadcast to the threads of that row.
//   step 1     (cm2rm): X column-major -> x1 row-major, plus a row-major copy of x0
//   step k<m   (rm):    x_k over x_{k-2}, both row-major (one pass: read x_{k-1}, x_{k-2}, write x_k)
//   step m     (rm2cm): x_m (scaled by 1/(m+1)) into X column-major
// Storage/compute: FP32 (c64) in MIXED precision, FP64 (c128) otherwise.
#include <cstring>
#include "rc_common.cuh"
#include "rc_internal.h"
#include "rc_rowops.cuh"

namespace rcb {

template <class TS>
struct alignas(16) Pack16 {
    static constexpr int V = 16 / sizeof(TS);
    TS v[V];
};

template <class TS>
__device__ __forceinline__ Pack16<TS> ld16_ro(const TS* p) {
    const uint4 u = __ldg(reinterpret_cast<const uint4*>(p));
    Pack16<TS> r;
    memcpy(&r, &u, 16);
    return r;
}
template <class TS>
__device__ __forceinline__ Pack16<TS> ld16(const TS* p) {
    const uint4 u = *reinterpret_cast<const uint4*>(p);
    Pack16<TS> r;
    memcpy(&r, &u, 16);
    return r;
}
template <class TS>
__device__ __forceinline__ void st16(TS* p, const Pack16<TS>& v) {
    uint4 u;
    memcpy(&u, &v, 16);
    *reinterpret_cast<uint4*>(p) = u;
}

constexpr int kRmThreads = 256;

// Middle step: thread t -> row i = t / nseg, slice seg = t % nseg (V = 16/sizeof(TS) columns).
template <class Pol, class TS, class TC>
__global__ void __launch_bounds__(kRmThreads)
rm_step_kernel(Pol op, int64_t n, int nseg, int64_t ld, const TS* __restrict__ x, const TS* z, TS* y, TC alpha,
               TC beta, TC gamma) {
    constexpr int V = Pack16<TS>::V;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t i = t / nseg;
    if (i >= n) return;
    const int64_t off = (t - i * nseg) * V;
    TC acc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) acc[v] = s_zero(TC());
    op.row(i, [&](int64_t j, TC a) {
        const Pack16<TS> p = ld16_ro(x + j * ld + off);
#pragma unroll
        for (int v = 0; v < V; ++v) acc[v] = s_fma(a, s_cvt<TC>(p.v[v]), acc[v]);
    });
    const Pack16<TS> xi = ld16_ro(x + i * ld + off);
    const Pack16<TS> zi = ld16(z + i * ld + off);
    Pack16<TS> out;
#pragma unroll
    for (int v = 0; v < V; ++v) {
        TC r = s_mul(alpha, acc[v]);
        r = s_fma(beta, s_cvt<TC>(xi.v[v]), r);
        r = s_fma(gamma, s_cvt<TC>(zi.v[v]), r);
        out.v[v] = s_cvt<TS>(r);
    }
    st16(y + i * ld + off, out);
}

// First step: one thread per row, CB columns per pass; reads the column-major input.
template <class Pol, class TX, class TS, class TC, int CB>
__global__ void __launch_bounds__(kRmThreads)
cm2rm_step_kernel(Pol op, int64_t n, int64_t s, const TX* __restrict__ x, int64_t ldx, TS* __restrict__ y,
                  TS* __restrict__ x0c, int64_t ld, TC alpha, TC beta) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int64_t c0 = 0; c0 < s; c0 += CB) {
        const int nb = (int)((s - c0) < CB ? (s - c0) : CB);
        TC acc[CB];
#pragma unroll
        for (int cc = 0; cc < CB; ++cc) acc[cc] = s_zero(TC());
        const TX* xc = x + c0 * ldx;
        op.row(i, [&](int64_t j, TC a) {
#pragma unroll
            for (int cc = 0; cc < CB; ++cc)
                if (cc < nb) acc[cc] = s_fma(a, s_cvt<TC>(xc[j + cc * ldx]), acc[cc]);
        });
#pragma unroll
        for (int cc = 0; cc < CB; ++cc) {
            if (cc < nb) {
                const TC xv = s_cvt<TC>(xc[i + cc * ldx]);
                TC r = s_mul(alpha, acc[cc]);
                r = s_fma(beta, xv, r);
                y[i * ld + c0 + cc] = s_cvt<TS>(r);
                x0c[i * ld + c0 + cc] = s_cvt<TS>(xv);
            }
        }
    }
}

// Last step: one thread per row; gathers row-major slices, writes the column-major output.
template <class Pol, class TS, class TY, class TC, int CB>
__global__ void __launch_bounds__(kRmThreads)
rm2cm_step_kernel(Pol op, int64_t n, int64_t s, int64_t ld, const TS* __restrict__ x, const TS* __restrict__ z,
                  TY* __restrict__ y, int64_t ldy, TC alpha, TC beta, TC gamma, real_t<TC> scale) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int64_t c0 = 0; c0 < s; c0 += CB) {
        const int nb = (int)((s - c0) < CB ? (s - c0) : CB);
        TC acc[CB];
#pragma unroll
        for (int cc = 0; cc < CB; ++cc) acc[cc] = s_zero(TC());
        op.row(i, [&](int64_t j, TC a) {
            const TS* xr = x + j * ld + c0;
#pragma unroll
            for (int cc = 0; cc < CB; ++cc)
                if (cc < nb) acc[cc] = s_fma(a, s_cvt<TC>(xr[cc]), acc[cc]);
        });
#pragma unroll
        for (int cc = 0; cc < CB; ++cc) {
            if (cc < nb) {
                TC r = s_mul(alpha, acc[cc]);
                r = s_fma(beta, s_cvt<TC>(x[i * ld + c0 + cc]), r);
                r = s_fma(gamma, s_cvt<TC>(z[i * ld + c0 + cc]), r);
                y[i + (c0 + cc) * ldy] = s_cvt<TY>(s_rscale(scale, r));
            }
        }
    }
}

// ---------------------------------------------------------------------------------------
// Driver
// ---------------------------------------------------------------------------------------
template <class Pol, class TS, class TC>
static rc_status run_rm_filter(rc_ctx* ctx, const Pol& pol, int64_t n, void* V, int64_t ldv, int64_t s,
                               int64_t degree, double a, double b, void* bufA, void* bufB, int64_t ld) {
    using TY = typename std::conditional<IsComplex<TC>::value, double2, double>::type;
    using R = real_t<TC>;
    constexpr int VEC = Pack16<TS>::V;
    constexpr int CB = sizeof(TS) >= 16 ? 2 : (sizeof(TS) == 8 ? 4 : 8);
    const TC ta = s_from<TC>(a, 0.0), tb = s_from<TC>(b, 0.0), tm1 = s_from<TC>(-1.0, 0.0);
    const unsigned grid_rows = (unsigned)((n + kRmThreads - 1) / kRmThreads);
    const int nseg = (int)(ld / VEC);
    const int64_t nthreads = n * nseg;
    const unsigned grid_seg = (unsigned)((nthreads + kRmThreads - 1) / kRmThreads);
    TS* A = (TS*)bufA;  // even k (x0 copy, x2, x4, ...)
    TS* B = (TS*)bufB;  // odd k (x1, x3, ...)
    cm2rm_step_kernel<Pol, TY, TS, TC, CB><<<grid_rows, kRmThreads, 0, ctx->stream>>>(
        pol, n, s, (const TY*)V, ldv, B, A, ld, ta, tb);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    for (int64_t k = 2; k < degree; ++k) {
        TS* xk1 = (k - 1) % 2 ? B : A;
        TS* xk2 = (k - 2) % 2 ? B : A;
        rm_step_kernel<Pol, TS, TC><<<grid_seg, kRmThreads, 0, ctx->stream>>>(pol, n, nseg, ld, xk1, xk2, xk2, ta,
                                                                               tb, tm1);
        ctx->launches++;
    }
    RC_CU(ctx, cudaGetLastError());
    {
        const int64_t k = degree;
        TS* xk1 = (k - 1) % 2 ? B : A;
        TS* xk2 = (k - 2) % 2 ? B : A;
        rm2cm_step_kernel<Pol, TS, TY, TC, CB><<<grid_rows, kRmThreads, 0, ctx->stream>>>(
            pol, n, s, ld, xk1, xk2, (TY*)V, ldv, ta, tb, tm1, (R)(1.0 / (double)(degree + 1)));
        ctx->launches++;
        RC_CU(ctx, cudaGetLastError());
    }
    return RC_OK;
}

template <class TS, class TC>
static rc_status rm_filter_dispatch(rc_ctx* ctx, rc_op* op, void* V, int64_t ldv, int64_t s, int64_t degree,
                                    double a, double b, void* bufA, void* bufB, int64_t ld) {
    const int64_t n = op->n;
    if (op->kind == 0) {
        CsrRows<TS, TC> pol{op->rowptr, op->colind, (const TS*)(sizeof(real_t<TS>) == 8 ? op->vals64 : op->vals32)};
        return run_rm_filter<CsrRows<TS, TC>, TS, TC>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB, ld);
    }
    using TD = real_t<TS>;
    const TD* dg = (const TD*)(sizeof(TD) == 8 ? (const void*)op->diag64 : (const void*)op->diag32);
    const double theta = 2.0 * 3.14159265358979323846 * op->flux;
    if (op->skind == 27) {
        StencilRows<TD, TC, 27> pol{op->nx, op->ny, op->nz, dg, op->offdiag, theta};
        return run_rm_filter<StencilRows<TD, TC, 27>, TS, TC>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB, ld);
    }
    if (op->skind == 7) {
        StencilRows<TD, TC, 7> pol{op->nx, op->ny, op->nz, dg, op->offdiag, theta};
        return run_rm_filter<StencilRows<TD, TC, 7>, TS, TC>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB, ld);
    }
    StencilRows<TD, TC, 5> pol{op->nx, op->ny, op->nz, dg, op->offdiag, theta};
    return run_rm_filter<StencilRows<TD, TC, 5>, TS, TC>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB, ld);
}

int64_t rm_leading_dim(int dtype, int prec, int64_t s) {
    const int64_t v = 16 / (int64_t)elem_bytes(dtype, prec);
    return ((s + v - 1) / v) * v;
}

rc_status rm_filter(rc_ctx* ctx, rc_op* op, void* V, int64_t ldv, int64_t s, int64_t degree, double a, double b,
                    int prec, void* bufA, void* bufB) {
    const bool cplx = op->dtype == RC_COMPLEX128;
    const int p = prec == RC_PREC_MIXED ? P32 : P64;
    const int64_t ld = rm_leading_dim(op->dtype, p, s);
    if (cplx && op->kind == 1 && op->skind == 27)
        return rc_fail(ctx, RC_ERR_UNSUPPORTED, "27-point stencil is real only");
    if (p == P32) {
        if (cplx) return rm_filter_dispatch<float2, float2>(ctx, op, V, ldv, s, degree, a, b, bufA, bufB, ld);
        return rm_filter_dispatch<float, float>(ctx, op, V, ldv, s, degree, a, b, bufA, bufB, ld);
    }
    if (cplx) return rm_filter_dispatch<double2, double2>(ctx, op, V, ldv, s, degree, a, b, bufA, bufB, ld);
    return rm_filter_dispatch<double, double>(ctx, op, V, ldv, s, degree, a, b, bufA, bufB, ld);
}

}  // namespace rcb
