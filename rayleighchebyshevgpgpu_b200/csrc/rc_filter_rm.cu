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
//   to_rm:     X column-major (FP64) -> x0 row-major (storage precision), 32x32 smem tiles
//   step k:    x_k over x_{k-2}, row-major (one pass: read x_{k-1}, x_{k-2}, write x_k)
//   to_cm:     x_m/(m+1) row-major -> X column-major (FP64)
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

// Middle step. Persistent grid (one wave): CTA b owns the contiguous rows
// [b*chunk, (b+1)*chunk) and walks them in order, rows_per_iter rows at a time; thread
// (r, seg) of an iteration owns the 16-byte slice seg of row r (V = 16/sizeof(TS) columns).
// Walking rows in order keeps the nearby neighbour rows (+-1, +-nx) in this SM's L1; the far
// ones (+-nx*ny) are fetched at about the same moment by a CTA a few chunks away (L2 hit).
// pf_z > 0: each 128-byte line of row i + pf_z of x_{k-2} and of row i + pf_x of x_{k-1} (the
// rows first touched from DRAM that many rows later) is prefetched into L2.
__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

template <class Pol, class TS, class TC>
__global__ void __launch_bounds__(kRmThreads)
rm_step_kernel(Pol op, int64_t n, int nseg, int64_t ld, int64_t chunk, const TS* __restrict__ x, const TS* z, TS* y,
               TC alpha, TC beta, TC gamma, int64_t pf_z, int64_t pf_x) {
    constexpr int V = Pack16<TS>::V;
    const int rows_per_iter = blockDim.x / nseg;
    const int rloc = threadIdx.x / nseg;
    if (rloc >= rows_per_iter) return;
    const int64_t off = (int64_t)(threadIdx.x - rloc * nseg) * V;
    const bool line_head = ((off * (int64_t)sizeof(TS)) & 127) == 0;
    const int64_t r_begin = (int64_t)blockIdx.x * chunk;
    const int64_t r_end = min(n, r_begin + chunk);
    for (int64_t i = r_begin + rloc; i < r_end; i += rows_per_iter) {
        if (pf_z > 0 && line_head) {
            if (i + pf_z < n) prefetch_l2(z + (i + pf_z) * ld + off);
            if (i + pf_x < n) prefetch_l2(x + (i + pf_x) * ld + off);
        }
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
}

// Middle step with the row's N entries gathered up front (padding (i, 0)); the 16-byte slices
// of up to 9 neighbour rows are then loaded back to back before any arithmetic, so every
// thread keeps several independent loads in flight.
template <class Pol, class TS, class TC, int N>
__global__ void __launch_bounds__(kRmThreads)
rm_step_batched_kernel(Pol op, int64_t n, int nseg, int64_t ld, int64_t chunk, const TS* __restrict__ x,
                       const TS* z, TS* y, TC alpha, TC beta, TC gamma) {
    constexpr int V = Pack16<TS>::V;
    constexpr int G = N <= 9 ? N : 9;
    const int rows_per_iter = blockDim.x / nseg;
    const int rloc = threadIdx.x / nseg;
    if (rloc >= rows_per_iter) return;
    const int64_t off = (int64_t)(threadIdx.x - rloc * nseg) * V;
    const int64_t r_begin = (int64_t)blockIdx.x * chunk;
    const int64_t r_end = min(n, r_begin + chunk);
    for (int64_t i = r_begin + rloc; i < r_end; i += rows_per_iter) {
        int64_t js[N];
        TC as[N];
        op.template gather<N>(i, js, as);
        const Pack16<TS> zi = ld16(z + i * ld + off);
        const Pack16<TS> xi = ld16_ro(x + i * ld + off);
        TC acc[V];
#pragma unroll
        for (int v = 0; v < V; ++v) acc[v] = s_zero(TC());
#pragma unroll
        for (int b0 = 0; b0 < N; b0 += G) {
            Pack16<TS> p[G];
#pragma unroll
            for (int g = 0; g < G; ++g)
                if (b0 + g < N) p[g] = ld16_ro(x + js[b0 + g] * ld + off);
#pragma unroll
            for (int g = 0; g < G; ++g)
                if (b0 + g < N) {
#pragma unroll
                    for (int v = 0; v < V; ++v) acc[v] = s_fma(as[b0 + g], s_cvt<TC>(p[g].v[v]), acc[v]);
                }
        }
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
}

// Layout change between the caller's column-major FP64 block and the row-major scratch, through
// 32x32 shared-memory tiles (coalesced on both sides), converting precision and scaling.
//   to_rm:  R[i*ld + c] = (TS) V[i + c*ldv]
//   to_cm:  V[i + c*ldv] = scale * R[i*ld + c]
template <class TV, class TS>
__global__ void __launch_bounds__(256)
to_rm_kernel(int64_t n, int64_t s, const TV* __restrict__ Vc, int64_t ldv, TS* __restrict__ Rr, int64_t ld) {
    __shared__ TS tile[32][33];
    const int64_t r0 = (int64_t)blockIdx.x * 32, c0 = (int64_t)blockIdx.y * 32;  // rows on x (no 65535 cap)
    const int tx = threadIdx.x, ty = threadIdx.y;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int64_t c = c0 + ty + 8 * j, r = r0 + tx;
        tile[ty + 8 * j][tx] = (r < n && c < s) ? s_cvt<TS>(Vc[r + c * ldv]) : s_zero(TS());
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int64_t r = r0 + ty + 8 * j, c = c0 + tx;
        if (r < n && c < s) Rr[r * ld + c] = tile[tx][ty + 8 * j];
    }
}

template <class TS, class TV>
__global__ void __launch_bounds__(256)
to_cm_kernel(int64_t n, int64_t s, const TS* __restrict__ Rr, int64_t ld, TV* __restrict__ Vc, int64_t ldv,
             double scale) {
    __shared__ TS tile[32][33];
    const int64_t r0 = (int64_t)blockIdx.x * 32, c0 = (int64_t)blockIdx.y * 32;  // rows on x (no 65535 cap)
    const int tx = threadIdx.x, ty = threadIdx.y;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int64_t r = r0 + ty + 8 * j, c = c0 + tx;
        tile[ty + 8 * j][tx] = (r < n && c < s) ? Rr[r * ld + c] : s_zero(TS());
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int64_t c = c0 + ty + 8 * j, r = r0 + tx;
        if (r < n && c < s) Vc[r + c * ldv] = s_rscale((real_t<TV>)scale, s_cvt<TV>(tile[tx][ty + 8 * j]));
    }
}

// ---------------------------------------------------------------------------------------
// Driver
// ---------------------------------------------------------------------------------------
// NB > 0: steps gather the row's NB entries up front (rm_step_batched_kernel);
// NB == 0: steps walk the row entry by entry (rm_step_kernel, with L2 prefetch).
//   A <- X (row-major copy of x0); x_k (k = 1..m) into B, A, B, ... (x_k over x_{k-2});
//   X <- x_m / (m+1) (column-major).
template <class Pol, class TS, class TC, int NB>
static rc_status run_rm_filter(rc_ctx* ctx, const Pol& pol, int64_t n, void* V, int64_t ldv, int64_t s,
                               int64_t degree, double a, double b, void* bufA, void* bufB, int64_t ld, int64_t band) {
    const int64_t pf_z = ctx->pf_rows;
    const int64_t pf_x = pf_z > 0 ? pf_z + band : 0;
    using TY = typename std::conditional<IsComplex<TC>::value, double2, double>::type;
    constexpr int VEC = Pack16<TS>::V;
    const TC ta = s_from<TC>(a, 0.0), tb = s_from<TC>(b, 0.0), tm1 = s_from<TC>(-1.0, 0.0);
    const int nseg = (int)(ld / VEC);
    if (nseg > kRmThreads) return rc_fail(ctx, RC_ERR_UNSUPPORTED, "row-major filter: block too wide");
    const int rows_per_iter = kRmThreads / nseg;
    int64_t chunk;
    if (ctx->rm_map == 1) {
        // one wave of persistent CTAs, each owning a contiguous chunk of rows
        int per_sm = 0;
        RC_CU(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rm_step_kernel<Pol, TS, TC>, kRmThreads, 0));
        if (per_sm < 1) per_sm = 1;
        const int64_t nb0 = (int64_t)per_sm * ctx->sm_count;
        chunk = (n + nb0 - 1) / nb0;
        chunk = ((chunk + rows_per_iter - 1) / rows_per_iter) * rows_per_iter;
    } else {
        // grid order: CTA b owns rows_per_iter consecutive rows, so the rows in flight form one
        // contiguous band and a row's far neighbours were read one band earlier (still in L2)
        chunk = rows_per_iter;
    }
    const unsigned grid_seg = (unsigned)((n + chunk - 1) / chunk);
    if ((s + 31) / 32 > 65535) return rc_fail(ctx, RC_ERR_UNSUPPORTED, "row-major filter: too many columns");
    const dim3 tgrid((unsigned)((n + 31) / 32), (unsigned)((s + 31) / 32)), tblk(32, 8);
    TS* A = (TS*)bufA;
    TS* B = (TS*)bufB;
    to_rm_kernel<TY, TS><<<tgrid, tblk, 0, ctx->stream>>>(n, s, (const TY*)V, ldv, A, ld);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    for (int64_t k = 1; k <= degree; ++k) {
        TS* xk1 = (k - 1) % 2 ? B : A;  // x_{k-1}
        TS* y = k % 2 ? B : A;          // x_k overwrites x_{k-2}
        // k = 1 has no x_{k-2}: z = x0 (finite data) with gamma = 0
        const TS* z = k >= 2 ? y : A;
        const TC g = k >= 2 ? tm1 : s_zero(TC());
        if constexpr (NB > 0)
            rm_step_batched_kernel<Pol, TS, TC, NB><<<grid_seg, kRmThreads, 0, ctx->stream>>>(
                pol, n, nseg, ld, chunk, xk1, z, y, ta, tb, g);
        else
            rm_step_kernel<Pol, TS, TC><<<grid_seg, kRmThreads, 0, ctx->stream>>>(pol, n, nseg, ld, chunk, xk1, z, y,
                                                                                   ta, tb, g, pf_z, pf_x);
        ctx->launches++;
    }
    RC_CU(ctx, cudaGetLastError());
    TS* xm = degree % 2 ? B : A;
    to_cm_kernel<TS, TY><<<tgrid, tblk, 0, ctx->stream>>>(n, s, xm, ld, (TY*)V, ldv, 1.0 / (double)(degree + 1));
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    return RC_OK;
}

template <class TS, class TC>
static rc_status rm_filter_dispatch(rc_ctx* ctx, rc_op* op, void* V, int64_t ldv, int64_t s, int64_t degree,
                                    double a, double b, void* bufA, void* bufB, int64_t ld) {
    const int64_t n = op->n;
    const int64_t band = op->kind == 0 ? op->band : (op->skind == 5 ? op->nx : op->nx * op->ny);
    if (op->kind == 0) {
        CsrRows<TS, TC> pol{op->rowptr, op->colind, (const TS*)(sizeof(real_t<TS>) == 8 ? op->vals64 : op->vals32)};
        using P = CsrRows<TS, TC>;
        if (ctx->csr_variant == 2 && op->max_row_nnz <= 8)
            return run_rm_filter<P, TS, TC, 8>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB, ld, band);
        if (ctx->csr_variant == 2 && op->max_row_nnz <= 32)
            return run_rm_filter<P, TS, TC, 32>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB, ld, band);
        return run_rm_filter<P, TS, TC, 0>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB, ld, band);
    }
    using TD = real_t<TS>;
    const TD* dg = (const TD*)(sizeof(TD) == 8 ? (const void*)op->diag64 : (const void*)op->diag32);
    const double theta = 2.0 * 3.14159265358979323846 * op->flux;
    if (op->skind == 27) {
        StencilRows<TD, TC, 27> pol{op->nx, op->ny, op->nz, dg, op->offdiag, theta};
        return ctx->csr_variant != 2
                   ? run_rm_filter<StencilRows<TD, TC, 27>, TS, TC, 0>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB, ld,
                                                                     band)
                   : run_rm_filter<StencilRows<TD, TC, 27>, TS, TC, 27>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB,
                                                                      ld, band);
    }
    if (op->skind == 7) {
        StencilRows<TD, TC, 7> pol{op->nx, op->ny, op->nz, dg, op->offdiag, theta};
        return ctx->csr_variant != 2
                   ? run_rm_filter<StencilRows<TD, TC, 7>, TS, TC, 0>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB, ld,
                                                                     band)
                   : run_rm_filter<StencilRows<TD, TC, 7>, TS, TC, 7>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB,
                                                                      ld, band);
    }
    StencilRows<TD, TC, 5> pol{op->nx, op->ny, op->nz, dg, op->offdiag, theta};
    return ctx->csr_variant != 2
                   ? run_rm_filter<StencilRows<TD, TC, 5>, TS, TC, 0>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB, ld,
                                                                     band)
                   : run_rm_filter<StencilRows<TD, TC, 5>, TS, TC, 5>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB,
                                                                      ld, band);
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
