// rc_resid.cu -- residual block of the Ritz vectors, R = A Y - Y diag(lam), in one pass over Y.
//
// The reference forms tmp = A*V with a second SpMM and then runs its residuals kernel
// (RayleighChebyshevLMCuda.h:2235, :2274-2280; cuda_kernels.cu:307-382). Here the sparse product,
// the subtraction, the column norms ||R_c|| (c < res_count) and, for the correction filter, the
// row-major bfloat16 (rc_corr_t) copy of R are one kernel over the row-major FP64 copy of Y that the Ritz GEMM
// writes beside the column-major one (xt2): the filter's degree-step arithmetic (rc_rmstep.cuh
// layout: 16-byte slices, consecutive row groups per CTA), so a neighbour row is one contiguous
// run and the far neighbours (i +- band) are L2 hits. Nothing n x s is written in FP64.
// Column norms: each thread sums the squares of its own columns over its rows, the threads of a
// CTA are combined in shared memory in a fixed order, and the per-CTA partials are summed in a
// fixed order by resid_norm_reduce_kernel (deterministic).
#include <algorithm>
#include "rc_common.cuh"
#include "rc_internal.h"
#include "rc_rmstep.cuh"

namespace rcb {

// 4 resident CTAs per SM (64 registers): the residual epilogue keeps per-column sums and Ritz
// values in registers, which spill at the filter steps' 40.
template <class Pol, int W, class IX>
__global__ void __launch_bounds__(kRmThreads, 4)
resid_rm_kernel(Pol op, int64_t n, int64_t s, int nseg, int64_t ld, int groups, const double* __restrict__ Y,
                const double* __restrict__ lam, int res_count, double* __restrict__ part, rc_corr_t* __restrict__ R32,
                int64_t ldr) {
    constexpr int V = Pack16<double>::V;  // 2 columns per 16-byte slice
    extern __shared__ double red[];        // [rows_per_iter][ld]
    const int rows_per_iter = blockDim.x / nseg;
    const int rloc = threadIdx.x / nseg;
    const bool active = rloc < rows_per_iter;
    const IX off = (IX)(threadIdx.x - rloc * nseg) * (IX)V;
    const IX wstride = (IX)nseg * (IX)V;
    const IX ldy = (IX)ld;
    double sq[W * V];
    double lm[W * V];
#pragma unroll
    for (int w = 0; w < W; ++w)
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int64_t c = (int64_t)(off + w * wstride + v);
            sq[w * V + v] = 0.0;
            lm[w * V + v] = (active && c < s) ? lam[c] : 0.0;
        }
    if (active) {
        const int64_t stride = rows_per_iter;
        int64_t i = (int64_t)blockIdx.x * groups * rows_per_iter + rloc;
        const int64_t i_end = min(n, ((int64_t)blockIdx.x + 1) * groups * rows_per_iter);
        typename Pol::Pre p0, p1;
        if (i < i_end) {
            op.fetch1(i, p0);
            op.fetch2(i, p0);
        }
        if (i + stride < i_end) op.fetch1(i + stride, p1);
        for (; i < i_end; i += stride) {
            typename Pol::Pre p2;
            if (i + stride < i_end) op.fetch2(i + stride, p1);
            if (i + 2 * stride < i_end) op.fetch1(i + 2 * stride, p2);
            double acc[W * V];
#pragma unroll
            for (int v = 0; v < W * V; ++v) acc[v] = 0.0;
            op.row(i, p0, [&](int64_t j, double a) {
                const double* yj = Y + ((IX)j * ldy + off);
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    const Pack16<double> q = ld16_ro(yj + w * wstride);
#pragma unroll
                    for (int v = 0; v < V; ++v) acc[w * V + v] = fma(a, q.v[v], acc[w * V + v]);
                }
            });
#pragma unroll
            for (int w = 0; w < W; ++w) {
                const IX o = (IX)i * ldy + off + w * wstride;
                const Pack16<double> yi = ld16_ro(Y + o);
                float rv[V];
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const int64_t c = (int64_t)(off + w * wstride + v);
                    const double d = c < s ? fma(-lm[w * V + v], yi.v[v], acc[w * V + v]) : 0.0;
                    sq[w * V + v] = fma(d, d, sq[w * V + v]);
                    rv[v] = (float)d;
                }
                if (R32) {
                    const int64_t c0 = (int64_t)(off + w * wstride);
#if RC_CORR_BF16
                    *reinterpret_cast<__nv_bfloat162*>(R32 + i * ldr + c0) = __floats2bfloat162_rn(rv[0], rv[1]);
#else
                    *reinterpret_cast<float2*>(R32 + i * ldr + c0) = make_float2(rv[0], rv[1]);
#endif
                }
            }
            p0 = p1;
            p1 = p2;
        }
    }
    if (res_count <= 0) return;
    // column sums over the CTA's rows: row slot rloc of the shared table, then slots in order
    if (active) {
#pragma unroll
        for (int w = 0; w < W; ++w)
#pragma unroll
            for (int v = 0; v < V; ++v) red[rloc * ld + off + w * wstride + v] = sq[w * V + v];
    }
    __syncthreads();
    for (int c = threadIdx.x; c < res_count; c += blockDim.x) {
        double t = 0.0;
        for (int r = 0; r < rows_per_iter; ++r) t += red[r * ld + c];
        part[(int64_t)blockIdx.x * res_count + c] = t;
    }
}

__global__ void resid_norm_reduce_kernel(int64_t nparts, int res_count, const double* __restrict__ part,
                                         double* __restrict__ res) {
    const int c = blockIdx.x;
    __shared__ double sc[32];
    double v = 0.0;
    for (int64_t b = threadIdx.x; b < nparts; b += blockDim.x) v += part[b * res_count + c];
    v = block_sum(v, sc);
    if (threadIdx.x == 0) res[c] = sqrt(v);
}

bool resid_supported(const rc_op* op, int64_t s) {
    return op->dtype == RC_REAL64 && s >= 1 && s <= 96 &&
           (op->kind == 0 || (op->kind == 1 && (op->skind == 5 || op->skind == 7 || op->skind == 27)));
}

template <class Pol, int W, class IX>
static rc_status resid_launch(rc_ctx* ctx, const Pol& pol, int64_t n, int64_t s, const double* Y, int64_t ld,
                              const double* lam, int64_t res_count, double* res, rc_corr_t* R32, int64_t ldr) {
    constexpr int V = Pack16<double>::V;
    if (ld % (V * W) != 0) return rc_fail(ctx, RC_ERR_INVALID, "residual block: leading dimension not padded");
    const int nseg = (int)(ld / (V * W));
    if (nseg > kRmThreads) return rc_fail(ctx, RC_ERR_UNSUPPORTED, "residual block: block too wide");
    const int rows_per_iter = kRmThreads / nseg;
    const int groups = 8;  // 80+ rows per CTA: fewer per-CTA column-sum epilogues and partials
    const int64_t rows_per_cta = (int64_t)groups * rows_per_iter;
    const int64_t grid = (n + rows_per_cta - 1) / rows_per_cta;
    double* part = nullptr;
    if (res_count > 0) {
        void* pp = nullptr;
        RC_TRY(rc_slot(ctx, S_RPART, (size_t)grid * res_count * sizeof(double), &pp));
        part = (double*)pp;
    }
    const size_t smem = res_count > 0 ? (size_t)rows_per_iter * ld * sizeof(double) : 0;
    resid_rm_kernel<Pol, W, IX><<<(unsigned)grid, kRmThreads, smem, ctx->stream>>>(
        pol, n, s, nseg, ld, groups, Y, lam, (int)res_count, part, R32, ldr);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    if (res_count > 0) {
        resid_norm_reduce_kernel<<<(unsigned)res_count, 256, 0, ctx->stream>>>(grid, (int)res_count, part, res);
        ctx->launches++;
        RC_CU(ctx, cudaGetLastError());
    }
    return RC_OK;
}

template <class Pol, int W>
static rc_status resid_ix(rc_ctx* ctx, const Pol& pol, int64_t n, int64_t s, const double* Y, int64_t ld,
                          const double* lam, int64_t res_count, double* res, rc_corr_t* R32, int64_t ldr) {
    if ((n + 1) * std::max(ld, ldr) < ((int64_t)1 << 32))
        return resid_launch<Pol, W, uint32_t>(ctx, pol, n, s, Y, ld, lam, res_count, res, R32, ldr);
    return resid_launch<Pol, W, int64_t>(ctx, pol, n, s, Y, ld, lam, res_count, res, R32, ldr);
}

rc_status resid_block(rc_ctx* ctx, const rc_op* op, const double* Yrm, int64_t ld, int64_t s, const double* lam,
                      int64_t res_count, double* res, rc_corr_t* R32, int64_t ldr) {
    if (!resid_supported(op, s)) return rc_fail(ctx, RC_ERR_UNSUPPORTED, "residual block: unsupported operator");
    if (res_count < 0 || res_count > s || ld != rm_leading_dim(RC_REAL64, P64, s) ||
        (R32 && ldr != rm_leading_dim(RC_REAL64, P32, s)))
        return rc_fail(ctx, RC_ERR_INVALID, "residual block: bad sizes");
    const int64_t n = op->n;
    if (op->kind == 0) {
        CsrRows<double, double> pol{op->rowptr, op->colind, (const double*)op->vals64};
        return resid_ix<CsrRows<double, double>, 2>(ctx, pol, n, s, Yrm, ld, lam, res_count, res, R32, ldr);
    }
    if (op->skind == 27) {
        StencilRows<double, double, 27> pol{op->nx, op->ny, op->nz, op->diag64, op->offdiag, 0.0};
        return resid_ix<StencilRows<double, double, 27>, 1>(ctx, pol, n, s, Yrm, ld, lam, res_count, res, R32, ldr);
    }
    if (op->skind == 7) {
        StencilRows<double, double, 7> pol{op->nx, op->ny, op->nz, op->diag64, op->offdiag, 0.0};
        return resid_ix<StencilRows<double, double, 7>, 1>(ctx, pol, n, s, Yrm, ld, lam, res_count, res, R32, ldr);
    }
    StencilRows<double, double, 5> pol{op->nx, op->ny, op->nz, op->diag64, op->offdiag, 0.0};
    return resid_ix<StencilRows<double, double, 5>, 1>(ctx, pol, n, s, Yrm, ld, lam, res_count, res, R32, ldr);
}

}  // namespace rcb
