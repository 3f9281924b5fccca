// rc_resid.cu -- residual block of the Ritz vectors, R = A Y - Y diag(lam), in one pass over Y.
//
// The reference forms tmp = A*V with a second SpMM and then runs its residuals kernel
// (RayleighChebyshevLMCuda.h:2235, :2274-2280; cuda_kernels.cu:307-382). Here the sparse product,
// the subtraction, the column norms ||R_c|| (c < res_count) and, for the correction filter, the
// row-major bfloat16 copy of R (rc_corr_t, or rc_corr2_t for complex operators) are one kernel over
// a row-major FP64 (c128) copy of Y: the filter's degree-step arithmetic (rc_rmstep.cuh layout:
// 16-byte slices, consecutive row groups per CTA), so a neighbour row is one contiguous run and the
// far neighbours (i +- band) are L2 hits. Nothing n x s is written in FP64.
// Column norms: each thread sums the squares of its own columns over its rows, the threads of a
// CTA are combined in shared memory in a fixed order, and the per-CTA partials are summed in a
// fixed order by resid_norm_reduce_kernel (deterministic).
#include <algorithm>
#include <type_traits>
#include "rc_common.cuh"
#include "rc_internal.h"
#include "rc_rmstep.cuh"

namespace rcb {

// Two FP32 values of the residual block at p: two real columns, or the real and imaginary part of
// one complex column. Written once: evict-first when RC_STREAM_HINTS is 1 (by default these
// bfloat16 or FP32 stores take no hint, as the correction filter's blocks).
__device__ __forceinline__ void corr_store2(void* p, float a, float b) {
#if RC_CORR_BF16
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
#if RC_STREAM_HINTS == 1
    unsigned u;
    memcpy(&u, &h, 4);
    __stcs(reinterpret_cast<unsigned*>(p), u);
#else
    *reinterpret_cast<__nv_bfloat162*>(p) = h;
#endif
#else
#if RC_STREAM_HINTS == 1
    __stcs(reinterpret_cast<float2*>(p), make_float2(a, b));
#else
    *reinterpret_cast<float2*>(p) = make_float2(a, b);
#endif
#endif
}
__device__ __forceinline__ double resid_sub(double lm, double y, double acc) { return fma(-lm, y, acc); }
__device__ __forceinline__ double2 resid_sub(double lm, double2 y, double2 acc) {
    return make_double2(fma(-lm, y.x, acc.x), fma(-lm, y.y, acc.y));
}

// The 27-point form (real): each thread walks kRun27 consecutive rows and keeps the 3x3
// cross-section sums of rows i-1, i and i+1 (rm_step_rows27's scheme), so a row gathers 9
// neighbours instead of 27: (A y)_i = (diag_i - offd) y_i + offd (Q(i-1) + Q(i) + Q(i+1)).
// Thread (r, seg) of CTA b takes rows (b*rows_per_iter + r)*kRun27 .. + kRun27.
template <int W, class IX>
__device__ __forceinline__ void resid_rows27(const StencilRows<double, double, 27>& op, int64_t n, int64_t s,
                                             int64_t ld, int rows_per_iter, int rloc, IX off, IX wstride,
                                             const double* __restrict__ Y, const double* __restrict__ lam,
                                             double (&sq)[W * 2], rc_corr_t* R, int64_t ldr) {
    constexpr int V = 2;
    const IX ldy = (IX)ld;
    const int64_t nx = op.nx, ny = op.ny, nz = op.nz, sy = nx, sz = nx * ny;
    const double woff = op.offd;
    const int64_t i0 = ((int64_t)blockIdx.x * rows_per_iter + rloc) * (int64_t)kRun27;
    const int64_t i1 = min(n, i0 + kRun27);
    auto cross = [&](int64_t j, bool vym, bool vyp, bool vzm, bool vzp, double (&q)[W * V]) {
#pragma unroll
        for (int v = 0; v < W * V; ++v) q[v] = 0.0;
#pragma unroll
        for (int dz = -1; dz <= 1; ++dz) {
            const bool vz = dz < 0 ? vzm : (dz > 0 ? vzp : true);
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy) {
                const bool vy = dy < 0 ? vym : (dy > 0 ? vyp : true);
                if (vz && vy) {
                    const double* yj = Y + ((IX)(j + dy * sy + dz * sz) * ldy + off);
#pragma unroll
                    for (int w = 0; w < W; ++w) {
                        const Pack16<double> pk = ld16_ro(yj + w * wstride);
#pragma unroll
                        for (int v = 0; v < V; ++v) q[w * V + v] += pk.v[v];
                    }
                }
            }
        }
    };
    double qm[W * V], q0[W * V], qp[W * V];
    for (int64_t i = i0; i < i1; ++i) {
        int64_t ix, iy, iz;
        op.coords(i, ix, iy, iz);
        const bool vym = iy > 0, vyp = iy + 1 < ny, vzm = iz > 0, vzp = iz + 1 < nz;
        if (i == i0 || ix == 0) {  // (re)start the window at the run's first row or a new x-line
            if (ix > 0) cross(i - 1, vym, vyp, vzm, vzp, qm);
            else
#pragma unroll
                for (int v = 0; v < W * V; ++v) qm[v] = 0.0;
            cross(i, vym, vyp, vzm, vzp, q0);
        }
        if (ix + 1 < nx) cross(i + 1, vym, vyp, vzm, vzp, qp);
        else
#pragma unroll
            for (int v = 0; v < W * V; ++v) qp[v] = 0.0;
        const double dmw = op.diag[i] - woff;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            const IX o = (IX)i * ldy + off + w * wstride;
            const Pack16<double> yi = ld16_ro(Y + o);
            float rv[V];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int e = w * V + v;
                const int64_t c = (int64_t)(off + w * wstride + v);
                const double ay = fma(woff, (qm[e] + q0[e]) + qp[e], dmw * yi.v[v]);
                const double d = c < s ? fma(-__ldg(lam + c), yi.v[v], ay) : 0.0;
                sq[e] = fma(d, d, sq[e]);
                rv[v] = (float)d;
            }
            if (R) corr_store2(R + i * ldr + (int64_t)(off + w * wstride), rv[0], rv[1]);
        }
#pragma unroll
        for (int v = 0; v < W * V; ++v) {
            qm[v] = q0[v];
            q0[v] = qp[v];
        }
    }
}

// RC_RESID_MIN_BLOCKS resident CTAs per SM (default 4, 64 registers): the residual epilogue keeps
// per-column sums in registers, which spill at the filter steps' 40 (the Ritz values are re-read from
// L1 per row). T = double (real) or double2 (complex).
#ifndef RC_RESID_MIN_BLOCKS
#define RC_RESID_MIN_BLOCKS 4
#endif
template <class Pol, class T, int W, class IX>
__global__ void __launch_bounds__(kRmThreads, RC_RESID_MIN_BLOCKS)
resid_rm_kernel(Pol op, int64_t n, int64_t s, int nseg, int64_t ld, int groups, const T* __restrict__ Y,
                const double* __restrict__ lam, int res_count, double* __restrict__ part, void* __restrict__ Rout,
                int64_t ldr) {
    constexpr int V = Pack16<T>::V;  // 2 real or 1 complex column per 16-byte slice
    using TR = typename std::conditional<IsComplex<T>::value, rc_corr2_t, rc_corr_t>::type;
    TR* R = reinterpret_cast<TR*>(Rout);
    extern __shared__ double red[];  // [rows_per_iter][ld]
    const int rows_per_iter = blockDim.x / nseg;
    const int rloc = threadIdx.x / nseg;
    const bool active = rloc < rows_per_iter;
    const IX off = (IX)(threadIdx.x - rloc * nseg) * (IX)V;
    const IX wstride = (IX)nseg * (IX)V;
    const IX ldy = (IX)ld;
    double sq[W * V];
#pragma unroll
    for (int v = 0; v < W * V; ++v) sq[v] = 0.0;
    if constexpr (IsStencil27<Pol>::value) {
        if (active)
            resid_rows27<W, IX>(op, n, s, ld, rows_per_iter, rloc, off, wstride, Y, lam, sq,
                                reinterpret_cast<rc_corr_t*>(Rout), ldr);
    } else if (active) {
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
            T acc[W * V];
#pragma unroll
            for (int v = 0; v < W * V; ++v) acc[v] = s_zero(T());
            op.row(i, p0, [&](int64_t j, T a) {
                const T* yj = Y + ((IX)j * ldy + off);
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    const Pack16<T> q = ld16_ro(yj + w * wstride);
#pragma unroll
                    for (int v = 0; v < V; ++v) acc[w * V + v] = s_fma(a, q.v[v], acc[w * V + v]);
                }
            });
#pragma unroll
            for (int w = 0; w < W; ++w) {
                const IX o = (IX)i * ldy + off + w * wstride;
                const Pack16<T> yi = ld16_ro(Y + o);
                float rv[2];
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const int64_t c = (int64_t)(off + w * wstride + v);
                    const T d = c < s ? resid_sub(__ldg(lam + c), yi.v[v], acc[w * V + v]) : s_zero(T());
                    if constexpr (IsComplex<T>::value) {
                        sq[w * V + v] = fma(d.y, d.y, fma(d.x, d.x, sq[w * V + v]));
                        rv[0] = (float)d.x;
                        rv[1] = (float)d.y;
                    } else {
                        sq[w * V + v] = fma(d, d, sq[w * V + v]);
                        rv[v] = (float)d;
                    }
                }
                if (R) corr_store2(R + i * ldr + (int64_t)(off + w * wstride), rv[0], rv[1]);
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
    if (s < 1 || s > kCorrMaxCols || op->kind == 2) return false;
    if (op->dtype == RC_REAL64) return op->kind == 0 || op->skind == 5 || op->skind == 7 || op->skind == 27;
    return op->dtype == RC_COMPLEX128 && (op->kind == 0 || op->skind == 5 || op->skind == 7);
}

template <class Pol, class T, int W, class IX>
static rc_status resid_launch(rc_ctx* ctx, const Pol& pol, int64_t n, int64_t s, const T* Y, int64_t ld,
                              const double* lam, int64_t res_count, double* res, void* R, int64_t ldr) {
    constexpr int V = Pack16<T>::V;
    if (ld % (V * W) != 0) return rc_fail(ctx, RC_ERR_INVALID, "residual block: leading dimension not padded");
    const int nseg = (int)(ld / (V * W));
    if (nseg > kRmThreads) return rc_fail(ctx, RC_ERR_UNSUPPORTED, "residual block: block too wide");
    const int rows_per_iter = kRmThreads / nseg;
    // 80+ rows per CTA: fewer per-CTA column-sum epilogues and partials (27-point: kRun27 rows a thread)
    const int groups = IsStencil27<Pol>::value ? kRun27 : 8;
    const int64_t rows_per_cta = (int64_t)groups * rows_per_iter;
    const int64_t grid = (n + rows_per_cta - 1) / rows_per_cta;
    double* part = nullptr;
    if (res_count > 0) {
        void* pp = nullptr;
        RC_TRY(rc_slot(ctx, S_RPART, (size_t)grid * res_count * sizeof(double), &pp));
        part = (double*)pp;
    }
    const size_t smem = res_count > 0 ? (size_t)rows_per_iter * ld * sizeof(double) : 0;
    resid_rm_kernel<Pol, T, W, IX><<<(unsigned)grid, kRmThreads, smem, ctx->stream>>>(
        pol, n, s, nseg, ld, groups, Y, lam, (int)res_count, part, R, ldr);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    if (res_count > 0) {
        resid_norm_reduce_kernel<<<(unsigned)res_count, 256, 0, ctx->stream>>>(grid, (int)res_count, part, res);
        ctx->launches++;
        RC_CU(ctx, cudaGetLastError());
    }
    return RC_OK;
}

// Slices per thread: the measured choices for real blocks of up to 96 columns (two for CSR, one for
// stencils); otherwise the count (1 or 2 real, up to 4 complex: more spill) that leaves the fewest
// of a CTA's threads idle.
template <class T>
static int resid_slices(int64_t ld, int64_t s, bool csr) {
    constexpr int V = Pack16<T>::V;
    if (!IsComplex<T>::value && s <= 96) return csr ? 2 : 1;
    int best = 0, best_idle = kRmThreads + 1;
    for (int w = 1; w <= (IsComplex<T>::value ? 4 : 2); ++w) {
        if (ld % (V * w) != 0 || ld / (V * w) > kRmThreads) continue;
        const int idle = kRmThreads % (int)(ld / (V * w));
        if (idle < best_idle) {
            best = w;
            best_idle = idle;
        }
    }
    return best;
}

template <class Pol, class T>
static rc_status resid_ix(rc_ctx* ctx, const Pol& pol, int64_t n, int64_t s, const T* Y, int64_t ld,
                          const double* lam, int64_t res_count, double* res, void* R, int64_t ldr) {
    const int w = resid_slices<T>(ld, s, Pol::kIsCsr);
    const bool small = (n + 1) * std::max(ld, ldr) < ((int64_t)1 << 32);
    switch (w) {
        case 1:
            return small ? resid_launch<Pol, T, 1, uint32_t>(ctx, pol, n, s, Y, ld, lam, res_count, res, R, ldr)
                         : resid_launch<Pol, T, 1, int64_t>(ctx, pol, n, s, Y, ld, lam, res_count, res, R, ldr);
        case 2:
            return small ? resid_launch<Pol, T, 2, uint32_t>(ctx, pol, n, s, Y, ld, lam, res_count, res, R, ldr)
                         : resid_launch<Pol, T, 2, int64_t>(ctx, pol, n, s, Y, ld, lam, res_count, res, R, ldr);
        default:
            break;
    }
    if constexpr (IsComplex<T>::value) {
        switch (w) {
            case 3:
                return small ? resid_launch<Pol, T, 3, uint32_t>(ctx, pol, n, s, Y, ld, lam, res_count, res, R, ldr)
                             : resid_launch<Pol, T, 3, int64_t>(ctx, pol, n, s, Y, ld, lam, res_count, res, R, ldr);
            case 4:
                return small ? resid_launch<Pol, T, 4, uint32_t>(ctx, pol, n, s, Y, ld, lam, res_count, res, R, ldr)
                             : resid_launch<Pol, T, 4, int64_t>(ctx, pol, n, s, Y, ld, lam, res_count, res, R, ldr);
            default:
                break;
        }
    }
    return rc_fail(ctx, RC_ERR_UNSUPPORTED, "residual block: block too wide");
}

template <class T>
static rc_status resid_dispatch(rc_ctx* ctx, const rc_op* op, const T* Y, int64_t ld, int64_t s, const double* lam,
                                int64_t res_count, double* res, void* R, int64_t ldr) {
    const int64_t n = op->n;
    if (op->kind == 0) {
        CsrRows<T, T> pol{op->rowptr, op->colind, (const T*)op->vals64};
        return resid_ix<CsrRows<T, T>, T>(ctx, pol, n, s, Y, ld, lam, res_count, res, R, ldr);
    }
    const double theta = 2.0 * 3.14159265358979323846 * op->flux;
    if constexpr (!IsComplex<T>::value) {
        if (op->skind == 27) {
            StencilRows<double, T, 27> pol{op->nx, op->ny, op->nz, op->diag64, op->offdiag, theta};
            return resid_ix<StencilRows<double, T, 27>, T>(ctx, pol, n, s, Y, ld, lam, res_count, res, R, ldr);
        }
    }
    if (op->skind == 7) {
        StencilRows<double, T, 7> pol{op->nx, op->ny, op->nz, op->diag64, op->offdiag, theta};
        pol.ph = (const T*)op->phase64;
        return resid_ix<StencilRows<double, T, 7>, T>(ctx, pol, n, s, Y, ld, lam, res_count, res, R, ldr);
    }
    StencilRows<double, T, 5> pol{op->nx, op->ny, op->nz, op->diag64, op->offdiag, theta};
    pol.ph = (const T*)op->phase64;
    return resid_ix<StencilRows<double, T, 5>, T>(ctx, pol, n, s, Y, ld, lam, res_count, res, R, ldr);
}

rc_status resid_block(rc_ctx* ctx, const rc_op* op, const void* Yrm, int64_t ld, int64_t s, const double* lam,
                      int64_t res_count, double* res, void* R, int64_t ldr) {
    if (!resid_supported(op, s)) return rc_fail(ctx, RC_ERR_UNSUPPORTED, "residual block: unsupported operator");
    if (res_count < 0 || res_count > s || ld != rm_leading_dim(op->dtype, P64, s) ||
        (R && ldr != corr_leading_dim(op->dtype, s)))
        return rc_fail(ctx, RC_ERR_INVALID, "residual block: bad sizes");
    if (op->dtype == RC_COMPLEX128)
        return resid_dispatch<double2>(ctx, op, (const double2*)Yrm, ld, s, lam, res_count, res, R, ldr);
    return resid_dispatch<double>(ctx, op, (const double*)Yrm, ld, s, lam, res_count, res, R, ldr);
}

}  // namespace rcb
