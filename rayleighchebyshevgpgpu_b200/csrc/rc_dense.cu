// rc_dense.cu -- FP64 (c128) dense kernels of the orthonormalisation and Rayleigh-Ritz steps.
//
//  gram      C = X^H Y for tall-skinny n x m and n x nc blocks: split over row chunks, each
//            CTA accumulates a 64x64 output tile in registers from shared-memory K-tiles,
//            partial tiles are summed by a second kernel in a fixed order (deterministic).
//            Replaces cublas{D,Z}gemm(OP_T/OP_C, OP_N) (RayleighChebyshevLMCuda.h:2139-2161).
//  xt        Y = beta*Y + X*T for tall-skinny X and a small T, optionally a second pair
//            (W*Q next to V*Q) with the residual ||W_c - lam_c V_c||^2 reduced in the epilogue.
//            Replaces cublas{D,Z}gemm(OP_N,OP_N) + normalize + memcpy + the second SpMM +
//            the residuals kernel (RayleighChebyshevLMCuda.h:2178-2285, cuda_kernels.cu:307-382).
//  chol      Cholesky of a column-scaled Gram matrix and the inverse of its factor (one CTA);
//            with xt it forms CholeskyQR, replacing cusolverDn geqrf+orgqr (:1979-2107).
//  eigh      one-CTA parallel cyclic Jacobi for a small Hermitian matrix, replacing host
//            DSYEV/ZHPEVX (:570-642) and JacobiDiagonalizer.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include "rc_common.cuh"
#include "rc_internal.h"

namespace rcb {

constexpr int TB = 64;   // output tile edge
constexpr int KT = 16;   // K-tile depth
constexpr int TPB = 256; // 16 x 16 threads, 4 x 4 outputs each

template <class T> struct Sel;
template <> struct Sel<double> { static constexpr int dt = RC_REAL64; };
template <> struct Sel<double2> { static constexpr int dt = RC_COMPLEX128; };

// ---------------------------------------------------------------------------------------
// Gram: partial[chunk] (m x nc, ld m) = X[rows of chunk]^H * Y[rows of chunk]
// grid: (nchunks, tiles_m, tiles_n); block 256.
// thread (tx,ty): output rows mi = m0 + tx + 16*i, cols nj = n0 + ty + 16*j.
// ---------------------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(TPB)
gram_partial_kernel(int64_t n, int64_t m, int64_t nc, const T* __restrict__ X, int64_t ldx, const T* __restrict__ Y,
                    int64_t ldy, T* __restrict__ part, int64_t rows_per_chunk, int upper) {
    const int tm = blockIdx.y, tn = blockIdx.z;
    if (upper && tm > tn) return;
    const int64_t m0 = (int64_t)tm * TB, n0 = (int64_t)tn * TB;
    const int64_t r_begin = (int64_t)blockIdx.x * rows_per_chunk;
    const int64_t r_end = min(n, r_begin + rows_per_chunk);
    __shared__ T Xs[KT][TB + 1];
    __shared__ T Ys[KT][TB + 1];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    T acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = s_zero(T());
    for (int64_t r0 = r_begin; r0 < r_end; r0 += KT) {
        // load KT x 64 of X and Y; element e: kk = e % KT (row), cc = e / KT (column)
#pragma unroll
        for (int it = 0; it < (KT * TB) / TPB; ++it) {
            const int e = tid + it * TPB;
            const int kk = e % KT, cc = e / KT;
            const int64_t r = r0 + kk;
            const int64_t cx = m0 + cc, cy = n0 + cc;
            Xs[kk][cc] = (r < r_end && cx < m) ? X[r + cx * ldx] : s_zero(T());
            Ys[kk][cc] = (r < r_end && cy < nc) ? Y[r + cy * ldy] : s_zero(T());
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < KT; ++kk) {
            T a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = Xs[kk][tx + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Ys[kk][ty + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = s_cfma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
    T* P = part + (size_t)blockIdx.x * m * nc;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int64_t mi = m0 + tx + 16 * i, nj = n0 + ty + 16 * j;
            if (mi < m && nj < nc) P[mi + nj * m] = acc[i][j];
        }
}

// C[i,j] = sum over chunks; upper: use i<=j and mirror (Hermitian, real diagonal).
template <class T>
__global__ void gram_reduce_kernel(int64_t m, int64_t nc, int64_t nchunks, const T* __restrict__ part, T* __restrict__ C,
                                   int upper) {
    const int64_t total = m * nc;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e % m, j = e / m;
        if (upper && i > j) continue;
        T sum = s_zero(T());
        for (int64_t c = 0; c < nchunks; ++c) sum = s_add(sum, part[(size_t)c * total + e]);
        if (upper) {
            if (i == j) {
                sum = s_from<T>(s_real(sum), 0.0);
                C[e] = sum;
            } else {
                C[e] = sum;
                C[j + i * m] = s_conj(sum);
            }
        } else {
            C[e] = sum;
        }
    }
}

template <class T>
static rc_status gram_t(rc_ctx* ctx, int64_t n, int64_t m, int64_t nc, const T* X, int64_t ldx, const T* Y,
                        int64_t ldy, T* C, bool upper) {
    const int tiles_m = (int)((m + TB - 1) / TB), tiles_n = (int)((nc + TB - 1) / TB);
    const int tiles = upper ? tiles_m * (tiles_m + 1) / 2 : tiles_m * tiles_n;
    // about 4 CTAs per SM in total, each chunk a multiple of KT rows
    int64_t nchunks = (4 * ctx->sm_count + tiles - 1) / tiles;
    int64_t rows = (n + nchunks - 1) / nchunks;
    rows = ((rows + KT - 1) / KT) * KT;
    if (rows < KT) rows = KT;
    nchunks = (n + rows - 1) / rows;
    if (nchunks < 1) nchunks = 1;
    void* part = nullptr;
    RC_TRY(rc_slot(ctx, S_PART, (size_t)nchunks * m * nc * sizeof(T), &part));
    dim3 grid((unsigned)nchunks, tiles_m, tiles_n);
    gram_partial_kernel<T><<<grid, TPB, 0, ctx->stream>>>(n, m, nc, X, ldx, Y, ldy, (T*)part, rows, upper ? 1 : 0);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    const int64_t total = m * nc;
    const unsigned g2 = (unsigned)std::min<int64_t>((total + 255) / 256, 4 * 148);
    gram_reduce_kernel<T><<<g2, 256, 0, ctx->stream>>>(m, nc, nchunks, (const T*)part, C, upper ? 1 : 0);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    return RC_OK;
}

rc_status gram(rc_ctx* ctx, int dtype, int64_t n, int64_t m, int64_t nc, const void* X, int64_t ldx, const void* Y,
               int64_t ldy, void* C, bool upper) {
    if (m <= 0 || nc <= 0) return RC_OK;
    if (upper && m != nc) return rc_fail(ctx, RC_ERR_INVALID, "gram: upper requires a square result");
    if (upper && gram2_supported(dtype, m))
        return gram2(ctx, n, m, (const double*)X, ldx, (const double*)Y, ldy, (double*)C, nullptr, 0, nullptr);
    if (upper && ctx->gram_c && gram_c_supported(dtype, m) && (uintptr_t)X % 16 == 0 && (uintptr_t)Y % 16 == 0)
        return gram_c(ctx, n, m, (const double2*)X, ldx, (const double2*)Y, ldy, (double2*)C);
    if (dtype == RC_COMPLEX128)
        return gram_t<double2>(ctx, n, m, nc, (const double2*)X, ldx, (const double2*)Y, ldy, (double2*)C, upper);
    return gram_t<double>(ctx, n, m, nc, (const double*)X, ldx, (const double*)Y, ldy, (double*)C, upper);
}

// ---------------------------------------------------------------------------------------
// XT: Y = beta*Y + X*T  (X: n x k, T: k x nc, Y: n x nc), optional dual + residuals.
// grid: (ceil(n/64), ceil(nc/64)); thread (tx,ty): rows r0 + tx + 16 i, cols c0 + ty + 16 j.
// ---------------------------------------------------------------------------------------
template <class T, bool DUAL>
__global__ void __launch_bounds__(TPB)
xt_kernel(int64_t n, int64_t k, int64_t nc, const T* __restrict__ X, int64_t ldx, const T* __restrict__ Tm,
          int64_t ldt, T* __restrict__ Y, int64_t ldy, double alpha, double beta, const T* __restrict__ X2, int64_t ldx2,
          T* __restrict__ Y2, int64_t ldy2, const double* __restrict__ lam, int64_t res_count,
          double* __restrict__ rpart) {
    constexpr int KX = IsComplex<T>::value ? 8 : 16;  // K-tile depth (complex: 48 KB static smem limit)
    const int64_t r0 = (int64_t)blockIdx.x * TB, c0 = (int64_t)blockIdx.y * TB;
    __shared__ T Xs[KX][TB + 1];
    __shared__ T X2s[DUAL ? KX : 1][TB + 1];
    __shared__ T Ts[KX][TB + 1];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    T acc[4][4], acc2[DUAL ? 4 : 1][DUAL ? 4 : 1];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = s_zero(T());
    if (DUAL) {
#pragma unroll
        for (int i = 0; i < (DUAL ? 4 : 1); ++i)
#pragma unroll
            for (int j = 0; j < (DUAL ? 4 : 1); ++j) acc2[i][j] = s_zero(T());
    }
    for (int64_t k0 = 0; k0 < k; k0 += KX) {
        // X tile: 64 rows x KX cols; element e: rr = e % 64 (row), kk = e / 64
#pragma unroll
        for (int it = 0; it < (KX * TB) / TPB; ++it) {
            const int e = tid + it * TPB;
            const int rr = e % TB, kk = e / TB;
            const int64_t r = r0 + rr, kc = k0 + kk;
            const bool ok = r < n && kc < k;
            Xs[kk][rr] = ok ? X[r + kc * ldx] : s_zero(T());
            if (DUAL) X2s[kk][rr] = ok ? X2[r + kc * ldx2] : s_zero(T());
        }
        // T tile: KX rows x 64 cols; element e: kk = e % KX, cc = e / KX
#pragma unroll
        for (int it = 0; it < (KX * TB) / TPB; ++it) {
            const int e = tid + it * TPB;
            const int kk = e % KX, cc = e / KX;
            const int64_t kr = k0 + kk, c = c0 + cc;
            Ts[kk][cc] = (kr < k && c < nc) ? Tm[kr + c * ldt] : s_zero(T());
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < KX; ++kk) {
            T a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = Xs[kk][tx + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Ts[kk][ty + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = s_fma(a[i], b[j], acc[i][j]);
            if (DUAL) {
                T a2[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) a2[i] = X2s[kk][tx + 16 * i];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc2[i % (DUAL ? 4 : 1)][j % (DUAL ? 4 : 1)] =
                        s_fma(a2[i], b[j], acc2[i % (DUAL ? 4 : 1)][j % (DUAL ? 4 : 1)]);
            }
        }
        __syncthreads();
    }
    // epilogue
    double rs[4] = {0, 0, 0, 0};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int64_t c = c0 + ty + 16 * j;
        const double lc = (DUAL && lam && c < res_count) ? lam[c] : 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int64_t r = r0 + tx + 16 * i;
            if (r < n && c < nc) {
                T v = alpha == 1.0 ? acc[i][j] : s_rscale(alpha, acc[i][j]);
                if (beta != 0.0) v = s_add(v, s_rscale(beta, Y[r + c * ldy]));
                Y[r + c * ldy] = v;
                if (DUAL) {
                    const T w = acc2[i % (DUAL ? 4 : 1)][j % (DUAL ? 4 : 1)];
                    if (Y2) Y2[r + c * ldy2] = w;
                    if (lam && c < res_count) rs[j] += s_abs2(s_sub(w, s_rscale(lc, v)));
                }
            }
        }
    }
    if (DUAL && lam) {
        // reduce over tx (16 lanes of a half-warp share ty)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            double v = rs[j];
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            const int64_t c = c0 + ty + 16 * j;
            if (tx == 0 && c < res_count) rpart[(size_t)blockIdx.x * res_count + c] = v;
        }
    }
}

__global__ void resid_reduce_kernel(int64_t nblocks, int64_t res_count, const double* __restrict__ rpart,
                                    double* __restrict__ res) {
    const int c = blockIdx.x;
    __shared__ double sc[32];
    double v = 0.0;
    for (int64_t b = threadIdx.x; b < nblocks; b += blockDim.x) v += rpart[(size_t)b * res_count + c];
    v = block_sum(v, sc);
    if (threadIdx.x == 0) res[c] = sqrt(v);
}

template <class T>
static rc_status xt_t(rc_ctx* ctx, const XtArgs& a) {
    const unsigned gx = (unsigned)((a.n + TB - 1) / TB), gy = (unsigned)((a.nc + TB - 1) / TB);
    dim3 grid(gx, gy);
    const bool dual = a.X2 != nullptr;
    double* rpart = nullptr;
    if (dual && a.lam && a.res_count > 0) {
        void* p = nullptr;
        RC_TRY(rc_slot(ctx, S_RPART, (size_t)gx * a.res_count * sizeof(double), &p));
        rpart = (double*)p;
    }
    if (dual)
        xt_kernel<T, true><<<grid, TPB, 0, ctx->stream>>>(
            a.n, a.k, a.nc, (const T*)a.X, a.ldx, (const T*)a.T, a.ldt, (T*)a.Y, a.ldy, a.alpha, a.beta, (const T*)a.X2,
            a.ldx2, (T*)a.Y2, a.ldy2, rpart ? a.lam : nullptr, a.res_count, rpart);
    else
        xt_kernel<T, false><<<grid, TPB, 0, ctx->stream>>>(a.n, a.k, a.nc, (const T*)a.X, a.ldx, (const T*)a.T,
                                                           a.ldt, (T*)a.Y, a.ldy, a.alpha, a.beta, nullptr, 0, nullptr, 0,
                                                           nullptr, 0, nullptr);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    if (rpart) {
        resid_reduce_kernel<<<(unsigned)a.res_count, 256, 0, ctx->stream>>>(gx, a.res_count, rpart, a.res);
        ctx->launches++;
        RC_CU(ctx, cudaGetLastError());
    }
    return RC_OK;
}

rc_status xt(rc_ctx* ctx, int dtype, const XtArgs& a) {
    if (a.n <= 0 || a.nc <= 0) return RC_OK;
    // real fast path: plain products and residual-only dual products
    const bool plain = a.alpha == 1.0 && a.beta == 0.0;
    const bool dual_res_only =
        a.X2 != nullptr && a.Y2 == nullptr && a.lam != nullptr && (a.res_count > 0 || a.R32 != nullptr);
    if (plain && (a.X2 == nullptr || dual_res_only) && xt2_supported(dtype, a.k, a.nc))
        return xt2(ctx, a.n, a.k, a.nc, (const double*)a.X, a.ldx, (const double*)a.T, a.ldt, (double*)a.Y, a.ldy,
                   (const double*)a.X2, a.ldx2, a.lam, dual_res_only ? a.res_count : 0, a.res, a.R32, a.ldr, a.Yrm,
                   a.ldyr);
    if (a.R32 || a.Yrm)
        return rc_fail(ctx, RC_ERR_UNSUPPORTED, "xt: row-major outputs need a real block of <= 96 columns");
    return dtype == RC_COMPLEX128 ? xt_t<double2>(ctx, a) : xt_t<double>(ctx, a);
}

// ---------------------------------------------------------------------------------------
// Cholesky factor of the column-scaled Gram matrix (one CTA, 1024 threads).
//   d_i = sqrt(G_ii), Gh = D^-1 G D^-1 (+ sigma I on breakdown), Gh = R^H R (R upper),
//   Tout = D^-1 R^-1 so that V*Tout has orthonormal columns.
// The factor M and the inverse X live in dynamic shared memory when they fit (mode 2: both,
// mode 1: M only), otherwise in global scratch that stays L2-resident. The inverse is formed
// row by row from the bottom (X[i,j] for all j >= i in parallel), so no thread walks a long
// dependent chain.
// flags[0] |= 1 if shifted, flags[1] = 1 if failed, flags[2] = 1 if a zero column was met.
template <class T>
__global__ void __launch_bounds__(1024)
chol_factor_kernel(int s, int64_t nrows, const T* __restrict__ G, T* Mg, T* Tout, double* dscg, int* flags, double* pivout,
                   int mode) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_bad;
    __shared__ double s_minpiv;
    // In shared memory the matrices have an odd leading dimension (s + 1), so that a warp reading
    // along a row (consecutive columns) hits distinct banks. The block is 32 x (blockDim/32):
    // lane tx walks rows, warp ty walks columns, so no index needs a division.
    const int lm = mode >= 1 ? s + 1 : s;
    const int lx = mode == 2 ? s + 1 : s;
    T* M = mode >= 1 ? (T*)smem_raw : Mg;
    T* X = mode == 2 ? M + (size_t)s * lm : Tout;
    double* dsc = mode == 2 ? (double*)(X + (size_t)s * lx) : (mode == 1 ? (double*)(M + (size_t)s * lm) : dscg);
    const int tid = threadIdx.x, nt = blockDim.x;
    const int tx = tid & 31, ty = tid >> 5, nwy = nt >> 5;
    for (int i = tid; i < s; i += nt) {
        const double gi = s_real(G[i + (int64_t)i * s]);
        double d = (gi > 0.0 && isfinite(gi)) ? sqrt(gi) : 0.0;
        if (d == 0.0) {
            atomicOr(flags + 2, 1);
            d = 1.0;
        }
        dsc[i] = d;
    }
    if (tid == 0) s_bad = 0;
    __syncthreads();
    const double eps = 2.220446049250313e-16;
    // Fukaya et al. shift 11 (m n + n (n+1)) u ||Gh||_2 with ||Gh||_2 <= trace(Gh) = s.
    const double sigma = 11.0 * ((double)nrows * s + (double)s * (s + 1)) * eps * (double)s;
    for (int attempt = 0; attempt < 2; ++attempt) {
        const double shift = attempt == 0 ? 0.0 : sigma;
        if (tid == 0) s_minpiv = 1e300;
        for (int j = ty; j < s; j += nwy)
            for (int i = tx; i < s; i += 32) {
                T g = G[i + (int64_t)j * s];
                if (!isfinite(s_real(g)) || !isfinite(s_imag(g))) g = s_zero(T());
                g = s_rscale(1.0 / (dsc[i] * dsc[j]), g);
                if (i == j) g = s_from<T>(s_real(g) + shift, 0.0);
                M[i + (int64_t)j * lm] = g;
            }
        __syncthreads();
        // right-looking upper Cholesky with one barrier per step: row k is final once step k-1
        // is done, so every thread reads the pivot p_k itself and updates the trailing matrix with
        // the unscaled row, M[i,j] -= conj(M[k,i]) M[k,j] / p_k (k < i <= j); the rows are scaled
        // by sqrt(p_k) after the loop.
        bool bad = false;
        for (int k = 0; k < s; ++k) {
            const double p = s_real(M[k + (int64_t)k * lm]);
            if (!(p > 1e-13)) bad = true;
            if (tid == 0) s_minpiv = fmin(s_minpiv, p);
            if (bad && attempt == 0) break;
            const double pinv = 1.0 / (p > 1e-300 ? p : 1e-300);
            for (int j = k + 1 + ty; j < s; j += nwy) {
                const T mkj = s_rscale(pinv, M[k + (int64_t)j * lm]);
                for (int i = k + 1 + tx; i <= j; i += 32)
                    M[i + (int64_t)j * lm] = s_sub(M[i + (int64_t)j * lm], s_mul(s_conj(M[k + (int64_t)i * lm]), mkj));
            }
            __syncthreads();
        }
        if (tid == 0 && bad) s_bad = 1;
        __syncthreads();
        if (!s_bad) break;
        if (attempt == 0) {
            if (tid == 0) {
                flags[0] |= 1;
                s_bad = 0;
            }
            __syncthreads();
        } else {
            if (tid == 0) flags[1] = 1;
        }
    }
    __syncthreads();
    // R[k,j] = M[k,j] / sqrt(p_k) (j > k), R[k,k] = sqrt(p_k); the pivots go through X first
    for (int k = tid; k < s; k += nt) {
        const double p = s_real(M[k + (int64_t)k * lm]);
        X[k] = s_from<T>(sqrt(p > 1e-300 ? p : 1e-300), 0.0);
    }
    __syncthreads();
    for (int j = ty; j < s; j += nwy)
        for (int i = tx; i <= j; i += 32) {
            const double rkk = s_real(X[i]);
            if (j > i) M[i + (int64_t)j * lm] = s_rscale(1.0 / rkk, M[i + (int64_t)j * lm]);
            else M[i + (int64_t)i * lm] = s_from<T>(rkk, 0.0);
        }
    __syncthreads();
    // X = R^-1 (upper), right-looking back substitution on all columns at once with one barrier
    // per step: Y starts as I; at step k (s-1 .. 1) row k of Y is final, and R[l,k] Y[k,:]/R[k,k]
    // is removed from the rows l < k. X[k,:] = Y[k,:]/R[k,k] is applied in the last pass.
    for (int j = ty; j < s; j += nwy)
        for (int i = tx; i < s; i += 32) X[i + (int64_t)j * lx] = s_from<T>(i == j ? 1.0 : 0.0, 0.0);
    __syncthreads();
    for (int k = s - 1; k >= 1; --k) {
        const double inv = 1.0 / s_real(M[k + (int64_t)k * lm]);
        for (int j = k + ty; j < s; j += nwy) {
            const T ykj = s_rscale(inv, X[k + (int64_t)j * lx]);
            for (int l = tx; l < k; l += 32)
                X[l + (int64_t)j * lx] = s_sub(X[l + (int64_t)j * lx], s_mul(M[l + (int64_t)k * lm], ykj));
        }
        __syncthreads();
    }
    if (tid == 0 && pivout) pivout[0] = s_minpiv;
    // Tout = D^-1 X = D^-1 diag(R)^-1 Y
    for (int j = ty; j < s; j += nwy)
        for (int i = tx; i < s; i += 32)
            Tout[i + (int64_t)j * s] = s_rscale(1.0 / (dsc[i] * s_real(M[i + (int64_t)i * lm])), X[i + (int64_t)j * lx]);
}

rc_status chol_factor(rc_ctx* ctx, int dtype, int64_t s, int64_t nrows, const void* G, void* Tout, int* flags,
                      double* pivout) {
    const size_t esz = dtype == RC_COMPLEX128 ? 16 : 8;
    void* base = nullptr;
    RC_TRY(rc_slot(ctx, S_LANCZOS, (size_t)s * s * esz + (size_t)s * 8 + 256, &base));
    double* dsc = (double*)((char*)base + (size_t)s * s * esz);
    const size_t budget = ctx->smem_optin > 4096 ? ctx->smem_optin - 4096 : 0;
    const size_t mat = (size_t)s * (s + 1) * esz;  // with the padded leading dimension
    int mode = 0;
    size_t dyn = 0;
    if (2 * mat + (size_t)s * 8 <= budget) {
        mode = 2;
        dyn = 2 * mat + (size_t)s * 8;
    } else if (mat + (size_t)s * 8 <= budget) {
        mode = 1;
        dyn = mat + (size_t)s * 8;
    }
    if (dtype == RC_COMPLEX128) {
        if (dyn > 48 * 1024)
            RC_CU(ctx, allow_max_smem(ctx, chol_factor_kernel<double2>));
        chol_factor_kernel<double2><<<1, 1024, dyn, ctx->stream>>>((int)s, nrows, (const double2*)G, (double2*)base,
                                                                  (double2*)Tout, dsc, flags, pivout, mode);
    } else {
        if (dyn > 48 * 1024)
            RC_CU(ctx, allow_max_smem(ctx, chol_factor_kernel<double>));
        chol_factor_kernel<double><<<1, 1024, dyn, ctx->stream>>>((int)s, nrows, (const double*)G, (double*)base,
                                                                 (double*)Tout, dsc, flags, pivout, mode);
    }
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    return RC_OK;
}

// ---------------------------------------------------------------------------------------
// Parallel cyclic Jacobi (Brent-Luk round-robin ordering), one CTA.
// A: s x s Hermitian (col-major, ld s, not modified), Q: eigenvectors (ld s), evals ascending.
// Rotation for pair (p,q), u = a_pq/|a_pq|:  G = [[c, s u], [-s conj(u), c]] on (p,q);
// A <- G^H A G zeroes a_pq (Golub & Van Loan, Alg. 8.4.1 after removing the phase of a_pq).
// Each round applies the s/2 disjoint rotations of the round-robin schedule at once: every
// thread owns 2x2 blocks A[{p_i,q_i},{p_j,q_j}] <- G_i^H A G_j (rows and columns in one pass)
// and, independently, pairs of columns of Q <- Q G_j. The working copies use an odd leading
// dimension (bank-conflict free rows and columns) in shared memory when they fit, otherwise
// in global scratch `work` (2*sp*(sp+1) scalars).
template <class T>
__device__ __forceinline__ void rr_pair(int r, int i, int M, int sp, int& p, int& q) {
    if (i == 0) {
        p = r % M;
        q = sp - 1;
    } else {
        p = (r + i) % M;
        q = (r - i + M) % M;
    }
    if (p > q) {
        const int t = p;
        p = q;
        q = t;
    }
}

// Whether pair (p, q) rotates: |a_pq| above the absolute and the relative threshold.
template <class T>
__device__ __forceinline__ bool jac_rotates(T apq, double app, double aqq, double abs_tol, double rel_tol) {
    if constexpr (!IsComplex<T>::value) {
        const double mag = fabs(s_real(apq));
        return mag > abs_tol && mag * mag > rel_tol * rel_tol * fabs(app * aqq);
    } else {
        const double mag = sqrt(s_abs2(apq));
        return mag > abs_tol && mag > rel_tol * sqrt(fabs(app * aqq));
    }
}

// Whether any pair of the s x s working copy A (leading dimension ld) would rotate: if none does, a
// sweep would change nothing. All threads of the CTA call it and get the same answer.
template <class T>
__device__ __forceinline__ bool jac_any_rotation(const T* A, int s, int ld, double abs_tol, double rel_tol) {
    int any = 0;
    for (int e = threadIdx.x; e < s * s; e += blockDim.x) {
        const int p = e % s, q = e / s;
        if (p < q && jac_rotates<T>(A[p + q * ld], s_real(A[p + p * ld]), s_real(A[q + q * ld]), abs_tol, rel_tol))
            any = 1;
    }
    return __syncthreads_or(any) != 0;
}

// Upper-triangle block index e -> (bi, bj), bi <= bj, bj-major: e = bj (bj + 1) / 2 + bi.
__device__ __forceinline__ void jac_tri(int e, int& bi, int& bj) {
    int j = (int)((sqrtf(8.0f * (float)e + 1.0f) - 1.0f) * 0.5f);
    while ((j + 1) * (j + 2) / 2 <= e) ++j;
    while (j * (j + 1) / 2 > e) --j;
    bj = j;
    bi = e - j * (j + 1) / 2;
}

// Rotation angle of pair (p, q) from a_pq, a_pp, a_qq; *sn = 0 (no rotation) when |a_pq| is below
// the absolute or relative threshold.
template <class T>
__device__ __forceinline__ void jac_angle(T apq, double app, double aqq, double abs_tol, double rel_tol, double& c,
                                          double& sn, T& u) {
    c = 1.0;
    sn = 0.0;
    u = s_from<T>(1.0, 0.0);
    if (!jac_rotates<T>(apq, app, aqq, abs_tol, rel_tol)) return;
    if constexpr (!IsComplex<T>::value) {
        // real: u = sign(apq), and the angle from one square root and one division,
        // t = sign(d) 2|apq| / (|d| + sqrt(d^2 + 4 apq^2)) with d = aqq - app
        const double mag = fabs(s_real(apq));
        {
            u = s_from<T>(s_real(apq) >= 0.0 ? 1.0 : -1.0, 0.0);
            const double d = aqq - app;
            const double t = copysign(2.0 * mag, d) / (fabs(d) + sqrt(d * d + 4.0 * mag * mag));
            c = rsqrt(1.0 + t * t);
            sn = t * c;
        }
    } else {
        const double mag = sqrt(s_abs2(apq));
        {
            u = s_rscale(1.0 / mag, apq);
            const double tau = (aqq - app) / (2.0 * mag);
            const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = 1.0 / sqrt(1.0 + t * t);
            sn = t * c;
        }
    }
}

// The 2x2 block A[{p_i,q_i},{p_j,q_j}] <- G_i^H A G_j: columns [b_p b_q] = [a_p a_q] G_j, then rows
// G_i^H [b_p.; b_q.]. On a diagonal block (bi == bj) with a rotation the off-diagonal entries are set
// to exact zeros and the diagonal to its real part.
template <class T>
__device__ __forceinline__ void jac_block(T& a_pp, T& a_qp, T& a_pq, T& a_qq, double ci, double si, T ui, double cj,
                                          double sj, T uj, bool diag) {
    const T sju = s_rscale(sj, uj), sjc = s_rscale(sj, s_conj(uj));
    const T b_pp = s_sub(s_rscale(cj, a_pp), s_mul(sjc, a_pq));
    const T b_qp = s_sub(s_rscale(cj, a_qp), s_mul(sjc, a_qq));
    const T b_pq = s_add(s_mul(sju, a_pp), s_rscale(cj, a_pq));
    const T b_qq = s_add(s_mul(sju, a_qp), s_rscale(cj, a_qq));
    const T siu = s_rscale(si, ui), sic = s_rscale(si, s_conj(ui));
    a_pp = s_sub(s_rscale(ci, b_pp), s_mul(siu, b_qp));
    a_qp = s_add(s_mul(sic, b_pp), s_rscale(ci, b_qp));
    a_pq = s_sub(s_rscale(ci, b_pq), s_mul(siu, b_qq));
    a_qq = s_add(s_mul(sic, b_pq), s_rscale(ci, b_qq));
    if (diag && si != 0.0) {
        a_qp = s_zero(T());
        a_pq = s_zero(T());
        a_pp = s_from<T>(s_real(a_pp), 0.0);
        a_qq = s_from<T>(s_real(a_qq), 0.0);
    }
}

// Row entries (q_p, q_q) of columns p_j, q_j of Q <- Q G_j.
template <class T>
__device__ __forceinline__ void jac_qrot(T& qp, T& qq, double cj, double sj, T uj) {
    const T np = s_sub(s_rscale(cj, qp), s_mul(s_rscale(sj, s_conj(uj)), qq));
    qq = s_add(s_mul(s_rscale(sj, uj), qp), s_rscale(cj, qq));
    qp = np;
}

// Threads of the one-CTA Jacobi (a multiple of 32, at most 1024).
#ifndef RC_JACOBI_THREADS
#define RC_JACOBI_THREADS 1024
#endif

template <class T>
__global__ void __launch_bounds__(1024)
jacobi_kernel(int s, const T* __restrict__ Ain, T* __restrict__ Qout, double* __restrict__ evals, int* info,
              T* work, int use_smem, int max_sweeps) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int sp = s + (s & 1);  // even number of indices (one zero dummy row/column when s is odd)
    const int npair = sp / 2;
    const int ld = sp + 1;       // odd leading dimension
    double* rc = (double*)smem_raw;
    double* rsn = rc + npair;
    T* ru = (T*)(rsn + npair);
    int* pp = (int*)(ru + npair);
    int* qq = pp + npair;
    T* A;
    T* Q;
    if (use_smem) {
        A = (T*)((char*)smem_raw + (((size_t)npair * (16 + sizeof(T) + 8) + 15) / 16) * 16);
    } else {
        A = work;
    }
    Q = A + (size_t)sp * ld;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = tid; e < sp * sp; e += nt) {
        const int i = e % sp, j = e / sp;
        A[i + j * ld] = (i < s && j < s) ? Ain[i + (int64_t)j * s] : s_zero(T());
        Q[i + j * ld] = s_from<T>(i == j ? 1.0 : 0.0, 0.0);
    }
    __shared__ double s_fro;
    __shared__ int s_rot;
    __shared__ unsigned long long s_maxsn;  // largest |sin| of the sweep's rotations (bits of a positive double)
    __shared__ double red[32];
    __syncthreads();
    double f = 0.0;
    for (int e = tid; e < sp * sp; e += nt) f += s_abs2(A[(e % sp) + (e / sp) * ld]);
    f = block_sum(f, red);
    if (tid == 0) s_fro = sqrt(f);
    __syncthreads();
    const double abs_tol = 1e-17 * s_fro;
    const double rel_tol = 1e-15;
    const int M = sp - 1;
    int sweep = 0;
    const int nblk = npair * (npair + 1) / 2;  // 2x2 blocks with bi <= bj
    // A thread's work is the same in every round: the 2x2 blocks tid, tid + nt, ... of the bj-major
    // upper triangle (for real matrices the first two mapped here once, any later ones per round;
    // complex ones, whose updates need more registers, all per round) and the (row, pair) entries
    // tid, tid + nt, ... of Q, walked by adding nt in (pair, row) form without a division.
    constexpr int kPre = IsComplex<T>::value ? 0 : 2;
    int blk_i[2], blk_j[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        blk_i[k] = -1;
        blk_j[k] = 0;
        if (k < kPre && tid + k * nt < nblk) jac_tri(tid + k * nt, blk_i[k], blk_j[k]);
    }
    const int q_b0 = tid / s, q_r0 = tid - (tid / s) * s;
    const int q_db = nt / s, q_dr = nt - (nt / s) * s;
    // A <- G^H A G on the 2x2 block (row pair bi, column pair bj); A stays Hermitian, so only the
    // blocks with bi <= bj are formed and each is mirrored into (bj, bi)
    auto block_update = [&](int bi, int bj) {
        const double si = rsn[bi], sj = rsn[bj];
        if (si == 0.0 && sj == 0.0) return;
        const int pi = pp[bi], qi = qq[bi], pj = pp[bj], qj = qq[bj];
        T a_pp = A[pi + pj * ld], a_qp = A[qi + pj * ld];
        T a_pq = A[pi + qj * ld], a_qq = A[qi + qj * ld];
        jac_block<T>(a_pp, a_qp, a_pq, a_qq, rc[bi], si, ru[bi], rc[bj], sj, ru[bj], bi == bj);
        A[pi + pj * ld] = a_pp;
        A[qi + pj * ld] = a_qp;
        A[pi + qj * ld] = a_pq;
        A[qi + qj * ld] = a_qq;
        if (bi != bj) {
            A[pj + pi * ld] = s_conj(a_pp);
            A[pj + qi * ld] = s_conj(a_qp);
            A[qj + pi * ld] = s_conj(a_pq);
            A[qj + qi * ld] = s_conj(a_qq);
        }
    };
    for (; sweep < max_sweeps; ++sweep) {
        // a sweep in which no pair rotates changes nothing: stop before it
        if (!jac_any_rotation<T>(A, s, ld, abs_tol, rel_tol)) break;
        if (tid == 0) {
            s_rot = 0;
            s_maxsn = 0ull;
        }
        __syncthreads();
        for (int r = 0; r < M; ++r) {
            unsigned long long snbits = 0ull;  // this thread's largest |sin| (bits of a positive double)
            for (int i = tid; i < npair; i += nt) {
                int p, q;
                rr_pair<T>(r, i, M, sp, p, q);
                double c = 1.0, sn = 0.0;
                T u = s_from<T>(1.0, 0.0);
                if (q < s) {
                    jac_angle<T>(A[p + q * ld], s_real(A[p + p * ld]), s_real(A[q + q * ld]), abs_tol, rel_tol, c, sn,
                                 u);
                    snbits = max(snbits, (unsigned long long)__double_as_longlong(fabs(sn)));
                }
                rc[i] = c;
                rsn[i] = sn;
                ru[i] = u;
                pp[i] = p;
                qq[i] = q;
            }
            // one shared-memory atomic per warp that computed angles (a rotation has sin != 0)
            if (tid < ((npair + 31) & ~31)) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) snbits = max(snbits, __shfl_xor_sync(0xffffffffu, snbits, o));
                if ((tid & 31) == 0 && snbits) {
                    atomicMax(&s_maxsn, snbits);
                    s_rot = 1;
                }
            }
            __syncthreads();
            // the 2x2 blocks, spread evenly over the threads
#pragma unroll
            for (int k = 0; k < kPre; ++k)
                if (blk_i[k] >= 0) block_update(blk_i[k], blk_j[k]);
            for (int e = tid + kPre * nt; e < nblk; e += nt) {
                int bi, bj;
                jac_tri(e, bi, bj);
                block_update(bi, bj);
            }
            // Q <- Q G_j (columns p_j, q_j of rows 0..s-1), the (row, pair) entries spread evenly
            // over the threads, rows fastest
            for (int bj = q_b0, row = q_r0; bj < npair;) {
                const double sj = rsn[bj];
                if (sj != 0.0) {
                    const int pj = pp[bj], qj = qq[bj];
                    T qp = Q[row + pj * ld], qv = Q[row + qj * ld];
                    jac_qrot<T>(qp, qv, rc[bj], sj, ru[bj]);
                    Q[row + pj * ld] = qp;
                    Q[row + qj * ld] = qv;
                }
                row += q_dr;
                bj += q_db;
                if (row >= s) {
                    row -= s;
                    ++bj;
                }
            }
            __syncthreads();
        }
        const int rot = s_rot;
        const double maxsn = __longlong_as_double((long long)s_maxsn);
        __syncthreads();
        // no rotation, or only rotations so small (|sin| < 1e-9) that the off-diagonal entries
        // they leave (of order sin^2) are below the rotation threshold of another sweep
        if (!rot || maxsn < 1e-9) {
            if (rot) ++sweep;
            break;
        }
    }
    // ascending order (rank sort, ties by index) over the s real indices
    for (int i = tid; i < s; i += nt) {
        const double li = s_real(A[i + i * ld]);
        int rank = 0;
        for (int j = 0; j < s; ++j) {
            const double lj = s_real(A[j + j * ld]);
            if (lj < li || (lj == li && j < i)) ++rank;
        }
        evals[rank] = li;
        for (int row = 0; row < s; ++row) Qout[row + (int64_t)rank * s] = Q[row + i * ld];
    }
    if (tid == 0 && info) info[0] = sweep;
}

// ---------------------------------------------------------------------------------------
// The same Jacobi over a grid of CTAs, for matrices whose working copies do not fit in one CTA's
// shared memory (complex s > 82, real s > 118). The working copies stay in global memory (L2), and
// one round's updates, which touch every entry of A and Q, are split over the CTAs: CTA b forms a
// contiguous share of the 2x2 blocks (bi <= bj) and of the (row, pair) entries of Q, then all CTAs
// meet at a grid barrier. Every CTA computes all the round's angles itself from the same entries,
// so the rotations, the convergence test and the number of sweeps agree in every CTA without
// further communication. A is kept twice: a round reads one copy and writes every entry of the
// other (blocks without a rotation are copied), because the CTAs leave the barrier at different
// times and one CTA's block updates must not reach the entries another CTA is still reading for
// its angles. Each (row, pair) entry of Q is read and written by one thread only, so Q is kept
// once. Global reads and writes of the working copies bypass L1 (ld/st .cg):
// another SM may have written them since the last barrier. The grid is launched cooperatively
// (all CTAs resident); the barrier's spin is bounded all the same, and on a timeout the kernel
// stops, writes -1 to info[0] and NaN eigenvalues.
// ---------------------------------------------------------------------------------------
constexpr int kJacGridThreads = 256;
constexpr long long kJacBarrierSpins = 1ll << 26;  // ~ seconds with the back-off below

// Grid barrier over `nblocks` CTAs on two words: bar[0] counts arrivals, bar[1] is the generation.
// Thread 0 arrives with an acquire-release add (after the CTA barrier, it releases the CTA's
// writes; the last arrival also acquires every other CTA's). The last arrival resets the count and
// publishes the next generation with a release store; the others poll the generation with acquire
// loads, so each CTA sees every CTA's writes once it leaves. bar[2] is the give-up flag: a CTA
// whose wait runs out sets it, and the CTAs waiting at this or a later barrier read it while they
// poll and stop too. Returns false when this CTA gave up.
__device__ __forceinline__ unsigned jac_ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned jac_ld_relaxed(const unsigned* p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ bool jac_grid_barrier(unsigned* bar, unsigned nblocks, unsigned& gen) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        unsigned old;
        asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(bar) : "memory");
        if (old == nblocks - 1) {
            asm volatile("st.relaxed.gpu.global.u32 [%0], 0;" ::"l"(bar) : "memory");
            asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(bar + 1), "r"(gen + 1) : "memory");
        } else {
            long long spins = 0;
            while (jac_ld_acquire(bar + 1) == gen) {
                if (++spins > kJacBarrierSpins || jac_ld_relaxed(bar + 2) != 0u) {
                    atomicExch(&bar[2], 1u);
                    ok = 0;
                    break;
                }
                if (spins > 64) __nanosleep(32);
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    ++gen;
    return s_ok != 0;
}

template <class T>
__global__ void __launch_bounds__(kJacGridThreads)
jacobi_grid_kernel(int s, const T* __restrict__ Ain, T* __restrict__ Qout, double* __restrict__ evals, int* info,
                   T* work, int max_sweeps) {
    const int sp = s + (s & 1);
    const int npair = sp / 2;
    const int ld = sp + 1;
    T* const Abuf[2] = {work, work + (size_t)sp * ld};  // the round's source and destination copies of A
    T* Q = work + 2 * (size_t)sp * ld;
    int par = 0;                                        // Abuf[par] holds the current A
    unsigned* bar = reinterpret_cast<unsigned*>(info + 1);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* rc = (double*)smem_raw;
    double* rsn = rc + npair;
    T* ru = (T*)(rsn + npair);
    int* pp = (int*)(ru + npair);
    int* qq = pp + npair;
    __shared__ int s_rot;
    __shared__ unsigned long long s_maxsn;
    __shared__ double red[32];
    const int tid = threadIdx.x, nt = blockDim.x;
    const int G = gridDim.x, b = blockIdx.x;
    unsigned gen = 0;
    bool ok = true;
    // working copies: CTA b initialises its share of the entries
    {
        const int64_t tot = (int64_t)sp * sp;
        for (int64_t e = (int64_t)b * nt + tid; e < tot; e += (int64_t)G * nt) {
            const int i = (int)(e % sp), j = (int)(e / sp);
            __stcg(Abuf[0] + i + (int64_t)j * ld, (i < s && j < s) ? Ain[i + (int64_t)j * s] : s_zero(T()));
            __stcg(Q + i + (int64_t)j * ld, s_from<T>(i == j ? 1.0 : 0.0, 0.0));
        }
    }
    // the Frobenius norm of the input, in the same order in every CTA
    double f = 0.0;
    for (int e = tid; e < s * s; e += nt) f += s_abs2(Ain[e]);
    f = block_sum(f, red);
    const double abs_tol = 1e-17 * sqrt(f);
    const double rel_tol = 1e-15;
    const int M = sp - 1;
    const int64_t nblk = (int64_t)npair * (npair + 1) / 2;         // 2x2 blocks with bi <= bj
    const int64_t blk0 = nblk * b / G, blk1 = nblk * (b + 1) / G;  // this CTA's share
    const int64_t nq = (int64_t)s * npair;                         // (row, pair) entries of Q
    const int64_t q0 = nq * b / G, q1 = nq * (b + 1) / G;
    // the first block and Q entry of this thread, mapped once; later ones are reached by adding nt
    // (the upper triangle has bj + 1 blocks in column bj; Q entries are (pair, row) with s rows)
    int blk_bi0 = 0, blk_bj0 = 0;
    if (blk0 + tid < blk1) {
        const int64_t e = blk0 + tid;
        int bj = (int)((sqrt(8.0 * (double)e + 1.0) - 1.0) * 0.5);
        while ((int64_t)(bj + 1) * (bj + 2) / 2 <= e) ++bj;
        while ((int64_t)bj * (bj + 1) / 2 > e) --bj;
        blk_bj0 = bj;
        blk_bi0 = (int)(e - (int64_t)bj * (bj + 1) / 2);
    }
    const int q_b0 = (int)((q0 + tid) / s), q_r0 = (int)((q0 + tid) - (int64_t)q_b0 * s);
    const int q_db = nt / s, q_dr = nt - (nt / s) * s;
    ok = jac_grid_barrier(bar, G, gen);
    int sweep = 0;
    for (; ok && sweep < max_sweeps; ++sweep) {
        // a sweep in which no pair rotates changes nothing: stop before it (every CTA reads the same
        // entries, written before the last barrier and not again before the next one, so all stop
        // together)
        {
            const T* A = Abuf[par];
            int any = 0;
            for (int e = tid; e < s * s; e += nt) {
                const int p = e % s, q = e / s;
                if (p < q && jac_rotates<T>(__ldcg(A + p + (int64_t)q * ld), s_real(__ldcg(A + p + (int64_t)p * ld)),
                                            s_real(__ldcg(A + q + (int64_t)q * ld)), abs_tol, rel_tol))
                    any = 1;
            }
            if (!__syncthreads_or(any)) break;
        }
        if (tid == 0) {
            s_rot = 0;
            s_maxsn = 0ull;
        }
        __syncthreads();
        for (int r = 0; r < M && ok; ++r) {
            const T* A = Abuf[par];   // read by every CTA during this round, written by none
            T* An = Abuf[par ^ 1];    // this round's result
            unsigned long long snbits = 0ull;
            for (int i = tid; i < npair; i += nt) {
                int p, q;
                rr_pair<T>(r, i, M, sp, p, q);
                double c = 1.0, sn = 0.0;
                T u = s_from<T>(1.0, 0.0);
                if (q < s) {
                    jac_angle<T>(__ldcg(A + p + (int64_t)q * ld), s_real(__ldcg(A + p + (int64_t)p * ld)),
                                 s_real(__ldcg(A + q + (int64_t)q * ld)), abs_tol, rel_tol, c, sn, u);
                    snbits = max(snbits, (unsigned long long)__double_as_longlong(fabs(sn)));
                }
                rc[i] = c;
                rsn[i] = sn;
                ru[i] = u;
                pp[i] = p;
                qq[i] = q;
            }
            if (tid < ((npair + 31) & ~31)) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) snbits = max(snbits, __shfl_xor_sync(0xffffffffu, snbits, o));
                if ((tid & 31) == 0 && snbits) {
                    atomicMax(&s_maxsn, snbits);
                    s_rot = 1;
                }
            }
            __syncthreads();
            // this CTA's 2x2 blocks: linear index e over bj-major upper triangle (bi <= bj)
            int bi = blk_bi0, bj = blk_bj0;
            for (int64_t e = blk0 + tid; e < blk1; e += nt, bi += nt) {
                while (bi > bj) {  // step to the block nt further along the triangle
                    bi -= bj + 1;
                    ++bj;
                }
                const double si = rsn[bi], sj = rsn[bj];
                const int pi = pp[bi], qi = qq[bi], pj = pp[bj], qj = qq[bj];
                const int64_t o0 = pi + (int64_t)pj * ld, o1 = qi + (int64_t)pj * ld;
                const int64_t o2 = pi + (int64_t)qj * ld, o3 = qi + (int64_t)qj * ld;
                T a_pp = __ldcg(A + o0), a_qp = __ldcg(A + o1), a_pq = __ldcg(A + o2), a_qq = __ldcg(A + o3);
                const int64_t m0 = pj + (int64_t)pi * ld, m1 = pj + (int64_t)qi * ld;
                const int64_t m2 = qj + (int64_t)pi * ld, m3 = qj + (int64_t)qi * ld;
                if (si == 0.0 && sj == 0.0) {
                    // no rotation touches this block: both halves carried over unchanged
                    __stcg(An + o0, a_pp);
                    __stcg(An + o1, a_qp);
                    __stcg(An + o2, a_pq);
                    __stcg(An + o3, a_qq);
                    if (bi != bj) {
                        __stcg(An + m0, __ldcg(A + m0));
                        __stcg(An + m1, __ldcg(A + m1));
                        __stcg(An + m2, __ldcg(A + m2));
                        __stcg(An + m3, __ldcg(A + m3));
                    }
                    continue;
                }
                jac_block<T>(a_pp, a_qp, a_pq, a_qq, rc[bi], si, ru[bi], rc[bj], sj, ru[bj], bi == bj);
                __stcg(An + o0, a_pp);
                __stcg(An + o1, a_qp);
                __stcg(An + o2, a_pq);
                __stcg(An + o3, a_qq);
                if (bi != bj) {
                    __stcg(An + m0, s_conj(a_pp));
                    __stcg(An + m1, s_conj(a_qp));
                    __stcg(An + m2, s_conj(a_pq));
                    __stcg(An + m3, s_conj(a_qq));
                }
            }
            // this CTA's (row, pair) entries of Q <- Q G_j, rows fastest (coalesced columns)
            int qb = q_b0, qr = q_r0;
            for (int64_t e = q0 + tid; e < q1; e += nt) {
                const double sj = rsn[qb];
                if (sj != 0.0) {
                    T* qpp = Q + qr + (int64_t)pp[qb] * ld;
                    T* qqp = Q + qr + (int64_t)qq[qb] * ld;
                    T qp = __ldcg(qpp), qv = __ldcg(qqp);
                    jac_qrot<T>(qp, qv, rc[qb], sj, ru[qb]);
                    __stcg(qpp, qp);
                    __stcg(qqp, qv);
                }
                qr += q_dr;
                qb += q_db;
                if (qr >= s) {
                    qr -= s;
                    ++qb;
                }
            }
            ok = jac_grid_barrier(bar, G, gen);
            par ^= 1;
        }
        const int rot = s_rot;
        const double maxsn = __longlong_as_double((long long)s_maxsn);
        __syncthreads();
        if (!ok) break;
        if (!rot || maxsn < 1e-9) {
            if (rot) ++sweep;
            break;
        }
    }
    if (!ok) {
        for (int i = b * nt + tid; i < s; i += G * nt) evals[i] = __longlong_as_double(0x7ff8000000000000ll);
        if (b == 0 && tid == 0 && info) info[0] = -1;
        return;
    }
    // ascending order (rank sort, ties by index); CTA b writes the columns i = b, b + G, ...
    const T* A = Abuf[par];
    for (int i = b; i < s; i += G) {
        const double li = s_real(__ldcg(A + i + (int64_t)i * ld));
        int rank = 0;
        for (int j = tid; j < s; j += nt) {
            const double lj = s_real(__ldcg(A + j + (int64_t)j * ld));
            if (lj < li || (lj == li && j < i)) ++rank;
        }
        rank = (int)block_sum((double)rank, red);
        if (tid == 0) evals[rank] = li;
        for (int row = tid; row < s; row += nt) Qout[row + (int64_t)rank * s] = __ldcg(Q + row + (int64_t)i * ld);
    }
    if (b == 0 && tid == 0 && info) info[0] = sweep;
}

size_t small_eigh_work_bytes(rc_ctx* ctx, int dtype, int64_t s) {
    const size_t esz = dtype == RC_COMPLEX128 ? 16 : 8;
    const int64_t sp = s + (s & 1);
    const int64_t npair = sp / 2;
    const size_t head = (((size_t)npair * (16 + esz + 8) + 15) / 16) * 16;
    const size_t mats = 2 * (size_t)sp * (sp + 1) * esz;
    // in global memory the grid form keeps A twice (3 matrices); the one-CTA kernel uses 2 of them
    return head + mats <= (size_t)ctx->smem_optin - 2048 ? 0 : 3 * (size_t)sp * (sp + 1) * esz;
}

rc_status small_eigh(rc_ctx* ctx, int dtype, int64_t s, void* A, void* Q, double* evals, int* info) {
    void* work = nullptr;
    const size_t wb = small_eigh_work_bytes(ctx, dtype, s);
    if (wb) RC_TRY(rc_slot(ctx, S_EIG, wb + 256, &work));
    return small_eigh_work(ctx, dtype, s, A, Q, evals, info, work);
}

rc_status small_eigh_work(rc_ctx* ctx, int dtype, int64_t s, void* A, void* Q, double* evals, int* info, void* work) {
    const size_t esz = dtype == RC_COMPLEX128 ? 16 : 8;
    const int64_t sp = s + (s & 1);
    const int64_t npair = sp / 2;
    const size_t head = (((size_t)npair * (16 + esz + 8) + 15) / 16) * 16;
    const size_t mats = 2 * (size_t)sp * (sp + 1) * esz;
    const bool fit = head + mats <= (size_t)ctx->smem_optin - 2048;
    const size_t dyn = fit ? head + mats : head;
    if (!fit && !work) return rc_fail(ctx, RC_ERR_INVALID, "small_eigh: work memory required");
    const int sweeps = 60;
    // working copies in global memory: the grid form over up to 32 CTAs (RCB200_JACOBI_CTAS; 1 keeps
    // the one-CTA kernel), launched cooperatively, with its barrier words in info[1..3]
    const int ctas = std::max(1, std::min(ctx->jacobi_ctas > 0 ? ctx->jacobi_ctas : 32, ctx->sm_count));
    if (!fit && ctas > 1 && info) {
        RC_CU(ctx, cudaMemsetAsync(info + 1, 0, 3 * sizeof(int), ctx->stream));
        int si = (int)s;
        int sw = sweeps;
        void* args[] = {&si, &A, &Q, &evals, &info, &work, &sw};
        const void* kern = dtype == RC_COMPLEX128 ? (const void*)jacobi_grid_kernel<double2>
                                                  : (const void*)jacobi_grid_kernel<double>;
        RC_CU(ctx, cudaLaunchCooperativeKernel(kern, dim3((unsigned)ctas), dim3(kJacGridThreads), args, dyn,
                                               ctx->stream));
        ctx->launches++;
        return RC_OK;
    }
    const int nthr = ctx->jacobi_threads > 0 ? ctx->jacobi_threads : RC_JACOBI_THREADS;
    if (dtype == RC_COMPLEX128) {
        if (dyn > 48 * 1024)
            RC_CU(ctx, allow_max_smem(ctx, jacobi_kernel<double2>));
        jacobi_kernel<double2><<<1, nthr, dyn, ctx->stream>>>((int)s, (const double2*)A, (double2*)Q, evals, info,
                                                              (double2*)work, fit ? 1 : 0, sweeps);
    } else {
        if (dyn > 48 * 1024)
            RC_CU(ctx, allow_max_smem(ctx, jacobi_kernel<double>));
        jacobi_kernel<double><<<1, nthr, dyn, ctx->stream>>>((int)s, (const double*)A, (double*)Q, evals, info,
                                                             (double*)work, fit ? 1 : 0, sweeps);
    }
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    return RC_OK;
}
// ---------------------------------------------------------------------------------------
// Small dense helpers on s x s matrices (column-major, ld s): C = op(A) B and C <- (C + C^H)/2.
// One thread per output element; the operands stay in L1/L2.
// ---------------------------------------------------------------------------------------
template <class T>
__global__ void small_gemm_kernel(int s, const T* __restrict__ A, int transA, const T* __restrict__ B,
                                  T* __restrict__ C) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= s * s) return;
    const int i = e % s, j = e / s;
    T acc = s_zero(T());
    if (transA) {
        for (int l = 0; l < s; ++l) acc = s_cfma(A[l + (int64_t)i * s], B[l + (int64_t)j * s], acc);
    } else {
        for (int l = 0; l < s; ++l) acc = s_fma(A[i + (int64_t)l * s], B[l + (int64_t)j * s], acc);
    }
    C[e] = acc;
}

template <class T>
__global__ void hermitize_kernel(int s, T* C) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= s * s) return;
    const int i = e % s, j = e / s;
    if (i > j) return;
    const T a = C[e], b = C[j + (int64_t)i * s];
    if (i == j) {
        C[e] = s_from<T>(s_real(a), 0.0);
    } else {
        const T m = s_rscale(0.5, s_add(a, s_conj(b)));
        C[e] = m;
        C[j + (int64_t)i * s] = s_conj(m);
    }
}

rc_status small_gemm(rc_ctx* ctx, int dtype, int64_t s, const void* A, bool transA, const void* B, void* C) {
    const unsigned g = (unsigned)((s * s + 255) / 256);
    if (dtype == RC_COMPLEX128)
        small_gemm_kernel<double2><<<g, 256, 0, ctx->stream>>>((int)s, (const double2*)A, transA ? 1 : 0,
                                                              (const double2*)B, (double2*)C);
    else
        small_gemm_kernel<double><<<g, 256, 0, ctx->stream>>>((int)s, (const double*)A, transA ? 1 : 0,
                                                             (const double*)B, (double*)C);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    return RC_OK;
}

rc_status hermitize(rc_ctx* ctx, int dtype, int64_t s, void* C) {
    const unsigned g = (unsigned)((s * s + 255) / 256);
    if (dtype == RC_COMPLEX128)
        hermitize_kernel<double2><<<g, 256, 0, ctx->stream>>>((int)s, (double2*)C);
    else
        hermitize_kernel<double><<<g, 256, 0, ctx->stream>>>((int)s, (double*)C);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    return RC_OK;
}

// ---------------------------------------------------------------------------------------
// Elementwise helpers
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
__device__ __forceinline__ double u11(uint64_t h) { return (double)(h >> 11) * (2.0 / 9007199254740992.0) - 1.0; }

template <class T>
__global__ void fill_random_kernel(T* X, int64_t ld, int64_t n, int64_t c0, int64_t c1, uint64_t seed) {
    const int64_t total = n * (c1 - c0);
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e % n, c = c0 + e / n;
        const uint64_t key = seed * 0x100000001B3ull + (uint64_t)c * (uint64_t)n + (uint64_t)i;
        const uint64_t h1 = splitmix64(key), h2 = splitmix64(key ^ 0xD1B54A32D192ED03ull);
        X[i + c * ld] = s_from<T>(u11(h1), u11(h2));
    }
}

rc_status fill_random(rc_ctx* ctx, int dtype, void* X, int64_t ld, int64_t n, int64_t c0, int64_t c1, uint64_t seed) {
    if (c1 <= c0 || n <= 0) return RC_OK;
    if (dtype == RC_COMPLEX128)
        fill_random_kernel<double2><<<8 * 148, 256, 0, ctx->stream>>>((double2*)X, ld, n, c0, c1, seed);
    else
        fill_random_kernel<double><<<8 * 148, 256, 0, ctx->stream>>>((double*)X, ld, n, c0, c1, seed);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    return RC_OK;
}

rc_status copy_cols(rc_ctx* ctx, int dtype, const void* X, int64_t ldx, void* Y, int64_t ldy, int64_t n, int64_t s) {
    if (s <= 0 || n <= 0) return RC_OK;
    const size_t esz = dtype == RC_COMPLEX128 ? 16 : 8;
    RC_CU(ctx, cudaMemcpy2DAsync(Y, (size_t)ldy * esz, X, (size_t)ldx * esz, (size_t)n * esz, (size_t)s,
                                 cudaMemcpyDeviceToDevice, ctx->stream));
    return RC_OK;
}

template <class T>
__global__ void axpby_kernel(int64_t n, int64_t s, double a, const T* X, int64_t ldx, double b, T* Y, int64_t ldy) {
    const int64_t total = n * s;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e % n, c = e / n;
        Y[i + c * ldy] = s_add(s_rscale(a, X[i + c * ldx]), s_rscale(b, Y[i + c * ldy]));
    }
}

rc_status axpby(rc_ctx* ctx, int dtype, double a, const void* X, int64_t ldx, double b, void* Y, int64_t ldy,
                int64_t n, int64_t s) {
    if (s <= 0 || n <= 0) return RC_OK;
    if (dtype == RC_COMPLEX128)
        axpby_kernel<double2><<<8 * 148, 256, 0, ctx->stream>>>(n, s, a, (const double2*)X, ldx, b, (double2*)Y, ldy);
    else
        axpby_kernel<double><<<8 * 148, 256, 0, ctx->stream>>>(n, s, a, (const double*)X, ldx, b, (double*)Y, ldy);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    return RC_OK;
}

// ---------------------------------------------------------------------------------------
// CholeskyQR with escalation: pass p computes G = V^H V, T = D^-1 R^-1, V' = V T (into the
// other buffer). Two passes (CholeskyQR2) normally; when a Cholesky pass needed the shift the
// block is ill-conditioned and one more pass follows (shifted CholeskyQR3), up to 4 passes.
// The result is in V when *swapped is false, else in tmp.
// ---------------------------------------------------------------------------------------
rc_status cholqr(rc_ctx* ctx, int dtype, void* V, int64_t ld, int64_t n, int64_t s, void* tmp, bool* swapped,
                 int* passes) {
    const size_t esz = dtype == RC_COMPLEX128 ? 16 : 8;
    void* small = nullptr;
    RC_TRY(rc_slot(ctx, S_SMALL, 4 * (size_t)s * s * esz + 1024, &small));
    void* G = small;
    void* Tm = (char*)small + (size_t)s * s * esz;
    int* flags = (int*)((char*)small + 4 * (size_t)s * s * esz);
    double* hflags = nullptr;
    RC_TRY(rc_host_small(ctx, 64, &hflags));
    void* cur = V;
    void* oth = tmp;
    int64_t ldc = ld, ldo = n;
    int np = 0;
    int max_pass = 2;
    for (int p = 0; p < max_pass && p < 4; ++p) {
        RC_CU(ctx, cudaMemsetAsync(flags, 0, 4 * sizeof(int), ctx->stream));
        RC_TRY(gram(ctx, dtype, n, s, s, cur, ldc, cur, ldc, G, true));
        RC_TRY(chol_factor(ctx, dtype, s, n, G, Tm, flags, nullptr));
        XtArgs xa;
        xa.n = n; xa.k = s; xa.nc = s;
        xa.X = cur; xa.ldx = ldc;
        xa.T = Tm; xa.ldt = s;
        xa.Y = oth; xa.ldy = ldo;
        RC_TRY(xt(ctx, dtype, xa));
        ++np;
        // read the flags of this pass
        RC_CU(ctx, cudaMemcpyAsync(hflags, flags, 4 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        RC_CU(ctx, cudaStreamSynchronize(ctx->stream));
        const int* hf = (const int*)hflags;
        if (hf[1]) return rc_fail(ctx, RC_ERR_BREAKDOWN, "CholeskyQR: Gram matrix not positive definite after shift");
        if (hf[0] && max_pass < 4) max_pass = std::min(4, p + 3);
        void* t = cur;
        cur = oth;
        oth = t;
        const int64_t tl = ldc;
        ldc = ldo;
        ldo = tl;
    }
    *swapped = (cur != V);
    if (passes) *passes = np;
    return RC_OK;
}

}  // namespace rcb
