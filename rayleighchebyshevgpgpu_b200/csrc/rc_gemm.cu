// rc_gemm.cu -- FP64 tall-skinny GEMMs of the Rayleigh-Ritz step for real blocks with s <= 96.
//
//  gram2: C_y = X^T Y_y for up to two right-hand blocks (G = V^T V and H = V^T (A V) in one
//         launch). Grid (row chunk, y): each CTA accumulates the whole s x s product of its row
//         chunk, 256 threads with 6x6 (in general R x R, 16R >= s) register tiles; the next
//         K-tile of X and Y is staged in registers while the current one is consumed from
//         shared memory (padded rows: conflict-free stores and broadcast/contiguous reads).
//         Per-chunk partials are summed by gram_reduce in a fixed order (deterministic).
//  xt2:   Y = X T (n x k times k x nc, k, nc <= 96), persistent CTAs holding T in shared
//         memory; the dual form also forms W T on the fly for the first res_count columns and
//         reduces only ||(W T)_c - lam_c (X T)_c||^2 per column (W T itself is not stored).
// These replace cublasDgemm(OP_T, OP_N) and cublasDgemm(OP_N, OP_N) plus the residual kernel
// of the reference (RayleighChebyshevLMCuda.h:2139-2161, :2200-2285).
#include <algorithm>
#include "rc_common.cuh"
#include "rc_internal.h"

namespace rcb {

constexpr int G2_THREADS = 256;
constexpr int G2_KT = 16;

template <int R>
__global__ void __launch_bounds__(G2_THREADS, (R >= 6 ? 1 : 2))
gram2_kernel(int64_t n, int m, int nc, const double* __restrict__ X, int64_t ldx, const double* __restrict__ Y0,
             int64_t ldy0, const double* __restrict__ Y1, int64_t ldy1, double* __restrict__ part, int64_t rows) {
    constexpr int TB = 16 * R;
    constexpr int S = TB + 1;  // padded smem row (conflict-free stores of consecutive rows)
    constexpr int NL = (G2_KT * TB) / G2_THREADS;  // elements per thread per operand per K-tile
    extern __shared__ __align__(16) double g2s[];
    double* Xs = g2s;                    // [2][KT][S]
    double* Ys = g2s + 2 * G2_KT * S;    // [2][KT][S]
    const double* Y = blockIdx.y == 0 ? Y0 : Y1;
    const int64_t ldy = blockIdx.y == 0 ? ldy0 : ldy1;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int64_t r_begin = (int64_t)blockIdx.x * rows;
    const int64_t r_end = min(n, r_begin + rows);
    double acc[R][R];
#pragma unroll
    for (int i = 0; i < R; ++i)
#pragma unroll
        for (int j = 0; j < R; ++j) acc[i][j] = 0.0;
    double rx[NL], ry[NL];
    auto fetch = [&](int64_t r0) {
#pragma unroll
        for (int l = 0; l < NL; ++l) {
            const int e = tid + l * G2_THREADS;
            const int kk = e % G2_KT, c = e / G2_KT;
            const int64_t r = r0 + kk;
            const bool ok = r < r_end;
            rx[l] = (ok && c < m) ? __ldg(X + r + (int64_t)c * ldx) : 0.0;
            ry[l] = (ok && c < nc) ? __ldg(Y + r + (int64_t)c * ldy) : 0.0;
        }
    };
    auto stash = [&](int buf) {
        double* xs = Xs + buf * G2_KT * S;
        double* ys = Ys + buf * G2_KT * S;
#pragma unroll
        for (int l = 0; l < NL; ++l) {
            const int e = tid + l * G2_THREADS;
            const int kk = e % G2_KT, c = e / G2_KT;
            xs[kk * S + c] = rx[l];
            ys[kk * S + c] = ry[l];
        }
    };
    int buf = 0;
    if (r_begin < r_end) {
        fetch(r_begin);
        stash(0);
    }
    __syncthreads();
    for (int64_t r0 = r_begin; r0 < r_end; r0 += G2_KT) {
        const bool more = r0 + G2_KT < r_end;
        if (more) fetch(r0 + G2_KT);
        const double* xs = Xs + buf * G2_KT * S;
        const double* ys = Ys + buf * G2_KT * S;
#pragma unroll
        for (int kk = 0; kk < G2_KT; ++kk) {
            double a[R], b[R];
#pragma unroll
            for (int i = 0; i < R; ++i) a[i] = xs[kk * S + tx + 16 * i];
#pragma unroll
            for (int j = 0; j < R; ++j) b[j] = ys[kk * S + ty + 16 * j];
#pragma unroll
            for (int i = 0; i < R; ++i)
#pragma unroll
                for (int j = 0; j < R; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        if (more) stash(buf ^ 1);
        __syncthreads();
        buf ^= 1;
    }
    double* P = part + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * (size_t)m * nc;
#pragma unroll
    for (int i = 0; i < R; ++i)
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const int mi = tx + 16 * i, nj = ty + 16 * j;
            if (mi < m && nj < nc) P[mi + (int64_t)nj * m] = acc[i][j];
        }
}

// C_y[i,j] = sum over chunks of part[y][chunk][i,j]; mirrored to exact symmetry (upper kept).
__global__ void gram2_reduce_kernel(int m, int64_t nchunks, int ny, const double* __restrict__ part, double* C0,
                                    double* C1) {
    const int64_t total = (int64_t)m * m;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < ny * total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int y = (int)(e / total);
        const int64_t f = e - y * total;
        const int i = (int)(f % m), j = (int)(f / m);
        if (i > j) continue;
        double sum = 0.0;
        const double* p = part + (size_t)y * nchunks * total + f;
        for (int64_t c = 0; c < nchunks; ++c) sum += p[(size_t)c * total];
        double* C = y == 0 ? C0 : C1;
        C[f] = sum;
        C[j + (int64_t)i * m] = sum;
    }
}

bool gram2_supported(int dtype, int64_t m) { return dtype == RC_REAL64 && m >= 1 && m <= 96; }

// C0 = X^T Y0 and (if Y1) C1 = X^T Y1, square m x m symmetric results (upper computed, mirrored).
rc_status gram2(rc_ctx* ctx, int64_t n, int64_t m, const double* X, int64_t ldx, const double* Y0, int64_t ldy0,
                double* C0, const double* Y1, int64_t ldy1, double* C1) {
    const int ny = Y1 ? 2 : 1;
    const int R = m <= 32 ? 2 : (m <= 48 ? 3 : (m <= 64 ? 4 : 6));
    int64_t nchunks = (2 * ctx->sm_count + ny - 1) / ny;
    int64_t rows = (n + nchunks - 1) / nchunks;
    rows = ((rows + G2_KT - 1) / G2_KT) * G2_KT;
    nchunks = (n + rows - 1) / rows;
    void* part = nullptr;
    RC_TRY(rc_slot(ctx, S_PART, (size_t)ny * nchunks * m * m * sizeof(double), &part));
    dim3 grid((unsigned)nchunks, ny);
    const size_t smem = (size_t)4 * G2_KT * (16 * R + 1) * sizeof(double);
#define RC_G2(RR)                                                                                             \
    do {                                                                                                      \
        if (smem > 48 * 1024)                                                                                 \
            RC_CU(ctx, cudaFuncSetAttribute(gram2_kernel<RR>, cudaFuncAttributeMaxDynamicSharedMemorySize,     \
                                            (int)smem));                                                      \
        gram2_kernel<RR><<<grid, G2_THREADS, smem, ctx->stream>>>(n, (int)m, (int)m, X, ldx, Y0, ldy0,       \
                                                                  Y1 ? Y1 : Y0, Y1 ? ldy1 : ldy0,            \
                                                                  (double*)part, rows);                       \
    } while (0)
    if (R == 2) RC_G2(2);
    else if (R == 3) RC_G2(3);
    else if (R == 4) RC_G2(4);
    else RC_G2(6);
#undef RC_G2
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    const int64_t total = (int64_t)ny * m * m;
    const unsigned g = (unsigned)std::min<int64_t>((total + 255) / 256, 4 * 148);
    gram2_reduce_kernel<<<g, 256, 0, ctx->stream>>>((int)m, nchunks, ny, (const double*)part, C0, C1);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    return RC_OK;
}

// ---------------------------------------------------------------------------------------
// xt2: Y = X T with T (k x nc) resident in shared memory; persistent CTAs over 64-row tiles.
// thread (tx, ty): rows tx + 16 i (i < 4), columns ty + 16 j (j < R).
// ---------------------------------------------------------------------------------------
constexpr int X2_THREADS = 256;
constexpr int X2_RM = 4;
constexpr int X2_BR = 16 * X2_RM;

template <int R, bool DUAL>
__global__ void __launch_bounds__(X2_THREADS, 1)
xt2_kernel(int64_t n, int k, int nc, const double* __restrict__ X, int64_t ldx, const double* __restrict__ Tm,
           int64_t ldt, double* __restrict__ Y, int64_t ldy, const double* __restrict__ W, int64_t ldw,
           const double* __restrict__ lam, int res_count, double* __restrict__ rpart) {
    constexpr int TB = 16 * R;
    constexpr int S = TB + 1;
    extern __shared__ __align__(16) double x2s[];
    double* Ts = x2s;                       // [k][S]
    double* Xs = Ts + (size_t)k * S;        // [k][BR]
    double* Ws = Xs + (size_t)k * X2_BR;    // [k][BR] (DUAL)
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    for (int e = tid; e < k * TB; e += X2_THREADS) {
        const int kk = e % k, c = e / k;
        Ts[kk * S + c] = c < nc ? Tm[kk + (int64_t)c * ldt] : 0.0;
    }
    double lamc[R];
    double rs[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
        const int c = ty + 16 * j;
        lamc[j] = (DUAL && c < res_count) ? lam[c] : 0.0;
        rs[j] = 0.0;
    }
    const int64_t ntiles = (n + X2_BR - 1) / X2_BR;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int64_t r0 = t * X2_BR;
        __syncthreads();
        for (int e = tid; e < k * X2_BR; e += X2_THREADS) {
            const int rr = e % X2_BR, kk = e / X2_BR;
            const int64_t r = r0 + rr;
            Xs[kk * X2_BR + rr] = r < n ? __ldg(X + r + (int64_t)kk * ldx) : 0.0;
            if (DUAL) Ws[kk * X2_BR + rr] = r < n ? __ldg(W + r + (int64_t)kk * ldw) : 0.0;
        }
        __syncthreads();
        double acc[X2_RM][R], acc2[DUAL ? X2_RM : 1][DUAL ? R : 1];
#pragma unroll
        for (int i = 0; i < X2_RM; ++i)
#pragma unroll
            for (int j = 0; j < R; ++j) {
                acc[i][j] = 0.0;
                if (DUAL) acc2[i % (DUAL ? X2_RM : 1)][j % (DUAL ? R : 1)] = 0.0;
            }
#pragma unroll 4
        for (int kk = 0; kk < k; ++kk) {
            double a[X2_RM], w[X2_RM], b[R];
#pragma unroll
            for (int i = 0; i < X2_RM; ++i) {
                a[i] = Xs[kk * X2_BR + tx + 16 * i];
                if (DUAL) w[i] = Ws[kk * X2_BR + tx + 16 * i];
            }
#pragma unroll
            for (int j = 0; j < R; ++j) b[j] = Ts[kk * S + ty + 16 * j];
#pragma unroll
            for (int i = 0; i < X2_RM; ++i)
#pragma unroll
                for (int j = 0; j < R; ++j) {
                    acc[i][j] = fma(a[i], b[j], acc[i][j]);
                    if (DUAL) acc2[i % (DUAL ? X2_RM : 1)][j % (DUAL ? R : 1)] =
                        fma(w[i], b[j], acc2[i % (DUAL ? X2_RM : 1)][j % (DUAL ? R : 1)]);
                }
        }
#pragma unroll
        for (int i = 0; i < X2_RM; ++i) {
            const int64_t r = r0 + tx + 16 * i;
            if (r >= n) continue;
#pragma unroll
            for (int j = 0; j < R; ++j) {
                const int c = ty + 16 * j;
                if (c < nc) {
                    Y[r + (int64_t)c * ldy] = acc[i][j];
                    if (DUAL && c < res_count) {
                        const double d = acc2[i % (DUAL ? X2_RM : 1)][j % (DUAL ? R : 1)] - lamc[j] * acc[i][j];
                        rs[j] = fma(d, d, rs[j]);
                    }
                }
            }
        }
    }
    if (DUAL) {
#pragma unroll
        for (int j = 0; j < R; ++j) {
            double v = rs[j];
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            const int c = ty + 16 * j;
            if (tx == 0 && c < res_count) rpart[(size_t)blockIdx.x * res_count + c] = v;
        }
    }
}

__global__ void resid2_reduce_kernel(int64_t nblocks, int res_count, const double* __restrict__ rpart,
                                     double* __restrict__ res) {
    const int c = blockIdx.x;
    __shared__ double sc[32];
    double v = 0.0;
    for (int64_t b = threadIdx.x; b < nblocks; b += blockDim.x) v += rpart[(size_t)b * res_count + c];
    v = block_sum(v, sc);
    if (threadIdx.x == 0) res[c] = sqrt(v);
}

bool xt2_supported(int dtype, int64_t k, int64_t nc) {
    return dtype == RC_REAL64 && k >= 1 && k <= 96 && nc >= 1 && nc <= 96;
}

// Y = X T; with W: residual norms ||(W T)_c - lam_c Y_c|| for c < res_count into res (device).
rc_status xt2(rc_ctx* ctx, int64_t n, int64_t k, int64_t nc, const double* X, int64_t ldx, const double* T,
              int64_t ldt, double* Y, int64_t ldy, const double* W, int64_t ldw, const double* lam, int64_t res_count,
              double* res) {
    const int R = nc <= 32 ? 2 : (nc <= 48 ? 3 : (nc <= 64 ? 4 : 6));
    const bool dual = W != nullptr && res_count > 0;
    const size_t smem = ((size_t)k * (16 * R + 1) + (size_t)k * X2_BR * (dual ? 2 : 1)) * sizeof(double);
    const int64_t ntiles = (n + X2_BR - 1) / X2_BR;
    const unsigned grid = (unsigned)std::min<int64_t>(ntiles, ctx->sm_count);
    double* rpart = nullptr;
    if (dual) {
        void* p = nullptr;
        RC_TRY(rc_slot(ctx, S_RPART, (size_t)grid * res_count * sizeof(double), &p));
        rpart = (double*)p;
    }
#define RC_X2(RR, DD)                                                                                          \
    do {                                                                                                       \
        RC_CU(ctx, cudaFuncSetAttribute(xt2_kernel<RR, DD>, cudaFuncAttributeMaxDynamicSharedMemorySize,        \
                                        (int)smem));                                                           \
        xt2_kernel<RR, DD><<<grid, X2_THREADS, smem, ctx->stream>>>(n, (int)k, (int)nc, X, ldx, T, ldt, Y, ldy, \
                                                                    W, ldw, lam, (int)res_count, rpart);       \
    } while (0)
    if (dual) {
        if (R == 2) RC_X2(2, true);
        else if (R == 3) RC_X2(3, true);
        else if (R == 4) RC_X2(4, true);
        else RC_X2(6, true);
    } else {
        if (R == 2) RC_X2(2, false);
        else if (R == 3) RC_X2(3, false);
        else if (R == 4) RC_X2(4, false);
        else RC_X2(6, false);
    }
#undef RC_X2
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    if (dual) {
        resid2_reduce_kernel<<<(unsigned)res_count, 256, 0, ctx->stream>>>(grid, (int)res_count, rpart, res);
        ctx->launches++;
        RC_CU(ctx, cudaGetLastError());
    }
    return RC_OK;
}

}  // namespace rcb
