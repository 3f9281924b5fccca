// rc_gemm.cu -- FP64 tall-skinny GEMMs of the Rayleigh-Ritz step for real blocks with s <= 96,
// on the FP64 tensor pipe (mma.sync m8n8k4 .f64, which runs at the full FP64 rate on sm_100a and
// needs a quarter of the shared-memory reads of a register-tiled DFMA loop).
//
//  gram2: C_y = X^T Y_y for up to two right-hand blocks (G = V^T V and H = V^T (A V) in one
//         launch), both symmetric: only the 32x32 super-blocks on and above the diagonal are
//         formed (the reference's CPU formVtAV also forms the upper triangle,
//         RayleighChebyshevLM.h:1928-1969). One CTA per SM walks its chunk of rows in 32-row
//         K-tiles, double-buffered in shared memory by cp.async; warp (y, bi, bj) accumulates
//         the 32x32 super-block (bi, bj) of C_y in 16 mma tiles. Per-chunk partials are summed
//         by gram2_reduce_kernel in a fixed order (deterministic).
//  xt2:   Y = X T (n x k times k x nc, k, nc <= 96), persistent CTAs with T resident in shared
//         memory. Plain form: 64-row tiles of X double-buffered, warp (slab, half) forms 16 rows x
//         48 columns. Dual form (32-row tiles of X and W, 8-row warp slabs) also forms W T for the
//         columns that need it and reduces
//         ||(W T)_c - lam_c (X T)_c||^2 for c < res_count; with R32 it writes the residual block
//         R = W T - (X T) diag(lam) in row-major FP32 (the source term of an FP32-storage
//         correction filter; native real operators take R from rc_resid.cu instead).
// These replace cublasDgemm(OP_T, OP_N) and cublasDgemm(OP_N, OP_N) plus the residual kernel
// of the reference (RayleighChebyshevLMCuda.h:2139-2161, :2200-2285).
//
// mma.m8n8k4 .f64 fragments (g = lane / 4, q = lane % 4): A (8x4, row) a = A[g][q];
// B (4x8, col) b = B[q][g]; C (8x8) {c0, c1} = C[g][2q], C[g][2q+1].
#include <algorithm>
#include "rc_common.cuh"
#include "rc_internal.h"

namespace rcb {

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// 16-byte (two rows) or 8-byte (one row) asynchronous copy global -> shared; bytes beyond
// src_bytes are zero-filled (src_bytes = 0 reads nothing).
__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src, int src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::); }

// Copy rows [r0, r0 + RT) of columns [0, ncols) of a column-major block into a shared tile laid
// out column by column with `rp` doubles per column (rows past r_end read as zero).
template <int RT, bool V16>
__device__ __forceinline__ void load_cols_async(double* tile, int rp, const double* __restrict__ src, int64_t ld,
                                                int ncols, int64_t r0, int64_t r_end, int tid, int nthreads) {
    if (V16) {
        constexpr int H = RT / 2;
        for (int e = tid; e < ncols * H; e += nthreads) {
            const int c = e / H, rr = 2 * (e - c * H);
            const int64_t r = r0 + rr;
            const int64_t left = r_end - r;
            const int bytes = left >= 2 ? 16 : (left == 1 ? 8 : 0);
            const double* gp = bytes ? src + r + (int64_t)c * ld : src;
            cp_async16(tile + c * rp + rr, gp, bytes);
        }
    } else {
        for (int e = tid; e < ncols * RT; e += nthreads) {
            const int c = e / RT, rr = e - c * RT;
            const int64_t r = r0 + rr;
            const bool ok = r < r_end;
            cp_async8(tile + c * rp + rr, ok ? src + r + (int64_t)c * ld : src, ok ? 8 : 0);
        }
    }
}

// A thread's share of the row-major tile copies below: column pair lp of rows lr0, lr0 + lrs, ...
// (threads past lrs * pairs copy nothing). Set up once per kernel, so the copies of every tile need no
// division by the runtime column count. Needs pairs = (ncols + 1) / 2 <= nthreads (true for the
// blocks of at most 96 columns and the CTAs of at least 32 threads per 32 columns here).
struct RowCopyMap {
    int lp, lr0, lrs;
    __device__ __forceinline__ RowCopyMap(int ncols, int tid, int nthreads) {
        const int pairs = (ncols + 1) / 2;
        lrs = nthreads / pairs;
        lp = tid % pairs;
        lr0 = tid < lrs * pairs ? tid / pairs : 1 << 30;
    }
};

// Copy rows [r0, r0 + RT) of columns [0, ncols) of a row-major block (leading dimension ld, even,
// rows 16-byte aligned) into a shared tile laid out row by row with `rp` doubles per row, in
// 16-byte pairs (an odd last column is copied with its neighbour zero-filled; rows past r_end read
// as zero).
template <int RT>
__device__ __forceinline__ void load_rows_async(double* tile, int rp, const double* __restrict__ src, int64_t ld,
                                                int ncols, int64_t r0, int64_t r_end, const RowCopyMap& cm) {
    const int c = 2 * cm.lp;
    for (int rr = cm.lr0; rr < RT; rr += cm.lrs) {
        const int64_t r = r0 + rr;
        const int bytes = r < r_end ? (c + 1 < ncols ? 16 : 8) : 0;
        cp_async16(tile + rr * rp + c, bytes ? src + r * ld + c : src, bytes);
    }
}

// ---------------------------------------------------------------------------------------
// gram2
// ---------------------------------------------------------------------------------------
constexpr int GM_KT = 32;          // rows per K-tile
constexpr int GM_KP = GM_KT + 4;   // doubles per column in shared memory (= 4 mod 16: conflict-free fragments)
// Shared-memory operand tile of gram_mma_kernel: column-major inputs are held column by column
// (GM_KP doubles per column), row-major inputs row by row (32 SB + 4 doubles per row, also = 4 mod
// 16); element (row rr, column c) lies at c * CS + rr * RS.
template <int SB, bool RM>
struct GmTile {
    static constexpr int RP = 32 * SB + 4;
    static constexpr int SIZE = RM ? GM_KT * RP : 32 * SB * GM_KP;
    static constexpr int CS = RM ? 1 : GM_KP;
    static constexpr int RS = RM ? RP : 1;
};

template <int SB, int NY>
constexpr int gm_threads() {
    return 32 * NY * SB * (SB + 1) / 2;
}

template <int SB, int NY, bool V16, bool RM = false>
__global__ void __launch_bounds__(gm_threads<SB, NY>(), 1)
gram_mma_kernel(int64_t n, int m, const double* __restrict__ X, int64_t ldx, const double* __restrict__ Y0,
                int64_t ldy0, const double* __restrict__ Y1, int64_t ldy1, double* __restrict__ part, int64_t rows) {
    using TL = GmTile<SB, RM>;
    constexpr int NT = gm_threads<SB, NY>();
    constexpr int NP = SB * (SB + 1) / 2;
    constexpr int SC = 32 * SB;                 // padded columns
    constexpr int OPS = 1 + NY;                 // operands per stage
    constexpr int OPSZ = TL::SIZE;              // doubles per operand tile
    constexpr int STAGE = OPS * OPSZ;           // doubles per stage
    extern __shared__ __align__(16) double gms[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, q = lane & 3;
    const int y = warp / NP;
    int pidx = warp - y * NP, bi = 0;
    while (pidx >= SB - bi) {  // (bi, bj) with bi <= bj, row by row over the upper triangle
        pidx -= SB - bi;
        ++bi;
    }
    const int bj = bi + pidx;
    const int64_t r_begin = (int64_t)blockIdx.x * rows;
    const int64_t r_end = min(n, r_begin + rows);
    // zero the padding columns m..SC of every operand of both stages once (never copied into, or
    // zero-filled by the copies)
    if constexpr (RM) {
        const int per = GM_KT * (SC - m);
        for (int e = tid; e < 2 * OPS * per; e += NT) {
            const int op = e / per, f = e - op * per;
            const int rr = f / (SC - m), c = m + (f - rr * (SC - m));
            gms[op * OPSZ + rr * TL::RP + c] = 0.0;
        }
    } else {
        const int per = (SC - m) * GM_KP;
        for (int e = tid; e < 2 * OPS * per; e += NT) {
            const int st = e / per, f = e - st * per;
            gms[st * SC * GM_KP + m * GM_KP + f] = 0.0;
        }
    }
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    const int64_t ntiles = r_end > r_begin ? (r_end - r_begin + GM_KT - 1) / GM_KT : 0;
    const RowCopyMap rcm(m, tid, NT);
    auto issue = [&](int64_t t) {
        double* st = gms + (t & 1) * STAGE;
        const int64_t r0 = r_begin + t * GM_KT;
        if constexpr (RM) {
            load_rows_async<GM_KT>(st, TL::RP, X, ldx, m, r0, r_end, rcm);
            load_rows_async<GM_KT>(st + OPSZ, TL::RP, Y0, ldy0, m, r0, r_end, rcm);
            if (NY == 2) load_rows_async<GM_KT>(st + 2 * OPSZ, TL::RP, Y1, ldy1, m, r0, r_end, rcm);
        } else {
            load_cols_async<GM_KT, V16>(st, GM_KP, X, ldx, m, r0, r_end, tid, NT);
            load_cols_async<GM_KT, V16>(st + SC * GM_KP, GM_KP, Y0, ldy0, m, r0, r_end, tid, NT);
            if (NY == 2) load_cols_async<GM_KT, V16>(st + 2 * SC * GM_KP, GM_KP, Y1, ldy1, m, r0, r_end, tid, NT);
        }
    };
    // two stages, one barrier per K-tile: after the barrier every warp has finished tile t-1, so
    // the copies of tile t+1 go into its stage while tile t is multiplied
    if (ntiles > 0) issue(0);
    cp_async_commit();
    for (int64_t t = 0; t < ntiles; ++t) {
        cp_async_wait0();
        __syncthreads();
        if (t + 1 < ntiles) issue(t + 1);
        cp_async_commit();
        const double* xs = gms + (t & 1) * STAGE + (bi * 32 + g) * TL::CS + q * TL::RS;
        const double* ys = gms + (t & 1) * STAGE + (1 + y) * OPSZ + (bj * 32 + g) * TL::CS + q * TL::RS;
#pragma unroll
        for (int k0 = 0; k0 < GM_KT; k0 += 4) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = xs[i * 8 * TL::CS + k0 * TL::RS];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = ys[j * 8 * TL::CS + k0 * TL::RS];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
    }
    double* P = part + ((size_t)y * gridDim.x + blockIdx.x) * (size_t)m * m;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int row = bi * 32 + i * 8 + g, col = bj * 32 + j * 8 + 2 * q + h;
                if (row < m && col < m) P[row + (int64_t)col * m] = acc[i][j][h];
            }
}

// C_y[i,j] = sum over chunks of part[y][chunk][i,j] for i <= j; mirrored to exact symmetry.
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

template <int SB, int NY, bool V16, bool RM>
static rc_status gram_mma_launch(rc_ctx* ctx, int64_t n, int64_t m, const double* X, int64_t ldx, const double* Y0,
                                 int64_t ldy0, const double* Y1, int64_t ldy1, double* part, int64_t nchunks,
                                 int64_t rows) {
    constexpr int NT = gm_threads<SB, NY>();
    const size_t smem = (size_t)2 * (1 + NY) * GmTile<SB, RM>::SIZE * sizeof(double);
    RC_CU(ctx, allow_max_smem(ctx, gram_mma_kernel<SB, NY, V16, RM>));
    gram_mma_kernel<SB, NY, V16, RM><<<(unsigned)nchunks, NT, smem, ctx->stream>>>(n, (int)m, X, ldx, Y0, ldy0, Y1,
                                                                                   ldy1, part, rows);
    return RC_OK;
}

// C0 = X^T Y0 and (if Y1) C1 = X^T Y1, square m x m symmetric results (upper computed, mirrored).
// rm: the blocks are row-major (leading dimensions even, rows 16-byte aligned).
rc_status gram2(rc_ctx* ctx, int64_t n, int64_t m, const double* X, int64_t ldx, const double* Y0, int64_t ldy0,
                double* C0, const double* Y1, int64_t ldy1, double* C1, bool rm) {
    const int ny = Y1 ? 2 : 1;
    const int sb = (int)((m + 31) / 32);
    // one CTA per SM for the widest blocks; narrower blocks run several CTAs per SM
    const int per_sm = sb == 3 ? 1 : (sb == 2 ? 2 : 4);
    int64_t nchunks = (int64_t)ctx->sm_count * per_sm;
    int64_t rows = (n + nchunks - 1) / nchunks;
    rows = ((rows + GM_KT - 1) / GM_KT) * GM_KT;
    nchunks = (n + rows - 1) / rows;
    void* part = nullptr;
    RC_TRY(rc_slot(ctx, S_PART, (size_t)ny * nchunks * m * m * sizeof(double), &part));
    // 16-byte copies need 16-byte aligned columns (rows, for row-major blocks)
    const bool v16 = ((uintptr_t)X % 16 == 0) && ((uintptr_t)Y0 % 16 == 0) && (ldx % 2 == 0) && (ldy0 % 2 == 0) &&
                     (!Y1 || (((uintptr_t)Y1 % 16 == 0) && (ldy1 % 2 == 0)));
    if (rm && (!v16 || ldx < m || ldy0 < m || (Y1 && ldy1 < m)))
        return rc_fail(ctx, RC_ERR_INVALID, "gram2: row-major blocks need even leading dimensions >= m, 16-byte aligned");
    const double* y1 = Y1 ? Y1 : Y0;
    const int64_t l1 = Y1 ? ldy1 : ldy0;
    double* pp = (double*)part;
#define RC_GM(SBV, NYV)                                                                                           \
    (rm ? gram_mma_launch<SBV, NYV, true, true>(ctx, n, m, X, ldx, Y0, ldy0, y1, l1, pp, nchunks, rows)           \
        : v16 ? gram_mma_launch<SBV, NYV, true, false>(ctx, n, m, X, ldx, Y0, ldy0, y1, l1, pp, nchunks, rows)    \
              : gram_mma_launch<SBV, NYV, false, false>(ctx, n, m, X, ldx, Y0, ldy0, y1, l1, pp, nchunks, rows))
    rc_status st;
    if (ny == 2) st = sb == 1 ? RC_GM(1, 2) : (sb == 2 ? RC_GM(2, 2) : RC_GM(3, 2));
    else st = sb == 1 ? RC_GM(1, 1) : (sb == 2 ? RC_GM(2, 1) : RC_GM(3, 1));
#undef RC_GM
    RC_TRY(st);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    const int64_t total = (int64_t)ny * m * m;
    const unsigned gr = (unsigned)std::min<int64_t>((total + 255) / 256, 4 * 148);
    gram2_reduce_kernel<<<gr, 256, 0, ctx->stream>>>((int)m, nchunks, ny, (const double*)part, C0, C1);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    return RC_OK;
}

// ---------------------------------------------------------------------------------------
// gram_c: the complex Hermitian Gram C = X^H Y (m x m, m <= 192) on the same FP64 tensor pipe.
// A complex column-major block with leading dimension ld is, read as doubles, a real column-major
// block of 2n rows (real and imaginary part of each entry on consecutive rows) with leading
// dimension 2 ld. With Xr, Yr those real blocks,
//   Re C = Xr^T Yr,   Im C = Xr^T (J Yr),   (J Yr)[2r] = Im y_r, (J Yr)[2r+1] = -Re y_r,
// so both parts are real Gram products over the same shared-memory tiles: the B fragments of the
// imaginary part are read from row k^1 of the tile and negated on odd rows k (K-tiles start on even
// rows), which costs no copy. Warp tasks are the upper 32x32 super-blocks of the real part and of
// the imaginary part (2 x SB(SB+1)/2 tasks); the tasks are split over `groups` CTAs per chunk of
// rows so that one CTA holds at most 16 warps, and each CTA copies the whole K-tile of X (and of Y,
// unless Y is X). Per-chunk partials of both parts are summed by gram_c_reduce_kernel in a fixed
// order (deterministic), which also mirrors C to exact Hermitian symmetry. This replaces the
// reference's complex cublasZgemm(OP_C, OP_N) of the Rayleigh-Ritz step
// (RayleighChebyshevLMCuda.h:2139-2161).
// ---------------------------------------------------------------------------------------
constexpr int GC_MAX_WARPS = 16;

template <int SB, bool SAME>
__global__ void __launch_bounds__(32 * GC_MAX_WARPS, 1)
gram_mma_cplx_kernel(int64_t n2, int m, const double* __restrict__ X, int64_t ldx2, const double* __restrict__ Y,
                     int64_t ldy2, double* __restrict__ part, int64_t rows, int tpg) {
    constexpr int NP = SB * (SB + 1) / 2;       // upper super-blocks of one part
    constexpr int SC = 32 * SB;                 // padded columns
    constexpr int OPS = SAME ? 1 : 2;           // operand tiles per stage
    constexpr int OPSZ = SC * GM_KP;            // doubles per operand tile (column by column)
    constexpr int STAGE = OPS * OPSZ;
    extern __shared__ __align__(16) double gcs[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int NT = blockDim.x;
    const int g = lane >> 2, q = lane & 3;
    const int task = blockIdx.y * tpg + warp;
    const bool active = task < 2 * NP;
    const int im = active && task >= NP ? 1 : 0;  // 0: real part, 1: imaginary part
    int pidx = active ? task - im * NP : 0, bi = 0;
    while (pidx >= SB - bi) {
        pidx -= SB - bi;
        ++bi;
    }
    const int bj = bi + pidx;
    const int64_t r_begin = (int64_t)blockIdx.x * rows;
    const int64_t r_end = min(n2, r_begin + rows);
    // zero the padding columns m..SC of every operand of both stages once
    {
        const int per = (SC - m) * GM_KP;
        for (int e = tid; e < 2 * OPS * per; e += NT) {
            const int op = e / per, f = e - op * per;
            gcs[op * OPSZ + m * GM_KP + f] = 0.0;
        }
    }
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    const int64_t ntiles = r_end > r_begin ? (r_end - r_begin + GM_KT - 1) / GM_KT : 0;
    auto issue = [&](int64_t t) {
        double* st = gcs + (t & 1) * STAGE;
        const int64_t r0 = r_begin + t * GM_KT;
        load_cols_async<GM_KT, true>(st, GM_KP, X, ldx2, m, r0, r_end, tid, NT);
        if (!SAME) load_cols_async<GM_KT, true>(st + OPSZ, GM_KP, Y, ldy2, m, r0, r_end, tid, NT);
    };
    // B fragment row of this lane (k0 + qb) and its sign: J for the imaginary part
    const int qb = im ? (q ^ 1) : q;
    const double sgn = (im && (q & 1)) ? -1.0 : 1.0;
    if (ntiles > 0) issue(0);
    cp_async_commit();
    for (int64_t t = 0; t < ntiles; ++t) {
        cp_async_wait0();
        __syncthreads();
        if (t + 1 < ntiles) issue(t + 1);
        cp_async_commit();
        if (active) {
            const double* st = gcs + (t & 1) * STAGE;
            const double* xs = st + (bi * 32 + g) * GM_KP + q;
            const double* ys = st + (SAME ? 0 : OPSZ) + (bj * 32 + g) * GM_KP + qb;
#pragma unroll
            for (int k0 = 0; k0 < GM_KT; k0 += 4) {
                double a[4], b[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) a[i] = xs[i * 8 * GM_KP + k0];
#pragma unroll
                for (int j = 0; j < 4; ++j) b[j] = sgn * ys[j * 8 * GM_KP + k0];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
            }
        }
    }
    if (!active) return;
    double* P = part + ((size_t)im * gridDim.x + blockIdx.x) * (size_t)m * m;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int row = bi * 32 + i * 8 + g, col = bj * 32 + j * 8 + 2 * q + h;
                if (row < m && col < m) P[row + (int64_t)col * m] = acc[i][j][h];
            }
}

// C[i,j] = (sum of the real-part partials, sum of the imaginary-part partials) for i <= j, the
// diagonal real, mirrored to C[j,i] = conj(C[i,j]).
__global__ void gram_c_reduce_kernel(int m, int64_t nchunks, const double* __restrict__ part, double2* __restrict__ C) {
    const int64_t total = (int64_t)m * m;
    for (int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; f < total; f += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(f % m), j = (int)(f / m);
        if (i > j) continue;
        double re = 0.0, im = 0.0;
        const double* pr = part + f;
        const double* pi = part + (size_t)nchunks * total + f;
        for (int64_t c = 0; c < nchunks; ++c) {
            re += pr[(size_t)c * total];
            im += pi[(size_t)c * total];
        }
        if (i == j) im = 0.0;
        C[f] = make_double2(re, im);
        C[j + (int64_t)i * m] = make_double2(re, -im);
    }
}

bool gram_c_supported(int dtype, int64_t m) { return dtype == RC_COMPLEX128 && m >= 1 && m <= 192; }

template <int SB, bool SAME>
static rc_status gram_c_launch(rc_ctx* ctx, int64_t n2, int m, const double* X, int64_t ldx2, const double* Y,
                               int64_t ldy2, double* part, int64_t nchunks, int groups, int tpg, int64_t rows,
                               size_t smem) {
    RC_CU(ctx, allow_max_smem(ctx, gram_mma_cplx_kernel<SB, SAME>));
    gram_mma_cplx_kernel<SB, SAME><<<dim3((unsigned)nchunks, (unsigned)groups), 32 * tpg, smem, ctx->stream>>>(
        n2, m, X, ldx2, Y, ldy2, part, rows, tpg);
    return RC_OK;
}

rc_status gram_c(rc_ctx* ctx, int64_t n, int64_t m, const double2* X, int64_t ldx, const double2* Y, int64_t ldy,
                 double2* C) {
    if (!gram_c_supported(RC_COMPLEX128, m)) return rc_fail(ctx, RC_ERR_INVALID, "gram_c: m out of range");
    const int sb = (int)((m + 31) / 32);
    const int np = sb * (sb + 1) / 2;
    const int tasks = 2 * np;
    const int groups = (tasks + GC_MAX_WARPS - 1) / GC_MAX_WARPS;
    const int tpg = (tasks + groups - 1) / groups;
    const bool same = X == Y && ldx == ldy;
    const int ops = same ? 1 : 2;
    const size_t smem = (size_t)2 * ops * 32 * sb * GM_KP * sizeof(double);
    // resident CTAs per SM: by shared memory and by registers (at most 128 per thread)
    int per_sm = std::max<int>(1, (int)(((size_t)ctx->smem_optin) / (smem + 1024)));
    per_sm = std::max(1, std::min(per_sm, 65536 / (32 * tpg * 128)));
    int64_t nchunks = std::max<int64_t>(1, (int64_t)ctx->sm_count * per_sm / groups);
    const int64_t n2 = 2 * n;
    int64_t rows = (n2 + nchunks - 1) / nchunks;
    rows = ((rows + GM_KT - 1) / GM_KT) * GM_KT;
    nchunks = (n2 + rows - 1) / rows;
    void* part = nullptr;
    RC_TRY(rc_slot(ctx, S_PART, (size_t)2 * nchunks * m * m * sizeof(double), &part));
    const double* xr = reinterpret_cast<const double*>(X);
    const double* yr = reinterpret_cast<const double*>(Y);
    double* pp = (double*)part;
#define RC_GC(SBV)                                                                                               \
    (same ? gram_c_launch<SBV, true>(ctx, n2, (int)m, xr, 2 * ldx, xr, 2 * ldx, pp, nchunks, groups, tpg, rows, smem) \
          : gram_c_launch<SBV, false>(ctx, n2, (int)m, xr, 2 * ldx, yr, 2 * ldy, pp, nchunks, groups, tpg, rows, smem))
    rc_status st;
    switch (sb) {
        case 1: st = RC_GC(1); break;
        case 2: st = RC_GC(2); break;
        case 3: st = RC_GC(3); break;
        case 4: st = RC_GC(4); break;
        case 5: st = RC_GC(5); break;
        default: st = RC_GC(6); break;
    }
#undef RC_GC
    RC_TRY(st);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    const int64_t total = m * m;
    const unsigned gr = (unsigned)std::min<int64_t>((total + 255) / 256, 4 * 148);
    gram_c_reduce_kernel<<<gr, 256, 0, ctx->stream>>>((int)m, nchunks, (const double*)part, C);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    return RC_OK;
}

// ---------------------------------------------------------------------------------------
// xt2
// ---------------------------------------------------------------------------------------
constexpr int XM_RT = 32;         // rows per tile
constexpr int XM_RP = XM_RT + 4;  // doubles per column of a shared X/W tile (= 4 mod 16)
constexpr int XM_CT = 6;          // 8-column mma tiles per warp (48 columns)

// Doubles per column of the shared T (>= k rounded up to 4, = 4 mod 16).
__host__ __device__ inline int xm_kpt(int k) {
    int k4 = (k + 3) / 4 * 4;
    while (k4 % 16 != 4) k4 += 4;
    return k4;
}

// Warps: 4 row slabs (8 rows each) x NH column halves (48 columns each).
template <int NH, bool DUAL, bool V16>
__global__ void __launch_bounds__(128 * NH, 1)
xt_mma_kernel(int64_t n, int k, int nc, const double* __restrict__ X, int64_t ldx, const double* __restrict__ Tm,
              int64_t ldt, double* __restrict__ Y, int64_t ldy, const double* __restrict__ W, int64_t ldw,
              const double* __restrict__ lam, int dual_cols, int res_count, double* __restrict__ rpart,
              float* __restrict__ R32, int64_t ldr) {
    constexpr int NT = 128 * NH;
    constexpr int OPS = DUAL ? 2 : 1;
    const int kpt = xm_kpt(k);
    const int k4 = (k + 3) / 4 * 4;
    extern __shared__ __align__(16) double xms[];
    double* Ts = xms;                                  // [NH*48][kpt]
    double* tiles = Ts + (size_t)NH * 48 * kpt;        // [2][OPS][k4][XM_RP]
    const int stage = OPS * k4 * XM_RP;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, q = lane & 3;
    const int slab = warp & 3, half = warp >> 2;
    const int cbase = half * 48;
    for (int e = tid; e < NH * 48 * kpt; e += NT) {
        const int c = e / kpt, kk = e - c * kpt;
        Ts[e] = (c < nc && kk < k) ? Tm[kk + (int64_t)c * ldt] : 0.0;
    }
    // zero the padding columns k..k4 of every operand of both stages once
    {
        const int per = (k4 - k) * XM_RP;
        for (int e = tid; e < 2 * OPS * per; e += NT) {
            const int st = e / per, f = e - st * per;
            tiles[st * k4 * XM_RP + k * XM_RP + f] = 0.0;
        }
    }
    // mma tiles of this warp whose columns need W T (warp-uniform)
    const int dtiles = DUAL ? max(0, min(XM_CT, (dual_cols - cbase + 7) / 8)) : 0;
    double lamc[XM_CT][2], rs[XM_CT][2];
#pragma unroll
    for (int j = 0; j < XM_CT; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int c = cbase + j * 8 + 2 * q + h;
            lamc[j][h] = (DUAL && c < dual_cols) ? lam[c] : 0.0;
            rs[j][h] = 0.0;
        }
    const int64_t ntiles = (n + XM_RT - 1) / XM_RT;
    auto issue = [&](int64_t t, int b) {
        double* st = tiles + b * stage;
        const int64_t r0 = t * XM_RT;
        load_cols_async<XM_RT, V16>(st, XM_RP, X, ldx, k, r0, n, tid, NT);
        if (DUAL) load_cols_async<XM_RT, V16>(st + k4 * XM_RP, XM_RP, W, ldw, k, r0, n, tid, NT);
    };
    // two stages, one barrier per tile (as in gram_mma_kernel)
    int buf = 0;
    int64_t t = blockIdx.x;
    if (t < ntiles) issue(t, 0);
    cp_async_commit();
    for (; t < ntiles; t += gridDim.x) {
        cp_async_wait0();
        __syncthreads();
        const int64_t tn = t + gridDim.x;
        if (tn < ntiles) issue(tn, buf ^ 1);
        cp_async_commit();
        const double* xs = tiles + buf * stage + slab * 8 + g + q * XM_RP;
        const double* ws = xs + k4 * XM_RP;
        const double* ts = Ts + (cbase + g) * kpt + q;
        double acc[XM_CT][2], acc2[XM_CT][2];
#pragma unroll
        for (int j = 0; j < XM_CT; ++j) acc[j][0] = acc[j][1] = acc2[j][0] = acc2[j][1] = 0.0;
#pragma unroll 2
        for (int k0 = 0; k0 < k4; k0 += 4) {
            const double a = xs[k0 * XM_RP];
            double b[XM_CT];
#pragma unroll
            for (int j = 0; j < XM_CT; ++j) b[j] = ts[j * 8 * kpt + k0];
#pragma unroll
            for (int j = 0; j < XM_CT; ++j) dmma(acc[j][0], acc[j][1], a, b[j]);
            if (DUAL && dtiles > 0) {
                const double w = ws[k0 * XM_RP];
#pragma unroll
                for (int j = 0; j < XM_CT; ++j)
                    if (j < dtiles) dmma(acc2[j][0], acc2[j][1], w, b[j]);
            }
        }
        const int64_t r = t * XM_RT + slab * 8 + g;
        if (r < n) {
#pragma unroll
            for (int j = 0; j < XM_CT; ++j) {
                const int c = cbase + j * 8 + 2 * q;
                if (c < nc) Y[r + (int64_t)c * ldy] = acc[j][0];
                if (c + 1 < nc) Y[r + (int64_t)(c + 1) * ldy] = acc[j][1];
                if (DUAL && j < dtiles) {
                    const double d0 = acc2[j][0] - lamc[j][0] * acc[j][0];
                    const double d1 = acc2[j][1] - lamc[j][1] * acc[j][1];
                    if (c < res_count) rs[j][0] = fma(d0, d0, rs[j][0]);
                    if (c + 1 < res_count) rs[j][1] = fma(d1, d1, rs[j][1]);
                    if (R32) {
                        if (c + 1 < nc) {
                            *reinterpret_cast<float2*>(R32 + r * ldr + c) = make_float2((float)d0, (float)d1);
                        } else if (c < nc) {
                            R32[r * ldr + c] = (float)d0;
                        }
                    }
                }
            }
        }
        buf ^= 1;
    }
    if (DUAL && res_count > 0) {
        __syncthreads();  // the last tile's reads are done before its stage is reused below
        // per column: sum over g (lanes with the same q), then over the four row slabs in order
        double* red = tiles;  // [4][NH*48]; the tiles are no longer read
#pragma unroll
        for (int j = 0; j < XM_CT; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                double v = rs[j][h];
                v += __shfl_xor_sync(0xffffffffu, v, 4);
                v += __shfl_xor_sync(0xffffffffu, v, 8);
                v += __shfl_xor_sync(0xffffffffu, v, 16);
                if (g == 0) red[slab * NH * 48 + cbase + j * 8 + 2 * q + h] = v;
            }
        __syncthreads();
        for (int c = tid; c < res_count; c += NT) {
            double v = 0.0;
#pragma unroll
            for (int sl = 0; sl < 4; ++sl) v += red[sl * NH * 48 + c];
            rpart[(size_t)blockIdx.x * res_count + c] = v;
        }
    }
}

// Plain product Y = X T (no dual): 64-row tiles, warp (slab, half) forms 16 rows x 48 columns
// (two mma row tiles share each B fragment: 8 shared-memory reads per 12 mma).
constexpr int XP_RT = 64;
constexpr int XP_RP = XP_RT + 4;  // = 4 mod 16

// X row-major (RM): the 64-row tiles are held row by row with kpt doubles per row (= 4 mod 16),
// element (row r, column kk) at r * RS + kk * CS in both layouts.
template <int NH, bool V16, bool RM = false>
__global__ void __launch_bounds__(128 * NH, 1)
xt_mma_plain_kernel(int64_t n, int k, int nc, const double* __restrict__ X, int64_t ldx,
                    const double* __restrict__ Tm, int64_t ldt, double* __restrict__ Y, int64_t ldy,
                    double* __restrict__ Yrm, int64_t ldyr) {
    constexpr int NT = 128 * NH;
    const int kpt = xm_kpt(k);
    const int k4 = (k + 3) / 4 * 4;
    extern __shared__ __align__(16) double xps[];
    double* Ts = xps;                            // [NH*48][kpt]
    double* tiles = Ts + (size_t)NH * 48 * kpt;  // [2][k4][XP_RP], or [2][XP_RT][kpt] when RM
    const int stage = RM ? XP_RT * kpt : k4 * XP_RP;
    const int CS = RM ? 1 : XP_RP, RS = RM ? kpt : 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, q = lane & 3;
    const int slab = warp & 3, half = warp >> 2;
    const int cbase = half * 48;
    for (int e = tid; e < NH * 48 * kpt; e += NT) {
        const int c = e / kpt, kk = e - c * kpt;
        Ts[e] = (c < nc && kk < k) ? Tm[kk + (int64_t)c * ldt] : 0.0;
    }
    if constexpr (RM) {  // padding columns k..k4 of every row of both stages
        const int w = k4 - k;
        for (int e = tid; e < 2 * XP_RT * w; e += NT) {
            const int row = e / w;  // stage-major: row in [0, 2 * XP_RT)
            tiles[row * kpt + k + (e - row * w)] = 0.0;
        }
    } else {
        const int per = (k4 - k) * XP_RP;
        for (int e = tid; e < 2 * per; e += NT) {
            const int st = e / per, f = e - st * per;
            tiles[st * stage + k * XP_RP + f] = 0.0;
        }
    }
    const RowCopyMap rcm(k, tid, NT);
    auto load = [&](double* dst, int64_t r0) {
        if constexpr (RM) load_rows_async<XP_RT>(dst, kpt, X, ldx, k, r0, n, rcm);
        else load_cols_async<XP_RT, V16>(dst, XP_RP, X, ldx, k, r0, n, tid, NT);
    };
    const int64_t ntiles = (n + XP_RT - 1) / XP_RT;
    int buf = 0;
    int64_t t = blockIdx.x;
    if (t < ntiles) load(tiles, t * XP_RT);
    cp_async_commit();
    for (; t < ntiles; t += gridDim.x) {
        cp_async_wait0();
        __syncthreads();
        const int64_t tn = t + gridDim.x;
        if (tn < ntiles) load(tiles + (buf ^ 1) * stage, tn * XP_RT);
        cp_async_commit();
        const double* xs = tiles + buf * stage + (slab * 16 + g) * RS + q * CS;
        const double* ts = Ts + (cbase + g) * kpt + q;
        double acc[2][XM_CT][2];
#pragma unroll
        for (int m = 0; m < 2; ++m)
#pragma unroll
            for (int j = 0; j < XM_CT; ++j) acc[m][j][0] = acc[m][j][1] = 0.0;
#pragma unroll 2
        for (int k0 = 0; k0 < k4; k0 += 4) {
            const double a0 = xs[k0 * CS], a1 = xs[k0 * CS + 8 * RS];
            double b[XM_CT];
#pragma unroll
            for (int j = 0; j < XM_CT; ++j) b[j] = ts[j * 8 * kpt + k0];
#pragma unroll
            for (int j = 0; j < XM_CT; ++j) {
                dmma(acc[0][j][0], acc[0][j][1], a0, b[j]);
                dmma(acc[1][j][0], acc[1][j][1], a1, b[j]);
            }
        }
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            const int64_t r = t * XP_RT + slab * 16 + m * 8 + g;
            if (r < n) {
#pragma unroll
                for (int j = 0; j < XM_CT; ++j) {
                    const int c = cbase + j * 8 + 2 * q;
                    if (c < nc) Y[r + (int64_t)c * ldy] = acc[m][j][0];
                    if (c + 1 < nc) Y[r + (int64_t)(c + 1) * ldy] = acc[m][j][1];
                    if (Yrm) {  // row-major copy (even leading dimension: 16-byte pairs)
                        if (c + 1 < nc)
                            *reinterpret_cast<double2*>(Yrm + r * ldyr + c) = make_double2(acc[m][j][0], acc[m][j][1]);
                        else if (c < nc)
                            Yrm[r * ldyr + c] = acc[m][j][0];
                    }
                }
            }
        }
        buf ^= 1;
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

template <int NH, bool DUAL, bool V16>
static rc_status xt_mma_launch(rc_ctx* ctx, unsigned grid, int64_t n, int64_t k, int64_t nc, const double* X,
                               int64_t ldx, const double* T, int64_t ldt, double* Y, int64_t ldy, const double* W,
                               int64_t ldw, const double* lam, int64_t dual_cols, int64_t res_count, double* rpart,
                               float* R32, int64_t ldr) {
    const int k4 = (int)((k + 3) / 4 * 4);
    const size_t smem =
        ((size_t)NH * 48 * xm_kpt((int)k) + (size_t)2 * (DUAL ? 2 : 1) * k4 * XM_RP) * sizeof(double);
    RC_CU(ctx, allow_max_smem(ctx, xt_mma_kernel<NH, DUAL, V16>));
    xt_mma_kernel<NH, DUAL, V16><<<grid, 128 * NH, smem, ctx->stream>>>(
        n, (int)k, (int)nc, X, ldx, T, ldt, Y, ldy, W, ldw, lam, (int)dual_cols, (int)res_count, rpart, R32, ldr);
    return RC_OK;
}

// Y = X T; with W: residual norms ||(W T)_c - lam_c Y_c|| for c < res_count into res (device),
// and with R32 the residual block (all nc columns) in row-major FP32 with leading dimension ldr.
rc_status xt2(rc_ctx* ctx, int64_t n, int64_t k, int64_t nc, const double* X, int64_t ldx, const double* T,
              int64_t ldt, double* Y, int64_t ldy, const double* W, int64_t ldw, const double* lam, int64_t res_count,
              double* res, float* R32, int64_t ldr, double* Yrm, int64_t ldyr) {
    const bool dual = W != nullptr && lam != nullptr && (res_count > 0 || R32 != nullptr);
    if (!dual) {
        res_count = 0;
        R32 = nullptr;
    }
    const int64_t dual_cols = dual ? (R32 ? nc : std::min(res_count, nc)) : 0;
    if (R32 && (ldr % 2 != 0 || (uintptr_t)R32 % 8 != 0))
        return rc_fail(ctx, RC_ERR_INVALID, "xt2: the residual block needs an even leading dimension");
    const int nh = nc <= 48 ? 1 : 2;
    const int64_t ntiles = (n + XM_RT - 1) / XM_RT;
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ntiles, ctx->sm_count));
    double* rpart = nullptr;
    if (res_count > 0) {
        void* p = nullptr;
        RC_TRY(rc_slot(ctx, S_RPART, (size_t)grid * res_count * sizeof(double), &p));
        rpart = (double*)p;
    }
    const bool v16 =
        ((uintptr_t)X % 16 == 0) && (ldx % 2 == 0) && (!dual || (((uintptr_t)W % 16 == 0) && ldw % 2 == 0));
    if (Yrm && (dual || ldyr % 2 != 0 || (uintptr_t)Yrm % 16 != 0))
        return rc_fail(ctx, RC_ERR_INVALID, "xt2: the row-major copy needs the plain product and an even leading dimension");
    if (!dual) {
        const int64_t pt = (n + XP_RT - 1) / XP_RT;
        const unsigned pg = (unsigned)std::max<int64_t>(1, std::min<int64_t>(pt, ctx->sm_count));
        const size_t psm = ((size_t)nh * 48 * xm_kpt((int)k) + (size_t)2 * ((k + 3) / 4 * 4) * XP_RP) * sizeof(double);
#define RC_XP(NHV, VV)                                                                                            \
    do {                                                                                                          \
        RC_CU(ctx, allow_max_smem(ctx, xt_mma_plain_kernel<NHV, VV>));                                            \
        xt_mma_plain_kernel<NHV, VV><<<pg, 128 * NHV, psm, ctx->stream>>>(n, (int)k, (int)nc, X, ldx, T, ldt, Y, ldy, \
                                                                          Yrm, ldyr);                            \
    } while (0)
        if (nh == 1) {
            if (v16) RC_XP(1, true); else RC_XP(1, false);
        } else {
            if (v16) RC_XP(2, true); else RC_XP(2, false);
        }
#undef RC_XP
        ctx->launches++;
        RC_CU(ctx, cudaGetLastError());
        return RC_OK;
    }
#define RC_XM(NHV, DV)                                                                                            \
    (v16 ? xt_mma_launch<NHV, DV, true>(ctx, grid, n, k, nc, X, ldx, T, ldt, Y, ldy, W, ldw, lam, dual_cols,      \
                                        res_count, rpart, R32, ldr)                                               \
         : xt_mma_launch<NHV, DV, false>(ctx, grid, n, k, nc, X, ldx, T, ldt, Y, ldy, W, ldw, lam, dual_cols,     \
                                         res_count, rpart, R32, ldr))
    rc_status st;
    st = nh == 1 ? RC_XM(1, true) : RC_XM(2, true);
#undef RC_XM
    RC_TRY(st);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    if (res_count > 0) {
        resid2_reduce_kernel<<<(unsigned)res_count, 256, 0, ctx->stream>>>(grid, (int)res_count, rpart, res);
        ctx->launches++;
        RC_CU(ctx, cudaGetLastError());
    }
    return RC_OK;
}

// Y = X T for a row-major X (leading dimension ldx, even, >= k, rows 16-byte aligned): Y column-major
// (ldy) and, when Yrm is given, a row-major copy (ldyr, even).
rc_status xt2_rm(rc_ctx* ctx, int64_t n, int64_t k, int64_t nc, const double* X, int64_t ldx, const double* T,
                 int64_t ldt, double* Y, int64_t ldy, double* Yrm, int64_t ldyr) {
    if (!xt2_supported(RC_REAL64, k, nc)) return rc_fail(ctx, RC_ERR_UNSUPPORTED, "xt2_rm: k, nc <= 96 only");
    if ((uintptr_t)X % 16 != 0 || ldx % 2 != 0 || ldx < k)
        return rc_fail(ctx, RC_ERR_INVALID, "xt2_rm: row-major X needs an even leading dimension >= k, 16-byte aligned");
    if (Yrm && (ldyr % 2 != 0 || (uintptr_t)Yrm % 16 != 0))
        return rc_fail(ctx, RC_ERR_INVALID, "xt2_rm: the row-major copy needs an even leading dimension");
    const int nh = nc <= 48 ? 1 : 2;
    const int64_t pt = (n + XP_RT - 1) / XP_RT;
    const unsigned pg = (unsigned)std::max<int64_t>(1, std::min<int64_t>(pt, ctx->sm_count));
    const int kpt = xm_kpt((int)k);
    const size_t psm = ((size_t)nh * 48 * kpt + (size_t)2 * XP_RT * kpt) * sizeof(double);
    if (nh == 1) {
        RC_CU(ctx, allow_max_smem(ctx, xt_mma_plain_kernel<1, true, true>));
        xt_mma_plain_kernel<1, true, true><<<pg, 128, psm, ctx->stream>>>(n, (int)k, (int)nc, X, ldx, T, ldt, Y,
                                                                          ldy, Yrm, ldyr);
    } else {
        RC_CU(ctx, allow_max_smem(ctx, xt_mma_plain_kernel<2, true, true>));
        xt_mma_plain_kernel<2, true, true><<<pg, 256, psm, ctx->stream>>>(n, (int)k, (int)nc, X, ldx, T, ldt, Y,
                                                                          ldy, Yrm, ldyr);
    }
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    return RC_OK;
}

}  // namespace rcb
