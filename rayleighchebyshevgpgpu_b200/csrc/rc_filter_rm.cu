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
#include <algorithm>
#include <atomic>
#include <cstring>
#include <type_traits>
#include "rc_common.cuh"
#include "rc_internal.h"
#include "rc_rowops.cuh"
#include "rc_rmstep.cuh"
#include "rc_staged.cuh"

namespace rcb {

template <class Pol, class TS, class TC, int W, class IX>
__global__ void __launch_bounds__(kRmThreads, rm_min_blocks<TS>())
rm_step_kernel(Pol op, int64_t n, int nseg, int64_t ld, int groups, const TS* __restrict__ x, const TS* z, TS* y,
               TC alpha, TC beta, TC gamma, int64_t pf_z, int64_t pf_x) {
    rm_step_rows<Pol, TS, TC, W, IX>(op, n, nseg, ld, groups, (int64_t)blockIdx.x, x, z, y, alpha, beta, gamma, pf_z,
                                     pf_x);
}

// Degree step of the correction filter: y = alpha A x + beta x + gamma z + sig[c] src, with x, z,
// y and src stored as TM (FP32, or bfloat16 with FP32 arithmetic).
template <class Pol, class TS, class TC, int W, class IX, class TM>
__global__ void __launch_bounds__(kRmThreads, rm_src_min_blocks<TM, IX, W>())
rm_step_src_kernel(Pol op, int64_t n, int nseg, int64_t ld, int groups, const TM* __restrict__ x, const TM* z, TM* y,
                   TC alpha, TC beta, TC gamma, int64_t pf_z, int64_t pf_x, const TM* __restrict__ src,
                   const float* __restrict__ sig) {
    rm_step_rows<Pol, TS, TC, W, IX, true, TM>(op, n, nseg, ld, groups, (int64_t)blockIdx.x, x, z, y, alpha, beta,
                                               gamma, pf_z, pf_x, src, sig);
}

// Two consecutive degree steps of the correction filter in one pass:
//   e_k     = a A e_{k-1} + b e_{k-1} + gA e_{k-2} + sig_k R        (phase A, into Y0; Y0 = Z in place)
//   e_{k+1} = a A e_k     + b e_k     -    e_{k-1} + sig_{k+1} R    (phase B, into Y1; Y1 = X1 in place, or a
//                                                                   separate block when X1 is R)
// Work items are blocks of `groups` row groups (the rows rm_step_rows gives CTA index b), taken in
// order from a ticket counter by persistent CTAs. Ticket t runs phase A of block t, then phase B of
// block t - lag. Phase B of block u reads e_k of the rows within `band` of it and overwrites e_{k-1} of
// its own rows, which phase A of those same neighbour rows reads: it waits until phase A is complete
// for every block within band_blocks of u, counted per group of `grp` blocks (grp_cnt). Those blocks
// hold earlier tickets, whose phase A never waits, so the kernel cannot deadlock; the waits are also
// bounded (on a timeout *err is set and every CTA stops). Phase A reads e_{k-2} (the block it
// overwrites with e_k) through L2 only, so no SM caches a line of it in L1 before it is final, and
// phase B gathers e_k through the read-only path; the waits extend one block past the band, past any
// line a gather brings in. e_k is read back from L2 shortly after it is written: the two steps move
// five block passes through DRAM instead of eight, with the same arithmetic per row as two launches
// of rm_step_src_kernel (bit-identical results).
constexpr long long kPairSpins = 1ll << 20;
// Resident CTAs per SM of rm_corr2_kernel (the two steps' code spills at the 40 registers of 6).
#ifndef RC_PAIR_MIN_BLOCKS
#define RC_PAIR_MIN_BLOCKS 5
#endif

template <class Pol, class TS, class TC, int W, class IX, class TM>
__global__ void __launch_bounds__(kRmThreads, RC_PAIR_MIN_BLOCKS)
rm_corr2_kernel(Pol op, int64_t n, int nseg, int64_t ld, int groups, const TM* X1, const TM* Z, TM* Y0, TM* Y1,
                TC alpha, TC beta, TC gammaA, const TM* __restrict__ R, const float* __restrict__ sigA,
                const float* __restrict__ sigB, int64_t pf_z, int64_t pf_x, int64_t nblk, int64_t lag,
                int64_t band_blocks, int grp, unsigned long long* ticket, unsigned* grp_cnt, int* err) {
    __shared__ long long s_t;
    const TC m1 = s_from<TC>(-1.0, 0.0);
    for (;;) {
        if (threadIdx.x == 0) s_t = (long long)atomicAdd(ticket, 1ull);
        __syncthreads();
        const int64_t t = s_t;
        __syncthreads();
        if (t >= nblk + lag) break;
        if (t < nblk) {
            rm_step_rows<Pol, TS, TC, W, IX, true, TM, true>(op, n, nseg, ld, groups, t, X1, Z, Y0, alpha, beta,
                                                             gammaA, pf_z, pf_x, R, sigA);
            __threadfence();  // this thread's rows of e_k, before the block is counted complete
            __syncthreads();
            if (threadIdx.x == 0) atomicAdd(&grp_cnt[t / grp], 1u);
        }
        if (t >= lag) {
            const int64_t u = t - lag;
            // the groups of blocks u - band_blocks .. u + band_blocks, polled in parallel (thread j polls
            // groups g0 + j, g0 + j + blockDim.x, ...)
            const int64_t b_lo = u - band_blocks > 0 ? u - band_blocks : 0;
            const int64_t b_hi = u + band_blocks < nblk - 1 ? u + band_blocks : nblk - 1;
            const int64_t g0 = b_lo / grp, g1 = b_hi / grp;
            long long spins = 0;
            for (;;) {
                int mine = 1;
                for (int64_t g = g0 + threadIdx.x; g <= g1; g += blockDim.x) {
                    const unsigned need = (unsigned)(nblk - g * grp < grp ? nblk - g * grp : grp);
                    mine &= *(volatile const unsigned*)(grp_cnt + g) >= need;
                }
                if (__syncthreads_and(mine)) break;
                // thread 0 decides whether to give up, the same answer for every thread
                if (__syncthreads_or(threadIdx.x == 0 && (++spins > kPairSpins || *(volatile const int*)err != 0))) {
                    if (threadIdx.x == 0) atomicExch(err, 1);
                    return;
                }
                __nanosleep(64);
            }
            __threadfence();
            rm_step_rows<Pol, TS, TC, W, IX, true, TM>(op, n, nseg, ld, groups, u, Y0, X1, Y1, alpha, beta, m1, pf_z,
                                                       pf_x, R, sigB);
        }
    }
}

// The 27-point steps with the box sum reused along x (rm_step_rows27).
// RC_RM27_MIN_BLOCKS resident CTAs per SM (default 4, 64 registers): the three cross-section sums
// need more than the 40 registers of the per-row steps.
#ifndef RC_RM27_MIN_BLOCKS
#define RC_RM27_MIN_BLOCKS 4
#endif
template <class TD, class TS, class TC, int W, class IX, bool SRC, class TM>
__global__ void __launch_bounds__(kRmThreads, RC_RM27_MIN_BLOCKS)
rm_step27_kernel(StencilRows<TD, TC, 27> op, int64_t n, int nseg, int64_t ld, const TM* __restrict__ x, const TM* z,
                 TM* y, TC alpha, TC beta, TC gamma, int64_t pf_z, int64_t pf_x, const TM* __restrict__ src,
                 const float* __restrict__ sig) {
    rm_step_rows27<TD, TS, TC, W, IX, SRC, TM>(op, n, nseg, ld, kRun27, (int64_t)blockIdx.x, x, z, y, alpha, beta,
                                               gamma, pf_z, pf_x, src, sig);
}
// The same with the lanes of a warp on consecutive rows (rm_step_rows27w), for rows of at most
// kMaxSeg27w slices (at least three rows per warp step).
template <class TD, class TS, class TC, class IX, bool SRC, class TM>
__global__ void __launch_bounds__(kRmThreads, RC_RM27_MIN_BLOCKS)
rm_step27w_kernel(StencilRows<TD, TC, 27> op, int64_t n, int nseg, int64_t ld, const TM* __restrict__ x, const TM* z,
                  TM* y, TC alpha, TC beta, TC gamma, int64_t pf_z, int64_t pf_x, const TM* __restrict__ src,
                  const float* __restrict__ sig) {
    rm_step_rows27w<TD, TS, TC, IX, SRC, TM>(op, n, nseg, ld, x, z, y, alpha, beta, gamma, pf_z, pf_x, src, sig);
}

// ---------------------------------------------------------------------------------------
// The staged step (rc_staged.cuh): its plan and launch
// ---------------------------------------------------------------------------------------
// The distinct column offsets of an operator's rows, when they are few, and its longest row.
struct StageOffsets {
    int n = 0;
    int64_t off[rc_op::kMaxOffsets] = {};
    int64_t max_row_nnz = 0;
};

static bool stage_offsets(const rc_op* op, StageOffsets* so) {
    so->n = 0;
    if (op->kind == 0) {
        if (op->n_offsets < 1) return false;
        so->n = op->n_offsets;
        for (int q = 0; q < op->n_offsets; ++q) so->off[q] = op->offsets[q];
        so->max_row_nnz = op->max_row_nnz;
        return true;
    }
    if (op->kind == 1 && (op->skind == 5 || op->skind == 7)) {
        const int64_t nx = op->nx, sz = op->nx * op->ny;
        int k = 0;
        if (op->skind == 7) so->off[k++] = -sz;
        so->off[k++] = -nx;
        so->off[k++] = -1;
        so->off[k++] = 0;
        so->off[k++] = 1;
        so->off[k++] = nx;
        if (op->skind == 7) so->off[k++] = sz;
        std::sort(so->off, so->off + k);
        so->n = (int)(std::unique(so->off, so->off + k) - so->off);
        so->max_row_nnz = op->skind;
        return true;
    }
    return false;
}

// Group the offsets into windows (offsets at most 4 rows apart share one), then take the largest
// chunk of rows whose stages fit half the SM's shared memory (two CTAs per SM), else the whole:
// three stages with at least 16 rows, else two with at least 8 (or the context's rows and stages,
// when it sets them).
static bool staged_plan(const rc_ctx* ctx, const StageOffsets& so, int64_t n, int64_t ld, int tm_bytes, bool has_z,
                        bool has_src, bool csr, int ta_bytes, StagedPlan* out) {
    int nw = 0;
    int64_t glo[kStagedMaxWin], ghi[kStagedMaxWin];
    for (int q = 0; q < so.n; ++q) {
        if (nw > 0 && so.off[q] - ghi[nw - 1] <= 4) {
            ghi[nw - 1] = so.off[q];
            continue;
        }
        if (nw == kStagedMaxWin) return false;
        glo[nw] = ghi[nw] = so.off[q];
        ++nw;
    }
    const int64_t rb = ld * tm_bytes;
    if (nw == 0 || rb % 16 != 0 || rb > 16384) return false;
    auto up = [](int64_t b) { return (b + 127) / 128 * 128; };
    // two CTAs per SM share the SM's shared memory (the per-block opt-in limit plus the 1 KB the
    // system reserves per block), with 1 KB reserved for each; blocks too wide for that take a
    // whole SM
    const int64_t budget2 = ((int64_t)ctx->smem_optin + 1024) / 2 - 1536;
    const int64_t budget1 = (int64_t)ctx->smem_optin - 4096;
    auto layout = [&](int R, StagedPlan& Q) {
        int64_t off = 0;
        Q.nwin = nw;
        for (int w = 0; w < nw; ++w) {
            Q.lo[w] = glo[w];
            Q.span[w] = (int)(ghi[w] - glo[w]);
            Q.win_off[w] = (int)off;
            off += up((R + Q.span[w]) * rb);
        }
        Q.z_off = Q.src_off = Q.rp_off = Q.ci_off = Q.va_off = -1;
        if (has_z) {
            Q.z_off = (int)off;
            off += up(R * rb);
        }
        if (has_src) {
            Q.src_off = (int)off;
            off += up(R * rb);
        }
        if (csr) {
            Q.rp_off = (int)off;
            off += up((int64_t)(R + 8) * 4);
            Q.csr_cap = (int)(R * so.max_row_nnz + 8);
            Q.ci_off = (int)off;
            off += up((int64_t)Q.csr_cap * 4);
            Q.va_off = (int)off;
            off += up((int64_t)Q.csr_cap * ta_bytes);
        }
        Q.R = R;
        Q.stage_bytes = (int)off;
        return off;
    };
    for (int per_sm = 2; per_sm >= 1; --per_sm) {
        const int64_t budget = per_sm == 2 ? budget2 : budget1;
        for (int nst = 4; nst >= 2; --nst) {
            if (ctx->staged_stages ? nst != ctx->staged_stages : nst == 4) continue;
            const int rmin = ctx->staged_rows ? ctx->staged_rows : (nst == 3 ? 16 : 8);
            const int rmax = ctx->staged_rows ? ctx->staged_rows : 256;
            for (int R = rmax; R >= rmin; R -= 4) {
                StagedPlan Q;
                if (nst * layout(R, Q) <= budget) {
                    Q.nstages = nst;
                    Q.nchunks = (n + R - 1) / R;
                    Q.ctas_per_sm = per_sm;
                    *out = Q;
                    return true;
                }
            }
        }
    }
    return false;
}

template <class P, class = void>
struct CsrValue {
    using type = float;
};
template <class P>
struct CsrValue<P, std::void_t<typename P::value_t>> {
    using type = typename P::value_t;
};

// Launch the staged step when the operator and the blocks allow it; false leaves the step to the
// per-row gather kernels.
template <class Pol, class TS, class TC, int W, bool SRC, class TM>
static bool try_staged_real(rc_ctx* ctx, const Pol& pol, const StageOffsets* so, int64_t n, int nseg, int64_t ld,
                            const TM* x, const TM* z, TM* y, TC a, TC b, TC g, const TM* src, const float* sig) {
    if (!so || !ctx->staged || so->n == 0 || nseg > kStagedThreads) return false;
    auto al16 = [](const void* p) { return ((uintptr_t)p & 15) == 0; };
    if (!al16(x) || (z && !al16(z)) || !al16(y) || (SRC && !al16(src))) return false;
    constexpr bool kCsr = Pol::kIsCsr;
    using TA = typename CsrValue<Pol>::type;
    StagedPlan P;
    if (!staged_plan(ctx, *so, n, ld, (int)sizeof(TM), z != nullptr, SRC, kCsr, (int)sizeof(TA), &P)) return false;
    StagedArgs<TM, TC> A;
    A.n = n;
    A.nseg = nseg;
    A.ld = ld;
    A.row_bytes = (int)(ld * (int64_t)sizeof(TM));
    A.x = x;
    A.z = z;
    A.y = y;
    A.src = src;
    A.sig = sig;
    A.alpha = a;
    A.beta = b;
    A.gamma = g;
    if constexpr (kCsr) {
        A.rowptr = pol.rowptr;
        A.colind = pol.colind;
        A.vals = pol.vals;
        if (!al16(pol.rowptr) || !al16(pol.colind) || !al16(pol.vals)) return false;
    }
    auto kern = rm_staged_kernel<Pol, kCsr, TS, TC, W, SRC, TM, TA>;
    // the dynamic shared-memory limit, once per device (the same value from every caller)
    static std::atomic<unsigned long long> limit_set{0};
    const unsigned long long bit = 1ull << (ctx->device & 63);
    if (!(limit_set.load() & bit)) {
        if (allow_max_smem(ctx, kern) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        limit_set.fetch_or(bit);
    }
    const unsigned grid = (unsigned)std::min<int64_t>(P.nchunks, (int64_t)P.ctas_per_sm * ctx->sm_count);
    kern<<<grid, kStagedThreads, (size_t)P.nstages * P.stage_bytes, ctx->stream>>>(P, A, pol);
    ctx->launches++;
    ctx->staged_launches++;
    return true;
}

template <class Pol, class TS, class TC, int W, bool SRC, class TM>
static bool try_staged(rc_ctx* ctx, const Pol& pol, const StageOffsets* so, int64_t n, int nseg, int64_t ld,
                       const TM* x, const TM* z, TM* y, TC a, TC b, TC g, const TM* src, const float* sig) {
    if constexpr (SRC && IsComplex<TC>::value) {
        return false;  // the staged kernel has no complex correction step
    } else {
        return try_staged_real<Pol, TS, TC, W, SRC, TM>(ctx, pol, so, n, nseg, ld, x, z, y, a, b, g, src, sig);
    }
}

template <class Pol, class TS, class TC, int W, class IX, bool SRC, class TM = TS>
static void launch_step(rc_ctx* ctx, const Pol& pol, int64_t n, int nseg, int64_t ld, int groups, const TM* x,
                        const TM* z, TM* y, TC a, TC b, TC g, int64_t pf_z, int64_t pf_x, const TM* src,
                        const float* sig, const StageOffsets* so = nullptr) {
    const int rows_per_iter = kRmThreads / nseg;
    if constexpr (IsStencil27<Pol>::value) {
        using TD = typename IsStencil27<Pol>::diag_t;
        if constexpr (W == 1) {
            if (ctx->rows27w && nseg <= kMaxSeg27w && 32 / nseg >= 3) {
                const int64_t rows_per_cta = (int64_t)(kRmThreads / 32) * (32 / nseg) * kSteps27w;
                const unsigned grid = (unsigned)((n + rows_per_cta - 1) / rows_per_cta);
                rm_step27w_kernel<TD, TS, TC, IX, SRC, TM><<<grid, kRmThreads, 0, ctx->stream>>>(
                    pol, n, nseg, ld, x, z, y, a, b, g, pf_z, pf_x, src, sig);
                return;
            }
        }
        const int64_t rows_per_cta = (int64_t)kRun27 * rows_per_iter;
        const unsigned grid = (unsigned)((n + rows_per_cta - 1) / rows_per_cta);
        rm_step27_kernel<TD, TS, TC, W, IX, SRC, TM><<<grid, kRmThreads, 0, ctx->stream>>>(pol, n, nseg, ld, x, z, y, a,
                                                                                           b, g, pf_z, pf_x, src, sig);
    } else {
        if (try_staged<Pol, TS, TC, W, SRC, TM>(ctx, pol, so, n, nseg, ld, x, z, y, a, b, g, src, sig)) return;
        const int64_t rows_per_cta = (int64_t)groups * rows_per_iter;
        const unsigned grid = (unsigned)((n + rows_per_cta - 1) / rows_per_cta);
        if constexpr (SRC)
            rm_step_src_kernel<Pol, TS, TC, W, IX, TM><<<grid, kRmThreads, 0, ctx->stream>>>(pol, n, nseg, ld, groups,
                                                                                             x, z, y, a, b, g, pf_z,
                                                                                             pf_x, src, sig);
        else
            rm_step_kernel<Pol, TS, TC, W, IX><<<grid, kRmThreads, 0, ctx->stream>>>(pol, n, nseg, ld, groups, x, z, y,
                                                                                     a, b, g, pf_z, pf_x);
    }
    ctx->launches++;
}

// One launch of rm_corr2_kernel: persistent CTAs (the resident count of rm_corr2_kernel), work items
// of `groups` row groups, a lag of the CTA count plus the band (in blocks) plus a group. scratch: the
// S_PAIR slot of pair_scratch_bytes(): ticket (8 bytes), the error word (at 8, zeroed by the caller
// once per filter application), the group counters (from 64); the ticket and counters are zeroed here.
inline size_t pair_scratch_bytes(int64_t n, int64_t rb) {
    const int64_t ngrp = ((n + rb - 1) / rb + 15) / 16;
    return 64 + (size_t)ngrp * sizeof(unsigned);
}

template <class Pol, class TS, class TC, int W, class IX, class TM>
static rc_status launch_pair(rc_ctx* ctx, const Pol& pol, int64_t n, int nseg, int64_t ld, int groups,
                             const TM* x1, const TM* z, TM* y0, TM* y1, TC a, TC b, TC ga, const TM* R,
                             const float* sigA, const float* sigB, int64_t pf_z, int64_t pf_x, int64_t band,
                             void* scratch) {
    const int rows_per_iter = kRmThreads / nseg;
    const int64_t rb = (int64_t)groups * rows_per_iter;
    const int64_t nblk = (n + rb - 1) / rb;
    constexpr int kGrp = 16;
    static std::atomic<int> per_sm{0};
    if (per_sm.load() == 0) {
        int v = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, rm_corr2_kernel<Pol, TS, TC, W, IX, TM>, kRmThreads,
                                                          0) != cudaSuccess ||
            v < 1) {
            cudaGetLastError();
            v = 1;
        }
        per_sm.store(v);
    }
    const int64_t grid = std::min<int64_t>(nblk, (int64_t)per_sm.load() * ctx->sm_count);
    const int64_t band_blocks = (band + rb - 1) / rb + 1;
    const int64_t lag = grid + band_blocks + kGrp + 1;
    unsigned long long* ticket = (unsigned long long*)scratch;
    int* err = (int*)((char*)scratch + 8);
    unsigned* cnt = (unsigned*)((char*)scratch + 64);
    RC_CU(ctx, cudaMemsetAsync(ticket, 0, 8, ctx->stream));
    RC_CU(ctx, cudaMemsetAsync(cnt, 0, pair_scratch_bytes(n, rb) - 64, ctx->stream));
    rm_corr2_kernel<Pol, TS, TC, W, IX, TM><<<(unsigned)grid, kRmThreads, 0, ctx->stream>>>(
        pol, n, nseg, ld, groups, x1, z, y0, y1, a, b, ga, R, sigA, sigB, pf_z, pf_x, nblk, lag, band_blocks, kGrp,
        ticket, cnt, err);
    ctx->launches++;
    ctx->pair_launches++;
    RC_CU(ctx, cudaGetLastError());
    return RC_OK;
}

// Scalar recurrence of the correction filter, one thread per column c:
//   c_0 = 1, c_1 = a lam_c + b, c_k = (a lam_c + b) c_{k-1} - c_{k-2};
//   sig[k*ld + c] = c_{k-1} for 2 <= k <= m (the source coefficient of step k),
//   coef[c] = c_m / (m+1) (the weight of v_c in the result). Columns s..ld get zeros.
__global__ void corr_coef_kernel(int64_t s, int64_t ld, int64_t m, double a, double b, const double* __restrict__ lam,
                                 float* __restrict__ sig, double* __restrict__ coef) {
    for (int64_t c = threadIdx.x; c < ld; c += blockDim.x) {
        const double t = c < s ? a * lam[c] + b : 0.0;
        double cm2 = 1.0, cm1 = t;  // c_0, c_1
        for (int64_t k = 2; k <= m; ++k) {
            sig[k * ld + c] = c < s ? (float)cm1 : 0.0f;
            const double ck = t * cm1 - cm2;
            cm2 = cm1;
            cm1 = ck;
        }
        if (c < s) coef[c] = (m >= 1 ? cm1 : 1.0) / (double)(m + 1);
    }
}

// fail (optional): the two-step kernel's error word; when set, V is filled with NaN so the failure
// reaches the caller (the solver's finite-residual check).
template <class TM, class TV>
__global__ void __launch_bounds__(256)
corr_to_cm_kernel(int64_t n, int64_t s, const TM* __restrict__ E, int64_t ld, TV* __restrict__ Vc, int64_t ldv,
                  const double* __restrict__ coef, double beta, const int* fail) {
    __shared__ CorrTile<TM> tile[32][33];
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    corr_to_cm_tile<TM, TV>(n, s, E, ld, Vc, ldv, coef, fail && *fail ? nan : beta, (int64_t)blockIdx.x * 32,
                            (int64_t)blockIdx.y * 32, tile);
}


// The same combination into a row-major FP64 block: Vf[i*ldf + c] = coef[c] * Yrm[i*ldy + c] +
// beta * E[i*lde + c] for c < s (zero in the padding columns s..ldf), with Yrm the row-major copy of
// V (the values corr_to_cm_kernel forms, with the same arithmetic). Real blocks; one 16-byte pair of
// columns per thread, grid-stride, coalesced on every block.
template <class TM>
__global__ void __launch_bounds__(256)
corr_to_rm_kernel(int64_t n, int64_t s, const double* __restrict__ Yrm, int64_t ldy, const TM* __restrict__ E,
                  int64_t lde, double* __restrict__ Vf, int64_t ldf, const double* __restrict__ coef, double beta,
                  const int* fail) {
    if (fail && *fail) beta = __longlong_as_double(0x7ff8000000000000ll);  // NaN out (see corr_to_cm_kernel)
    const int64_t pairs = ldf / 2;
    const int64_t total = n * pairs;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / pairs, c = 2 * (e - i * pairs);
        double2 out = make_double2(0.0, 0.0);
        if (c < s) {
            const double2 y = *reinterpret_cast<const double2*>(Yrm + i * ldy + c);
            const float e0 = elem_f(E[i * lde + c]);
            out.x = fma(coef[c], y.x, beta * (double)e0);
            if (c + 1 < s) out.y = fma(coef[c + 1], y.y, beta * (double)elem_f(E[i * lde + c + 1]));
        }
        *reinterpret_cast<double2*>(Vf + i * ldf + c) = out;
    }
}

template <class TV, class TS>
__global__ void __launch_bounds__(256)
to_rm_kernel(int64_t n, int64_t s, const TV* __restrict__ Vc, int64_t ldv, TS* __restrict__ Rr, int64_t ld) {
    __shared__ TS tile[32][33];
    // rows on x (no 65535 cap)
    to_rm_tile<TV, TS>(n, s, Vc, ldv, Rr, ld, (int64_t)blockIdx.x * 32, (int64_t)blockIdx.y * 32, tile);
}

template <class TS, class TV>
__global__ void __launch_bounds__(256)
to_cm_kernel(int64_t n, int64_t s, const TS* __restrict__ Rr, int64_t ld, TV* __restrict__ Vc, int64_t ldv,
             double scale) {
    __shared__ TS tile[32][33];
    to_cm_tile<TS, TV>(n, s, Rr, ld, Vc, ldv, scale, (int64_t)blockIdx.x * 32, (int64_t)blockIdx.y * 32, tile);
}

// ---------------------------------------------------------------------------------------
// Driver
// ---------------------------------------------------------------------------------------
//   A <- X (row-major copy of x0); x_k (k = 1..m) into B, A, B, ... (x_k over x_{k-2});
//   X <- x_m / (m+1) (column-major).
template <class Pol, class TS, class TC, int W, class IX>
static rc_status run_rm_filter(rc_ctx* ctx, const Pol& pol, int64_t n, void* V, int64_t ldv, int64_t s,
                               int64_t degree, double a, double b, void* bufA, void* bufB, int64_t ld, int64_t band,
                               const StageOffsets* so) {
    const int64_t pf_z = ctx->pf_rows;
    const int64_t pf_x = pf_z > 0 ? pf_z + band : 0;
    using TY = typename std::conditional<IsComplex<TC>::value, double2, double>::type;
    constexpr int VEC = Pack16<TS>::V;
    const TC ta = s_from<TC>(a, 0.0), tb = s_from<TC>(b, 0.0), tm1 = s_from<TC>(-1.0, 0.0);
    if (ld % (VEC * W) != 0) return rc_fail(ctx, RC_ERR_INVALID, "row-major filter: leading dimension not padded");
    const int nseg = (int)(ld / (VEC * W));
    if (nseg > kRmThreads) return rc_fail(ctx, RC_ERR_UNSUPPORTED, "row-major filter: block too wide");
    // consecutive row groups per CTA (measured on 128^3 7-point operators, 96 columns):
    // CSR 4 (FP32) / 2 (FP64), stencil 8 (FP32) / 4 (FP64)
    constexpr bool kCsr = Pol::kIsCsr;
    constexpr bool kF32 = sizeof(real_t<TS>) == 4;
    const int groups = ctx->rm_groups > 0 ? ctx->rm_groups : (kCsr ? (kF32 ? 4 : 2) : (kF32 ? 8 : 4));
    if ((s + 31) / 32 > 65535) return rc_fail(ctx, RC_ERR_UNSUPPORTED, "row-major filter: too many columns");
    const dim3 tgrid((unsigned)((n + 31) / 32), (unsigned)((s + 31) / 32)), tblk(32, 8);
    TS* A = (TS*)bufA;
    TS* B = (TS*)bufB;
    to_rm_kernel<TY, TS><<<tgrid, tblk, 0, ctx->stream>>>(n, s, (const TY*)V, ldv, A, ld);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    step_mark(ctx);
    for (int64_t k = 1; k <= degree; ++k) {
        const TS* xk1 = (k - 1) % 2 ? B : A;  // x_{k-1}
        TS* y = k % 2 ? B : A;                // x_k overwrites x_{k-2}
        // k = 1 has no x_{k-2} (gamma = 0): z is not read
        const TS* z = k >= 2 ? y : nullptr;
        launch_step<Pol, TS, TC, W, IX, false>(ctx, pol, n, nseg, ld, groups, xk1, z, y, ta, tb,
                                               k >= 2 ? tm1 : s_zero(TC()), pf_z, pf_x, (const TS*)nullptr, nullptr,
                                               so);
    }
    RC_CU(ctx, cudaGetLastError());
    step_mark(ctx);
    const TS* xm = degree % 2 ? B : A;
    to_cm_kernel<TS, TY><<<tgrid, tblk, 0, ctx->stream>>>(n, s, xm, ld, (TY*)V, ldv, 1.0 / (double)(degree + 1));
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    return RC_OK;
}

// The correction filter (blocks stored as TM: rc_corr_t for real operators, rc_corr2_t for complex
// Hermitian ones, bfloat16 by default; FP32 / c64 arithmetic). V holds Ritz vectors v_c with Ritz
// values lam_c (real), and R = A V - V diag(lam) (row-major, leading dimension ld). With
// x_k = c_k v + a e_k (c_k the real scalar recurrence at lam_c) the recurrence of run_rm_filter becomes
//   e_0 = 0, e_1 = R, e_k = a A e_{k-1} + b e_{k-1} - e_{k-2} + c_{k-1} R,
// and the result x_m/(m+1) = coef_c v_c + a e_m/(m+1) is formed in FP64. e_k is small (of the size
// of the residual), so its rounding perturbs the filtered block by the storage rounding times the
// residual instead of times the block: the subspace keeps converging past the FP32 floor of the
// plain FP32 filter. e_2 -> A, e_3 -> B (e_1 = R is read as x_{k-2}), then e_k over e_{k-2}.
// Where a correction-filter application leaves its result: V (column-major), or, with vf set, the
// row-major FP64 block vf formed from the row-major copy yrm of V.
struct CorrRmOut {
    const double* yrm = nullptr;
    int64_t ldy = 0;
    double* vf = nullptr;
    int64_t ldf = 0;
};

template <class Pol, class TS, class TC, int W, class IX, class TM, class TV>
static rc_status run_rm_corr(rc_ctx* ctx, const Pol& pol, int64_t n, TV* V, int64_t ldv, int64_t s,
                             int64_t degree, double a, double b, const TM* R, const float* sig, const double* coef,
                             TM* A, TM* B, int64_t ld, int64_t band, const StageOffsets* so, const CorrRmOut& ro) {
    const int64_t pf_z = ctx->pf_rows;
    const int64_t pf_x = pf_z > 0 ? pf_z + band : 0;
    constexpr int VEC = Slice<TS, TM>::V;  // 8 values per 16-byte slice for bfloat16 blocks
    const TC ta = s_from<TC>(a, 0.0), tb = s_from<TC>(b, 0.0), tm1 = s_from<TC>(-1.0, 0.0);
    if (ld % (VEC * W) != 0) return rc_fail(ctx, RC_ERR_INVALID, "correction filter: leading dimension not padded");
    const int nseg = (int)(ld / (VEC * W));
    if (nseg > kRmThreads) return rc_fail(ctx, RC_ERR_UNSUPPORTED, "correction filter: block too wide");
    constexpr bool kCsr = Pol::kIsCsr;
    // row groups per CTA: 2 with several slices per thread (configuration 2, CSR: filter phase 642-648 ms
    // against 658-665 ms with 4; configuration 3, complex stencil: 624 ms against 637 ms with 4 and 698 ms
    // with 8), else 4 for CSR and 8 for stencils
    const int groups = ctx->rm_groups > 0 ? ctx->rm_groups : (W > 1 ? 2 : (kCsr ? 4 : 8));
    step_mark(ctx);
    // pairs of steps in one pass (rm_corr2_kernel) where the per-row kernels run; the 27-point stencil
    // and the staged kernel take one step per launch
    const bool pairs = ctx->corr_pair && degree >= 3 && !IsStencil27<Pol>::value && !(ctx->staged && so && so->n > 0);
    void* pscr = nullptr;
    const int* fail = nullptr;  // the two-step kernel's error word: the combination below writes NaN if set
    if (pairs) {
        RC_TRY(rc_slot(ctx, S_PAIR, pair_scratch_bytes(n, (int64_t)groups * (kRmThreads / nseg)), &pscr));
        RC_CU(ctx, cudaMemsetAsync((char*)pscr + 8, 0, 8, ctx->stream));
        fail = (const int*)((char*)pscr + 8);
    }
    for (int64_t k = 2; k <= degree;) {
        const TM* xk1 = k == 2 ? R : ((k - 1) % 2 == 0 ? A : B);   // e_{k-1}
        TM* y = k % 2 == 0 ? A : B;                                  // e_k
        const TM* z = k == 2 ? nullptr : (k == 3 ? R : y);           // e_{k-2}
        if (pairs && k + 1 <= degree) {
          if constexpr (!IsStencil27<Pol>::value) {
            TM* y1 = (k + 1) % 2 == 0 ? A : B;                       // e_{k+1}, over e_{k-1} unless that is R
            const rc_status st = launch_pair<Pol, TS, TC, W, IX, TM>(ctx, pol, n, nseg, ld, groups, xk1, z, y, y1, ta,
                                                                     tb, k == 2 ? s_zero(TC()) : tm1, R, sig + k * ld,
                                                                     sig + (k + 1) * ld, pf_z, pf_x, band, pscr);
            if (st != RC_OK) return st;
            k += 2;
            continue;
          }
        }
        launch_step<Pol, TS, TC, W, IX, true, TM>(ctx, pol, n, nseg, ld, groups, xk1, z, y, ta, tb,
                                                  k == 2 ? s_zero(TC()) : tm1, pf_z, pf_x, R, sig + k * ld, so);
        ++k;
    }
    RC_CU(ctx, cudaGetLastError());
    step_mark(ctx);
    const TM* em = degree == 1 ? R : (degree % 2 == 0 ? A : B);
    if (ro.vf) {
        if constexpr (IsComplex<TC>::value) {
            return rc_fail(ctx, RC_ERR_UNSUPPORTED, "correction filter: row-major result for real blocks only");
        } else {
            const int64_t total = n * (ro.ldf / 2);
            const unsigned grid = (unsigned)std::min<int64_t>((total + 255) / 256, (int64_t)ctx->sm_count * 16);
            corr_to_rm_kernel<TM><<<grid, 256, 0, ctx->stream>>>(n, s, ro.yrm, ro.ldy, em, ld, ro.vf, ro.ldf, coef,
                                                                 a / (double)(degree + 1), fail);
        }
    } else {
        const dim3 tgrid((unsigned)((n + 31) / 32), (unsigned)((s + 31) / 32)), tblk(32, 8);
        corr_to_cm_kernel<TM, TV><<<tgrid, tblk, 0, ctx->stream>>>(n, s, em, ld, V, ldv, coef,
                                                                   a / (double)(degree + 1), fail);
    }
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    return RC_OK;
}

// Offset type and slices per thread: 32-bit offsets when the block's last element offset fits;
// two 16-byte slices per thread for CSR with FP64 storage and one otherwise (the faster choice
// on 128^3 7-point operators with 96 columns), unless the context sets the count
// (RCB200_RM_SLICES=1 or 2).
template <class Pol, class TS, class TC>
static rc_status run_rm_select(rc_ctx* ctx, const Pol& pol, int64_t n, void* V, int64_t ldv, int64_t s,
                               int64_t degree, double a, double b, void* bufA, void* bufB, int64_t ld, int64_t band,
                               const StageOffsets* so) {
    const bool small = (n + 1) * ld < ((int64_t)1 << 32);
    const int slices = ctx->rm_slices ? ctx->rm_slices : (Pol::kIsCsr && sizeof(real_t<TS>) == 8 ? 2 : 1);
    if (slices == 1)
        return small ? run_rm_filter<Pol, TS, TC, 1, uint32_t>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB, ld, band,
                                                                  so)
                     : run_rm_filter<Pol, TS, TC, 1, int64_t>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB, ld, band,
                                                              so);
    return small ? run_rm_filter<Pol, TS, TC, 2, uint32_t>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB, ld, band,
                                                           so)
                 : run_rm_filter<Pol, TS, TC, 2, int64_t>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB, ld, band,
                                                          so);
}

template <class TS, class TC>
static rc_status rm_filter_dispatch(rc_ctx* ctx, rc_op* op, void* V, int64_t ldv, int64_t s, int64_t degree,
                                    double a, double b, void* bufA, void* bufB, int64_t ld) {
    const int64_t n = op->n;
    const int64_t band = op->kind == 0 ? op->band : (op->skind == 5 ? op->nx : op->nx * op->ny);
    StageOffsets so_v;
    const StageOffsets* so = stage_offsets(op, &so_v) ? &so_v : nullptr;
    if (op->kind == 0) {
        const TS* vals = (const TS*)(sizeof(real_t<TS>) == 8 ? op->vals64 : op->vals32);
        CsrRows<TS, TC> pol{op->rowptr, op->colind, vals};
        return run_rm_select<CsrRows<TS, TC>, TS, TC>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB, ld, band, so);
    }
    using TD = real_t<TS>;
    const TD* dg = (const TD*)(sizeof(TD) == 8 ? (const void*)op->diag64 : (const void*)op->diag32);
    const double theta = 2.0 * 3.14159265358979323846 * op->flux;
    if (op->skind == 27) {
        if constexpr (IsComplex<TC>::value) {
            return rc_fail(ctx, RC_ERR_UNSUPPORTED, "27-point stencil is real only");
        } else {
            StencilRows<TD, TC, 27> pol{op->nx, op->ny, op->nz, dg, op->offdiag, theta};
            return run_rm_select<StencilRows<TD, TC, 27>, TS, TC>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB,
                                                                  ld, band, so);
        }
    }
    if (op->skind == 7) {
        StencilRows<TD, TC, 7> pol{op->nx, op->ny, op->nz, dg, op->offdiag, theta};
        pol.ph = (const TC*)(sizeof(TD) == 8 ? op->phase64 : op->phase32);
        return run_rm_select<StencilRows<TD, TC, 7>, TS, TC>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB, ld,
                                                             band, so);
    }
    StencilRows<TD, TC, 5> pol{op->nx, op->ny, op->nz, dg, op->offdiag, theta};
    pol.ph = (const TC*)(sizeof(TD) == 8 ? op->phase64 : op->phase32);
    return run_rm_select<StencilRows<TD, TC, 5>, TS, TC>(ctx, pol, n, V, ldv, s, degree, a, b, bufA, bufB, ld, band,
                                                         so);
}

template <class Pol, class TS, class TM, class TV>
static rc_status rm_corr_select(rc_ctx* ctx, const Pol& pol, int64_t n, TV* V, int64_t ldv, int64_t s,
                                int64_t degree, double a, double b, const TM* R, const float* sig,
                                const double* coef, TM* A, TM* B, int64_t ld, int64_t band,
                                const StageOffsets* so, const CorrRmOut& ro) {
    // CSR operators with real bfloat16 blocks: RC_CORR_W 16-byte slices per thread when the padded
    // width allows it. Measured on the 128^3 CSR operator with 96 columns (4 threads per row instead
    // of 12, so each row's index data serve 24 columns per thread): the filter phase of the mixed
    // solve 642-648 ms with 3 slices, 4 resident CTAs and 2 row groups per CTA, against 716-721 ms
    // with 1 slice; 2, 4 and 6 slices were no faster.
#ifndef RC_CORR_W
#define RC_CORR_W 3
#endif
    // Complex blocks (bfloat16 pairs, 4 values per slice; CSR and 5/7-point stencils) likewise: on the
    // 96^3 7-point tight-binding operator with 192 columns (16 threads per row instead of 48, and all
    // 256 threads of a CTA busy instead of 240) the filter phase took 698-699 ms with 3 slices and 4
    // resident CTAs, against 807-808 ms with 1 slice at 6, 734-736 ms with 3 slices at 3 and 831 ms
    // with 2 slices at 4.
#ifndef RC_CORR_W_CPLX
#define RC_CORR_W_CPLX 3
#endif
    constexpr int kWc = std::is_same<TM, __nv_bfloat162>::value && !IsStencil27<Pol>::value ? RC_CORR_W_CPLX : 1;
    if constexpr (kWc > 1) {
        if ((n + 1) * ld < ((int64_t)1 << 32) && ld % (Slice<TS, TM>::V * kWc) == 0)
            return run_rm_corr<Pol, TS, TS, kWc, uint32_t, TM, TV>(ctx, pol, n, V, ldv, s, degree, a, b, R, sig, coef, A,
                                                                   B, ld, band, so, ro);
    }
    if constexpr (RC_CORR_W > 1 && Pol::kIsCsr && std::is_same<TM, __nv_bfloat16>::value) {
        if ((n + 1) * ld < ((int64_t)1 << 32) && ld % (Slice<TS, TM>::V * RC_CORR_W) == 0)
            return run_rm_corr<Pol, TS, TS, RC_CORR_W, uint32_t, TM, TV>(ctx, pol, n, V, ldv, s, degree, a, b, R, sig,
                                                                         coef, A, B, ld, band, so, ro);
    }
    if ((n + 1) * ld < ((int64_t)1 << 32))
        return run_rm_corr<Pol, TS, TS, 1, uint32_t, TM, TV>(ctx, pol, n, V, ldv, s, degree, a, b, R, sig, coef, A, B,
                                                             ld, band, so, ro);
    return run_rm_corr<Pol, TS, TS, 1, int64_t, TM, TV>(ctx, pol, n, V, ldv, s, degree, a, b, R, sig, coef, A, B, ld,
                                                        band, so, ro);
}

// Real operators (CSR, 5/7/27-point stencils) and complex Hermitian ones (CSR, 5/7-point stencils
// with Peierls phases), blocks of up to 256 columns.
bool rm_corr_supported(const rc_op* op, int64_t s) {
    if (op->kind == 2 || s < 1 || s > kCorrMaxCols) return false;
    if (op->dtype == RC_REAL64) return op->kind == 0 || op->skind == 5 || op->skind == 7 || op->skind == 27;
    return op->dtype == RC_COMPLEX128 && (op->kind == 0 || op->skind == 5 || op->skind == 7);
}

template <class TS, class TM, class TV>
static rc_status rm_corr_dispatch(rc_ctx* ctx, rc_op* op, TV* V, int64_t ldv, int64_t s, int64_t degree, double a,
                                  double b, const TM* R, const float* sig, const double* coef, TM* A, TM* B,
                                  int64_t ld, const CorrRmOut& ro) {
    const int64_t n = op->n;
    const int64_t band = op->kind == 0 ? op->band : (op->skind == 5 ? op->nx : op->nx * op->ny);
    StageOffsets so_v;
    const StageOffsets* so = stage_offsets(op, &so_v) ? &so_v : nullptr;
    if (op->kind == 0) {
        CsrRows<TS, TS> pol{op->rowptr, op->colind, (const TS*)op->vals32};
        return rm_corr_select<CsrRows<TS, TS>, TS>(ctx, pol, n, V, ldv, s, degree, a, b, R, sig, coef, A, B, ld, band,
                                                   so, ro);
    }
    const double theta = 2.0 * 3.14159265358979323846 * op->flux;
    if constexpr (!IsComplex<TS>::value) {
        if (op->skind == 27) {
            StencilRows<float, TS, 27> pol{op->nx, op->ny, op->nz, op->diag32, op->offdiag, theta};
            return rm_corr_select<StencilRows<float, TS, 27>, TS>(ctx, pol, n, V, ldv, s, degree, a, b, R, sig, coef,
                                                                  A, B, ld, band, so, ro);
        }
    }
    if (op->skind == 7) {
        StencilRows<float, TS, 7> pol{op->nx, op->ny, op->nz, op->diag32, op->offdiag, theta};
        pol.ph = (const TS*)op->phase32;
        return rm_corr_select<StencilRows<float, TS, 7>, TS>(ctx, pol, n, V, ldv, s, degree, a, b, R, sig, coef, A,
                                                             B, ld, band, so, ro);
    }
    StencilRows<float, TS, 5> pol{op->nx, op->ny, op->nz, op->diag32, op->offdiag, theta};
    pol.ph = (const TS*)op->phase32;
    return rm_corr_select<StencilRows<float, TS, 5>, TS>(ctx, pol, n, V, ldv, s, degree, a, b, R, sig, coef, A, B,
                                                         ld, band, so, ro);
}

rc_status rm_filter_corr(rc_ctx* ctx, rc_op* op, void* V, int64_t ldv, int64_t s, int64_t degree, double a,
                         double b, const double* lam_dev, const void* R, void* bufA, void* bufB, const double* Yrm,
                         int64_t ldy, double* Vf, int64_t ldf) {
    if (!rm_corr_supported(op, s)) return rc_fail(ctx, RC_ERR_UNSUPPORTED, "correction filter: unsupported operator");
    if (Vf && (op->dtype != RC_REAL64 || ctx->serve || !Yrm || ldy < s || ldf < s || ldy % 2 || ldf % 2))
        return rc_fail(ctx, RC_ERR_INVALID, "correction filter: bad row-major result arguments");
    if (degree < 1) return RC_OK;
    RC_TRY(ensure_fp32(ctx, op));
    const bool cplx = op->dtype == RC_COMPLEX128;
    const int64_t ld = corr_leading_dim(op->dtype, s);
    void* tab = nullptr;
    RC_TRY(rc_slot(ctx, S_CORR, corr_table_bytes(degree, ld), &tab));
    float* sig = (float*)tab;
    double* coef = (double*)((char*)tab + corr_table_coef_offset(degree, ld));
    RC_TRY(corr_coefficients(ctx, s, ld, degree, a, b, lam_dev, sig, coef));
    if (ctx->serve && !cplx) {  // under the request server: one job of a batched launch
        bool handled = false;
        RC_TRY(serve_filter_corr(ctx, op, (double*)V, ldv, s, degree, a, b, (const rc_corr_t*)R, sig, coef, bufA,
                                 bufB, &handled));
        if (handled) return RC_OK;
    }
    CorrRmOut ro;
    ro.yrm = Yrm;
    ro.ldy = ldy;
    ro.vf = Vf;
    ro.ldf = ldf;
    if (cplx)
        return rm_corr_dispatch<float2, rc_corr2_t, double2>(ctx, op, (double2*)V, ldv, s, degree, a, b,
                                                            (const rc_corr2_t*)R, sig, coef, (rc_corr2_t*)bufA,
                                                            (rc_corr2_t*)bufB, ld, ro);
    return rm_corr_dispatch<float, rc_corr_t, double>(ctx, op, (double*)V, ldv, s, degree, a, b, (const rc_corr_t*)R,
                                                      sig, coef, (rc_corr_t*)bufA, (rc_corr_t*)bufB, ld, ro);
}

// ---------------------------------------------------------------------------------------
// One degree step on caller-owned row-major blocks (rc_filter_step_rm): the kernels of the
// filter above with the same slice, group and offset choices, so a step over any row range of
// an operator computes each row exactly as the filter does.
// ---------------------------------------------------------------------------------------
template <class Pol, class TS, class TC, int W>
static rc_status step_once_w(rc_ctx* ctx, const Pol& pol, int64_t n, int64_t ld, const TS* x, const TS* z, TS* y,
                             TC a, TC b, TC g, int64_t band, const StageOffsets* so) {
    constexpr int VEC = Pack16<TS>::V;
    const int nseg = (int)(ld / (VEC * W));
    if (nseg > kRmThreads) return rc_fail(ctx, RC_ERR_UNSUPPORTED, "degree step: block too wide");
    constexpr bool kCsr = Pol::kIsCsr;
    constexpr bool kF32 = sizeof(real_t<TS>) == 4;
    const int groups = ctx->rm_groups > 0 ? ctx->rm_groups : (kCsr ? (kF32 ? 4 : 2) : (kF32 ? 8 : 4));
    const int64_t pf_z = ctx->pf_rows;
    const int64_t pf_x = pf_z > 0 ? pf_z + band : 0;
    if ((n + 1) * ld < ((int64_t)1 << 32))
        launch_step<Pol, TS, TC, W, uint32_t, false>(ctx, pol, n, nseg, ld, groups, x, z, y, a, b, g, pf_z, pf_x,
                                                     (const TS*)nullptr, nullptr, so);
    else
        launch_step<Pol, TS, TC, W, int64_t, false>(ctx, pol, n, nseg, ld, groups, x, z, y, a, b, g, pf_z, pf_x,
                                                    (const TS*)nullptr, nullptr, so);
    RC_CU(ctx, cudaGetLastError());
    return RC_OK;
}

template <class Pol, class TS, class TC>
static rc_status step_once(rc_ctx* ctx, const Pol& pol, int64_t n, int64_t ld, const void* x, const void* z, void* y,
                           const double* al, const double* be, const double* ga, int64_t band,
                           const StageOffsets* so) {
    const TC a = s_from<TC>(al[0], al[1]), b = s_from<TC>(be[0], be[1]);
    const TC g = z ? s_from<TC>(ga[0], ga[1]) : s_zero(TC());
    const int slices = ctx->rm_slices ? ctx->rm_slices : (Pol::kIsCsr && sizeof(real_t<TS>) == 8 ? 2 : 1);
    if (slices == 2)
        return step_once_w<Pol, TS, TC, 2>(ctx, pol, n, ld, (const TS*)x, (const TS*)z, (TS*)y, a, b, g, band, so);
    return step_once_w<Pol, TS, TC, 1>(ctx, pol, n, ld, (const TS*)x, (const TS*)z, (TS*)y, a, b, g, band, so);
}

template <class TS, class TC>
static rc_status step_dispatch(rc_ctx* ctx, rc_op* op, int64_t ld, const void* x, const void* z, void* y,
                               const double* al, const double* be, const double* ga) {
    const int64_t n = op->n;
    const int64_t band = op->kind == 0 ? op->band : (op->skind == 5 ? op->nx : op->nx * op->ny);
    StageOffsets so_v;
    const StageOffsets* so = stage_offsets(op, &so_v) ? &so_v : nullptr;
    if (op->kind == 0) {
        const TS* vals = (const TS*)(sizeof(real_t<TS>) == 8 ? op->vals64 : op->vals32);
        CsrRows<TS, TC> pol{op->rowptr, op->colind, vals};
        return step_once<CsrRows<TS, TC>, TS, TC>(ctx, pol, n, ld, x, z, y, al, be, ga, band, so);
    }
    using TD = real_t<TS>;
    const TD* dg = (const TD*)(sizeof(TD) == 8 ? (const void*)op->diag64 : (const void*)op->diag32);
    const double theta = 2.0 * 3.14159265358979323846 * op->flux;
    if (op->skind == 27) {
        if constexpr (IsComplex<TC>::value) {
            return rc_fail(ctx, RC_ERR_UNSUPPORTED, "27-point stencil is real only");
        } else {
            StencilRows<TD, TC, 27> pol{op->nx, op->ny, op->nz, dg, op->offdiag, theta};
            return step_once<StencilRows<TD, TC, 27>, TS, TC>(ctx, pol, n, ld, x, z, y, al, be, ga, band, so);
        }
    }
    if (op->skind == 7) {
        StencilRows<TD, TC, 7> pol{op->nx, op->ny, op->nz, dg, op->offdiag, theta};
        pol.ph = (const TC*)(sizeof(TD) == 8 ? op->phase64 : op->phase32);
        return step_once<StencilRows<TD, TC, 7>, TS, TC>(ctx, pol, n, ld, x, z, y, al, be, ga, band, so);
    }
    StencilRows<TD, TC, 5> pol{op->nx, op->ny, op->nz, dg, op->offdiag, theta};
    pol.ph = (const TC*)(sizeof(TD) == 8 ? op->phase64 : op->phase32);
    return step_once<StencilRows<TD, TC, 5>, TS, TC>(ctx, pol, n, ld, x, z, y, al, be, ga, band, so);
}

rc_status rm_step(rc_ctx* ctx, rc_op* op, const void* x, const void* z, void* y, int64_t ld, int64_t s,
                  const double* alpha, const double* beta, const double* gamma, int prec) {
    if (op->kind == 2) return rc_fail(ctx, RC_ERR_UNSUPPORTED, "degree step: callback operators have no row form");
    const bool cplx = op->dtype == RC_COMPLEX128;
    const int p = prec == RC_PREC_MIXED ? P32 : P64;
    const int64_t q = rm_leading_dim(op->dtype, p, 1);  // the row length quantum (32 bytes)
    if (ld < s || ld % q != 0)
        return rc_fail(ctx, RC_ERR_INVALID, "degree step: ld must be >= s and a multiple of 32 bytes of elements");
    if (p == P32) {
        RC_TRY(ensure_fp32(ctx, op));
        if (cplx) return step_dispatch<float2, float2>(ctx, op, ld, x, z, y, alpha, beta, gamma);
        return step_dispatch<float, float>(ctx, op, ld, x, z, y, alpha, beta, gamma);
    }
    if (cplx) return step_dispatch<double2, double2>(ctx, op, ld, x, z, y, alpha, beta, gamma);
    return step_dispatch<double, double>(ctx, op, ld, x, z, y, alpha, beta, gamma);
}

rc_status corr_coefficients(rc_ctx* ctx, int64_t s, int64_t ld, int64_t degree, double a, double b,
                            const double* lam_dev, float* sig, double* coef) {
    corr_coef_kernel<<<1, 128, 0, ctx->stream>>>(s, ld, degree, a, b, lam_dev, sig, coef);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    return RC_OK;
}

rc_status to_row_major(rc_ctx* ctx, int dtype, int64_t n, int64_t s, const void* V, int64_t ldv, void* Yrm,
                       int64_t ld) {
    if ((s + 31) / 32 > 65535) return rc_fail(ctx, RC_ERR_UNSUPPORTED, "row-major copy: too many columns");
    const dim3 tgrid((unsigned)((n + 31) / 32), (unsigned)((s + 31) / 32)), tblk(32, 8);
    if (dtype == RC_COMPLEX128)
        to_rm_kernel<double2, double2><<<tgrid, tblk, 0, ctx->stream>>>(n, s, (const double2*)V, ldv, (double2*)Yrm,
                                                                        ld);
    else
        to_rm_kernel<double, double><<<tgrid, tblk, 0, ctx->stream>>>(n, s, (const double*)V, ldv, (double*)Yrm, ld);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    return RC_OK;
}

rc_status to_col_major(rc_ctx* ctx, int dtype, int64_t n, int64_t s, const void* Yrm, int64_t ld, void* V,
                       int64_t ldv) {
    if ((s + 31) / 32 > 65535) return rc_fail(ctx, RC_ERR_UNSUPPORTED, "column-major copy: too many columns");
    const dim3 tgrid((unsigned)((n + 31) / 32), (unsigned)((s + 31) / 32)), tblk(32, 8);
    if (dtype == RC_COMPLEX128)
        to_cm_kernel<double2, double2><<<tgrid, tblk, 0, ctx->stream>>>(n, s, (const double2*)Yrm, ld, (double2*)V,
                                                                        ldv, 1.0);
    else
        to_cm_kernel<double, double><<<tgrid, tblk, 0, ctx->stream>>>(n, s, (const double*)Yrm, ld, (double*)V, ldv,
                                                                      1.0);
    ctx->launches++;
    RC_CU(ctx, cudaGetLastError());
    return RC_OK;
}

// Row length padded to 32 bytes (two 16-byte slices); the padding columns are never read back.
int64_t rm_leading_dim(int dtype, int prec, int64_t s) {
    const int64_t v = 32 / (int64_t)elem_bytes(dtype, prec);
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
