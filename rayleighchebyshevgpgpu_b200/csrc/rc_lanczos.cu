// rc_lanczos.cu -- spectral bounds by single-vector Lanczos on the GPU.
//
// Follows LanczosMaxMinFinder::getMinMaxEigenvalues (LanczosMaxMinFinder.h:248-544): the
// reference runs the recurrence on HOST vectors through the operator's host apply(Vtype&)
// (:341) and calls the f2c dstebz every 5 steps (:395-414). Here the vectors stay on the
// device, alpha_k/beta_k are reduced on the device (last-block reduction in a fixed order,
// so results are deterministic), and the extreme eigenvalues of the k x k tridiagonal are
// found by Sturm-count multisection in one warp per extreme. The host reads two doubles
// every 5 steps and applies the reference's stopping rule unchanged.
#include <cmath>
#include <cstdio>
#include <vector>
#include "rc_common.cuh"
#include "rc_internal.h"

namespace rcb {

constexpr int LZ_THREADS = 256;

struct LzScalars {
    double* alpha;      // [max_iter]
    double* beta;       // [max_iter]
    double2* part;      // [nblocks]
    unsigned* counter;  // [2]
    int* flags;         // [2]: [0] non-Hermitian
    double* ext;        // [2]: min, max
    double* alpha_im;   // [max_iter] imaginary part of w.v (diagnostic)
};

__device__ __forceinline__ bool last_block(unsigned* counter) {
    __shared__ bool s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned t = atomicAdd(counter, 1u);
        s_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    return s_last;
}

// Sum of the per-block partials in a fixed order (called by the last block only).
__device__ double2 sum_parts(const double2* part, int nblocks, double* scratch) {
    double sx = 0.0, sy = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        const double2 p = __ldcg(part + b);
        sx += p.x;
        sy += p.y;
    }
    sx = block_sum(sx, scratch);
    sy = block_sum(sy, scratch);
    return make_double2(sx, sy);
}

// (a) swap of LanczosMaxMinFinder.h:329-338: if |beta_{k-1}| > 1e-14
//     w <- v / beta_{k-1},  v <- -beta_{k-1} * w_old
template <class T>
__global__ void lz_prep_kernel(int64_t n, T* w, T* v, const double* beta, int64_t km1) {
    const double b = beta[km1];
    if (!(fabs(b) > 1e-14)) return;
    const double ib = 1.0 / b;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const T wo = w[i];
        w[i] = s_rscale(ib, v[i]);
        v[i] = s_rscale(-b, wo);
    }
}

// (c) v <- v + A w (Aw precomputed in aw), alpha_k = w.dot(v) = sum w_i conj(v_i) (:343-356)
template <class T>
__global__ void lz_combine_kernel(int64_t n, const T* __restrict__ w, T* __restrict__ v, const T* __restrict__ aw,
                                  LzScalars sc, int64_t k, int zero_v) {
    __shared__ double scratch[32];
    double sx = 0.0, sy = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const T vn = zero_v ? aw[i] : s_add(v[i], aw[i]);
        v[i] = vn;
        // w_i * conj(v_i)
        const T wi = w[i];
        if constexpr (IsComplex<T>::value) {
            sx += wi.x * vn.x + wi.y * vn.y;
            sy += wi.y * vn.x - wi.x * vn.y;
        } else {
            sx += s_real(wi) * s_real(vn);
        }
    }
    sx = block_sum(sx, scratch);
    sy = block_sum(sy, scratch);
    if (threadIdx.x == 0) sc.part[blockIdx.x] = make_double2(sx, sy);
    if (last_block(sc.counter)) {
        const double2 a = sum_parts(sc.part, gridDim.x, scratch);
        if (threadIdx.x == 0) {
            sc.alpha[k] = a.x;
            sc.alpha_im[k] = a.y;
            if (fabs(a.y) > (1.0 + fabs(a.x)) * 1e-12) sc.flags[0] = 1;
            if (!isfinite(a.x) || !isfinite(a.y)) sc.flags[1] = 1;
            *sc.counter = 0u;
        }
    }
}

// (d) v <- v - alpha_k w; beta_k = ||v|| (:358-363)
template <class T>
__global__ void lz_update_kernel(int64_t n, const T* __restrict__ w, T* __restrict__ v, LzScalars sc, int64_t k) {
    __shared__ double scratch[32];
    const double a = sc.alpha[k];
    double s2 = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const T vn = s_sub(v[i], s_rscale(a, w[i]));
        v[i] = vn;
        s2 += s_abs2(vn);
    }
    s2 = block_sum(s2, scratch);
    if (threadIdx.x == 0) sc.part[blockIdx.x] = make_double2(s2, 0.0);
    if (last_block(sc.counter)) {
        const double2 t = sum_parts(sc.part, gridDim.x, scratch);
        if (threadIdx.x == 0) {
            sc.beta[k] = sqrt(fabs(t.x));
            if (!isfinite(t.x)) sc.flags[1] = 1;
            *sc.counter = 0u;
        }
    }
}

// Normalise the start vector: w <- v/||v||, v <- 0 (:272-281).
template <class T>
__global__ void lz_norm_kernel(int64_t n, const T* __restrict__ v, double2* part, unsigned* counter, double* out) {
    __shared__ double scratch[32];
    double s2 = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        s2 += s_abs2(v[i]);
    s2 = block_sum(s2, scratch);
    if (threadIdx.x == 0) part[blockIdx.x] = make_double2(s2, 0.0);
    if (last_block(counter)) {
        const double2 t = sum_parts(part, gridDim.x, scratch);
        if (threadIdx.x == 0) {
            out[0] = sqrt(fabs(t.x));
            *counter = 0u;
        }
    }
}

template <class T>
__global__ void lz_start_kernel(int64_t n, T* w, T* v, const double* nrm) {
    const double inv = 1.0 / nrm[0];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        w[i] = s_rscale(inv, v[i]);
        v[i] = s_zero(T());
    }
}

// Number of eigenvalues of the symmetric tridiagonal (d, e) below x (Sturm sequence).
__device__ int sturm_count(int k, const double* d, const double* e, double x, double pivmin) {
    int cnt = 0;
    double q = d[0] - x;
    if (fabs(q) < pivmin) q = -pivmin;
    cnt += q < 0.0;
    for (int i = 1; i < k; ++i) {
        q = d[i] - x - e[i - 1] * e[i - 1] / q;
        if (fabs(q) < pivmin) q = -pivmin;
        cnt += q < 0.0;
    }
    return cnt;
}

// Warp 0: smallest eigenvalue, warp 1: largest. Multisection with 32 probes per round,
// to the absolute tolerance 1e-14 of getLargestSymTriEigValues (LanczosMaxMinFinder.h:620).
__global__ void tridiag_extremes_kernel(int k, const double* __restrict__ alpha, const double* __restrict__ beta,
                                        double* __restrict__ out) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (wid > 1) return;
    double lo = 1e300, hi = -1e300, emax2 = 0.0;
    for (int i = lane; i < k; i += 32) {
        const double el = i > 0 ? fabs(beta[i - 1]) : 0.0;
        const double er = i < k - 1 ? fabs(beta[i]) : 0.0;
        lo = fmin(lo, alpha[i] - el - er);
        hi = fmax(hi, alpha[i] + el + er);
        emax2 = fmax(emax2, er * er);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        emax2 = fmax(emax2, __shfl_xor_sync(0xffffffffu, emax2, o));
    }
    const double pivmin = 2.2250738585072014e-308 * fmax(1.0, emax2);
    const double spread = fmax(hi - lo, 1e-300);
    double a = lo - 1e-12 * spread - 1e-300, b = hi + 1e-12 * spread + 1e-300;
    const int target = wid == 0 ? 0 : k - 1;  // 0-based index in ascending order
    const double abstol = 1e-14, eps = 2.220446049250313e-16;
    for (int it = 0; it < 64; ++it) {
        if (b - a <= fmax(abstol, 2.0 * eps * fmax(fabs(a), fabs(b)))) break;
        const double x = a + (b - a) * (double)(lane + 1) / 33.0;
        const int c = sturm_count(k, alpha, beta, x, pivmin);
        const unsigned le = __ballot_sync(0xffffffffu, c <= target);  // prefix of lanes
        const int p = __popc(le);
        const double xa = __shfl_sync(0xffffffffu, x, p > 0 ? p - 1 : 0);
        const double xb = __shfl_sync(0xffffffffu, x, p < 32 ? p : 31);
        if (p > 0) a = xa;
        if (p < 32) b = xb;
    }
    if (lane == 0) out[wid] = 0.5 * (a + b);
}

static double rel_factor(double val, double tol) {
    // LanczosMaxMinFinder::getRelErrorFactor (LanczosMaxMinFinder.h:161-168), LANCZOS_SMALL_TOL_ = 1e-10
    if (std::fabs(val) * tol > 1e-10) return std::fabs(val);
    return 1e-10 / tol;
}

template <class T>
static rc_status lanczos_t(rc_ctx* ctx, rc_op* op, const void* v0_host, uint64_t seed, double errorTolerance,
                           int which, int64_t max_iter, LanczosResult* res) {
    const int64_t n = op->n;
    const int dtype = op->dtype;
    const size_t esz = sizeof(T);
    const int nblk = (int)std::min<int64_t>((n + LZ_THREADS - 1) / LZ_THREADS, 4 * ctx->sm_count);
    if (max_iter < 1) max_iter = 1;
    // layout in S_LANCZOS: w, v, aw (n each), then scalars
    const size_t vec_bytes = ((n * esz + 255) / 256) * 256;
    const size_t scal_bytes = (size_t)max_iter * 8 * 3 + (size_t)nblk * 16 + 64 + 64 + 64;
    void* base = nullptr;
    RC_TRY(rc_slot(ctx, S_LANCZOS, 3 * vec_bytes + scal_bytes + 1024, &base));
    T* w = (T*)base;
    T* v = (T*)((char*)base + vec_bytes);
    T* aw = (T*)((char*)base + 2 * vec_bytes);
    char* sp = (char*)base + 3 * vec_bytes;
    LzScalars sc;
    sc.alpha = (double*)sp;
    sc.beta = sc.alpha + max_iter;
    sc.alpha_im = sc.beta + max_iter;
    sc.part = (double2*)(sc.alpha_im + max_iter);
    sc.counter = (unsigned*)(sc.part + nblk);
    sc.flags = (int*)(sc.counter + 4);
    sc.ext = (double*)(sc.flags + 4);
    double* nrm = sc.ext + 2;
    RC_CU(ctx, cudaMemsetAsync(sp, 0, scal_bytes, ctx->stream));
    // start vector into v
    if (v0_host) {
        RC_CU(ctx, cudaMemcpyAsync(v, v0_host, n * esz, cudaMemcpyHostToDevice, ctx->stream));
    } else {
        RC_TRY(fill_random(ctx, dtype, v, n, n, 0, 1, seed));
    }
    lz_norm_kernel<T><<<nblk, LZ_THREADS, 0, ctx->stream>>>(n, v, sc.part, sc.counter, nrm);
    lz_start_kernel<T><<<nblk, LZ_THREADS, 0, ctx->stream>>>(n, w, v, nrm);
    ctx->launches += 2;
    RC_CU(ctx, cudaGetLastError());

    double* hbuf = nullptr;
    RC_TRY(rc_host_small(ctx, 64, &hbuf));

    if (errorTolerance > 0.01) errorTolerance = 0.01;  // (:286)
    double tol = errorTolerance;
    if (tol < 1e-10) tol = 1e-10;
    const bool maxEigFlag = which != 2, minEigFlag = which != 1;

    double minDiffError = 1.0e10, maxDiffError = 1.0e10;
    double lanczosMin = 0.0, lanczosMax = 0.0;
    double rateFactorMax = 9.0, rateFactorMin = 9.0;
    double rateEigMax = 1.0, rateEigMin = 1.0;
    double eigMaxOld = 0.0, eigMinOld = 0.0;
    double diffMaxA = 0.0, diffMinA = 0.0, diffMaxB = 0.0, diffMinB = 0.0;
    int diffCompareFlag = 0, rateCompareFlag = 0;
    bool exitFlag = false;
    int64_t k = 0;
    StepArgs st;
    st.s = 1;
    st.x = w; st.xp = P64; st.ldx = n;
    st.y = aw; st.yp = P64; st.ldy = n;
    st.cp = P64;
    while (k < max_iter && !exitFlag) {
        if (k != 0) {
            lz_prep_kernel<T><<<nblk, LZ_THREADS, 0, ctx->stream>>>(n, w, v, sc.beta, k - 1);
            ctx->launches++;
        }
        RC_TRY(op_step(ctx, op, st));  // aw = A w
        lz_combine_kernel<T><<<nblk, LZ_THREADS, 0, ctx->stream>>>(n, w, v, aw, sc, k, 0);
        lz_update_kernel<T><<<nblk, LZ_THREADS, 0, ctx->stream>>>(n, w, v, sc, k);
        ctx->launches += 2;
        RC_CU(ctx, cudaGetLastError());
        k += 1;
        if ((k % 5) == 0) {
            tridiag_extremes_kernel<<<1, 64, 0, ctx->stream>>>((int)k, sc.alpha, sc.beta, sc.ext);
            ctx->launches++;
            RC_CU(ctx, cudaGetLastError());
            RC_CU(ctx, cudaMemcpyAsync(hbuf, sc.ext, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
            RC_CU(ctx, cudaMemcpyAsync(hbuf + 2, sc.flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
            RC_CU(ctx, cudaStreamSynchronize(ctx->stream));
            if (((const int*)(hbuf + 2))[0])
                return rc_fail(ctx, RC_ERR_NOT_HERMITIAN,
                               "Lanczos max/min finder: input complex valued operator not Hermitian");
            lanczosMin = hbuf[0];
            lanczosMax = hbuf[1];
            if (((const int*)(hbuf + 2))[1] || !std::isfinite(lanczosMin) || !std::isfinite(lanczosMax))
                return rc_fail(ctx, RC_ERR_BREAKDOWN, "Lanczos produced a non-finite value (NaN/Inf in the operator?)");
            // stopping rule of LanczosMaxMinFinder.h:416-523
            if (diffCompareFlag == 0) {
                eigMaxOld = lanczosMax;
                eigMinOld = lanczosMin;
                diffCompareFlag = 1;
            } else {
                maxDiffError = std::fabs(lanczosMax - eigMaxOld) / rel_factor(lanczosMax, tol);
                minDiffError = std::fabs(lanczosMin - eigMinOld) / rel_factor(lanczosMin, tol);
                if (rateCompareFlag == 0) {
                    diffMaxA = std::fabs(lanczosMax - eigMaxOld);
                    diffMinA = std::fabs(lanczosMin - eigMinOld);
                    rateCompareFlag = 1;
                } else {
                    if (maxDiffError > 1.0e-09) {
                        diffMaxB = std::fabs(lanczosMax - eigMaxOld);
                        rateEigMax = diffMaxB / diffMaxA;
                    } else {
                        rateEigMax = 0.95;
                    }
                    if (minDiffError > 1.0e-09) {
                        diffMinB = std::fabs(lanczosMin - eigMinOld);
                        rateEigMin = diffMinB / diffMinA;
                    } else {
                        rateEigMin = 0.95;
                    }
                    rateFactorMax = 9.0;
                    rateFactorMin = 9.0;
                    if (rateEigMax < 0.90) rateFactorMax = rateEigMax / (1.0 - rateEigMax);
                    if (rateEigMin < 0.90) rateFactorMin = rateEigMin / (1.0 - rateEigMin);
                    diffMaxA = diffMaxB;
                    diffMinA = diffMinB;
                }
                eigMaxOld = lanczosMax;
                eigMinOld = lanczosMin;
                minDiffError *= rateFactorMin;
                maxDiffError *= rateFactorMax;
            }
            if (maxEigFlag && minEigFlag) {
                if ((minDiffError < tol) && (maxDiffError < tol)) exitFlag = true;
            } else if (maxEigFlag) {
                if (maxDiffError < tol) exitFlag = true;
            } else if (minEigFlag) {
                if (minDiffError < tol) exitFlag = true;
            }
        }
    }
    if (k % 5 != 0 || k == 0) {
        // iteration cap reached between checks: evaluate the final tridiagonal once more
        if (k > 0) {
            tridiag_extremes_kernel<<<1, 64, 0, ctx->stream>>>((int)k, sc.alpha, sc.beta, sc.ext);
            ctx->launches++;
            RC_CU(ctx, cudaMemcpyAsync(hbuf, sc.ext, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
            RC_CU(ctx, cudaStreamSynchronize(ctx->stream));
            lanczosMin = hbuf[0];
            lanczosMax = hbuf[1];
        }
    }
    if (lanczosMin > lanczosMax) std::swap(lanczosMin, lanczosMax);
    res->lmin = lanczosMin;
    res->lmax = lanczosMax;
    res->iters = k;
    return RC_OK;
}

rc_status lanczos_bounds(rc_ctx* ctx, rc_op* op, const void* v0_host, uint64_t seed, double tol, int which,
                         int64_t max_iter, LanczosResult* res) {
    if (op->dtype == RC_COMPLEX128)
        return lanczos_t<double2>(ctx, op, v0_host, seed, tol, which, max_iter, res);
    return lanczos_t<double>(ctx, op, v0_host, seed, tol, which, max_iter, res);
}

}  // namespace rcb
