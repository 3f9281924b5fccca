// rc_staged.cuh -- the filter's degree step with its operands staged in shared memory.
//
// The row-major step (rc_rmstep.cuh) reads every neighbour row of x_{k-1} with a 16-byte gather
// from L1/L2 and waits on each. For operators whose rows couple to a few fixed row offsets (the
// 5/7-point stencils, and CSR matrices with at most a few distinct column offsets, such as the
// stencil operators stored as CSR), the rows a chunk of R consecutive rows needs form a few
// contiguous windows of x_{k-1}: one per group of nearby offsets, e.g. for the 7-point stencil on an
// nx*ny*nz grid the windows at offsets -nx*ny, -nx, [-1, +1], +nx, +nx*ny. The CTA copies those
// windows, the chunk's rows of x_{k-2} and of the source block, and (CSR) the chunk's row pointers,
// column indices and values into shared memory with asynchronous 16-byte copies (cp.async, every
// thread taking a share, so each SM keeps thousands of requests in flight), several chunks ahead
// of the chunk it computes. The compute reads shared memory with the arithmetic of rm_step_rows --
// the same products in the same order, so the results equal the unstaged kernel's bit for bit --
// and stores the rows of x_k. CTAs are persistent (two per SM) and take chunks blockIdx.x,
// blockIdx.x + gridDim.x, ..., so the rows in flight still form one band moving down the block and
// the windows' far rows are L2 hits; DRAM sees each row of every block once per step.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "rc_rmstep.cuh"

namespace rcb {

constexpr int kStagedMaxWin = 6;
constexpr int kStagedMaxStages = 4;
constexpr int kStagedThreads = 256;

// Where a chunk's operands live in one pipeline stage (byte offsets from the stage base, each a
// multiple of 128), and the windows of x_{k-1}: window w holds rows [r0 + lo[w], r0 + lo[w] + R + span[w])
// of the chunk starting at row r0 (rows outside [0, n) are not copied and never read).
struct StagedPlan {
    int nwin = 0;
    int64_t lo[kStagedMaxWin] = {};
    int span[kStagedMaxWin] = {};
    int win_off[kStagedMaxWin] = {};
    int R = 0;              // rows per chunk, a multiple of 4
    int nstages = 2;
    int ctas_per_sm = 2;
    int64_t nchunks = 0;
    int z_off = -1, src_off = -1;             // own rows of x_{k-2} and of the source block
    int rp_off = -1, ci_off = -1, va_off = -1;  // CSR: row pointers, column indices, values
    int csr_cap = 0;        // staged CSR entries per chunk (with the 16-byte alignment slack)
    int stage_bytes = 0;
};

// ---- PTX wrappers: asynchronous copies and shared-memory loads ------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
// 16 bytes global -> shared, cached in L2 only (a staged row is read from shared memory afterwards).
__device__ __forceinline__ void cpasync16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cpasync_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Wait until at most n of this thread's copy groups are pending (n = 0..3).
__device__ __forceinline__ void cpasync_wait(int n) {
    switch (n) {
        case 0: asm volatile("cp.async.wait_group 0;" ::: "memory"); break;
        case 1: asm volatile("cp.async.wait_group 1;" ::: "memory"); break;
        case 2: asm volatile("cp.async.wait_group 2;" ::: "memory"); break;
        default: asm volatile("cp.async.wait_group 3;" ::: "memory"); break;
    }
}
// The CTA's share of copying `bytes` (a multiple of 16) from global src to shared dst.
__device__ __forceinline__ void copy_span(uint32_t dst, const void* src, int64_t bytes) {
    const unsigned char* s = (const unsigned char*)src;
    for (int64_t o = (int64_t)threadIdx.x * 16; o < bytes; o += (int64_t)blockDim.x * 16) cpasync16(dst + (uint32_t)o, s + o);
}

// Shared-memory loads by 32-bit shared address (16-byte slices as one 128-bit access; volatile so
// they stay after the barrier that makes the staged data visible).
__device__ __forceinline__ uint4 lds128(uint32_t a) {
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a));
    return v;
}
__device__ __forceinline__ int32_t lds32(uint32_t a) {
    int32_t v;
    asm volatile("ld.shared.b32 %0, [%1];" : "=r"(v) : "r"(a));
    return v;
}
template <class T>
__device__ __forceinline__ T lds_val(uint32_t a) {
    if constexpr (sizeof(T) == 4) {
        uint32_t u;
        asm volatile("ld.shared.b32 %0, [%1];" : "=r"(u) : "r"(a));
        T v;
        memcpy(&v, &u, 4);
        return v;
    } else if constexpr (sizeof(T) == 8) {
        unsigned long long u;
        asm volatile("ld.shared.b64 %0, [%1];" : "=l"(u) : "r"(a));
        T v;
        memcpy(&v, &u, 8);
        return v;
    } else {
        const uint4 u = lds128(a);
        T v;
        memcpy(&v, &u, 16);
        return v;
    }
}

// ---- staged row policies: f(j, a_ij) for every entry of row i ---------------------------------
// CSR with the chunk's rows pointers, column indices and values in shared memory: rp holds
// rowptr[r0 ..], ci/va hold the entries from kbase (rowptr[r0] rounded down to a multiple of 4).
template <class TA, class TC>
struct StagedCsr {
    uint32_t rp, ci, va;  // shared addresses of the staged row pointers, column indices, values
    int64_t r0;
    int32_t kbase;
    template <class F>
    __device__ __forceinline__ void row(int64_t i, F&& f) const {
        const int32_t k0 = lds32(rp + 4u * (uint32_t)(i - r0)), k1 = lds32(rp + 4u * (uint32_t)(i - r0 + 1));
#pragma unroll 4
        for (int32_t k = k0; k < k1; ++k) {
            const uint32_t e = (uint32_t)(k - kbase);
            f((int64_t)lds32(ci + 4u * e), s_cvt<TC>(lds_val<TA>(va + (uint32_t)sizeof(TA) * e)));
        }
    }
};

// The stencil policies of rc_rowops.cuh compute their entries; nothing to stage.
template <class Pol>
struct StagedStencil {
    Pol pol;
    template <class F>
    __device__ __forceinline__ void row(int64_t i, F&& f) const {
        pol.row(i, f);
    }
};

template <class TM, class TC>
struct StagedArgs {
    int64_t n = 0;
    int nseg = 0;
    int64_t ld = 0;         // elements per row
    int row_bytes = 0;      // ld * sizeof(TM)
    const TM* x = nullptr;  // x_{k-1}
    const TM* z = nullptr;  // x_{k-2} (null: no gamma term)
    TM* y = nullptr;        // x_k (may alias z)
    const TM* src = nullptr;
    const float* sig = nullptr;
    TC alpha{}, beta{}, gamma{};
    // CSR operator arrays (global; null for stencils)
    const int32_t* rowptr = nullptr;
    const int32_t* colind = nullptr;
    const void* vals = nullptr;
};

// Every thread's share of the copies of chunk c into the stage at shared address `stage`. CSR:
// k0, k1 = rowptr[r0], rowptr[r0 + own] of the chunk (loaded ahead by the caller).
template <class TM, class TC, class TA>
__device__ __forceinline__ void staged_issue(const StagedPlan& P, const StagedArgs<TM, TC>& a, int64_t c,
                                             uint32_t stage, int32_t k0, int32_t k1) {
    const int64_t r0 = c * P.R;
    const int64_t own = min((int64_t)P.R, a.n - r0);
    const int64_t rb = a.row_bytes;
    for (int w = 0; w < P.nwin; ++w) {
        const int64_t lo = r0 + P.lo[w], hi = lo + P.R + P.span[w];
        const int64_t cl = max(lo, (int64_t)0), ch = min(hi, a.n);
        if (ch > cl)
            copy_span(stage + (uint32_t)P.win_off[w] + (uint32_t)((cl - lo) * rb), (const unsigned char*)a.x + cl * rb,
                      (ch - cl) * rb);
    }
    if (a.z) copy_span(stage + (uint32_t)P.z_off, (const unsigned char*)a.z + r0 * rb, own * rb);
    if (a.src) copy_span(stage + (uint32_t)P.src_off, (const unsigned char*)a.src + r0 * rb, own * rb);
    if (a.rowptr) {
        const int64_t rcount = ((own + 1) + 3) & ~(int64_t)3;  // rowptr[r0 .. r0 + own], rounded up to 16 bytes
        copy_span(stage + (uint32_t)P.rp_off, a.rowptr + r0, rcount * 4);
        const int64_t ka = k0 & ~(int64_t)3, kb = ((int64_t)k1 + 3) & ~(int64_t)3;
        if (kb > ka) {
            copy_span(stage + (uint32_t)P.ci_off, a.colind + ka, (kb - ka) * 4);
            copy_span(stage + (uint32_t)P.va_off, (const TA*)a.vals + ka, (kb - ka) * (int64_t)sizeof(TA));
        }
    }
}

// One chunk on the CTA's threads, from the stage at shared address `stage`.
template <class Pol, class TS, class TC, int W, bool SRC, class TM>
__device__ __forceinline__ void staged_compute(const StagedPlan& P, const StagedArgs<TM, TC>& a, const Pol& op,
                                               int64_t r0, uint32_t stage) {
    constexpr int V = Slice<TS, TM>::V;
    const int nseg = a.nseg;
    const int rows_per_iter = kStagedThreads / nseg;
    const int rloc = threadIdx.x / nseg;
    if (rloc >= rows_per_iter) return;
    const int64_t off = (int64_t)(threadIdx.x - rloc * nseg) * V;
    const uint32_t boff = (uint32_t)(off * (int64_t)sizeof(TM));             // this thread's byte offset in a row
    const uint32_t bstride = (uint32_t)((int64_t)nseg * V * (int64_t)sizeof(TM));  // between its W slices
    const int64_t wstride = (int64_t)nseg * V;
    const uint32_t rb = (uint32_t)a.row_bytes;
    const int64_t own = min((int64_t)P.R, a.n - r0);
    constexpr bool kPacked = sizeof(TM) == 2;
    // the shared address of row j of x_{k-1} (relative row d = j - r0): the first window holding it,
    // or ~0u when no window does (then global memory). Per-chunk window constants are hoisted:
    // wbase[q] = address of relative row 0 in window q, wlo[q] = its first relative row, wlen[q]
    // its row count (0 past nwin); the lookup is branchless 32-bit arithmetic.
    uint32_t wbase[kStagedMaxWin];
    int32_t wlo[kStagedMaxWin], wlen[kStagedMaxWin];
#pragma unroll
    for (int q = 0; q < kStagedMaxWin; ++q) {
        const bool on = q < P.nwin;
        wlo[q] = on ? (int32_t)P.lo[q] : 0;
        wlen[q] = on ? P.R + P.span[q] : 0;
        wbase[q] = stage + (uint32_t)(on ? P.win_off[q] : 0) - (uint32_t)wlo[q] * rb + boff;
    }
    auto xaddr = [&](int64_t j) -> uint32_t {
        const int32_t d = (int32_t)(j - r0);
        uint32_t addr = ~0u;
#pragma unroll
        for (int q = kStagedMaxWin - 1; q >= 0; --q)
            addr = (uint32_t)(d - wlo[q]) < (uint32_t)wlen[q] ? wbase[q] + (uint32_t)d * rb : addr;
        return addr;
    };
    auto xslice = [&](uint32_t addr, int64_t j, int w) -> Slice<TS, TM> {
        if (addr != ~0u) return slice_from<TS, TM>(lds128(addr + (uint32_t)w * bstride));
        return ldv_ro<TS, TM>(a.x + j * a.ld + off + w * wstride);
    };
    for (int64_t li = rloc; li < own; li += rows_per_iter) {
        const int64_t i = r0 + li;
        TC acc[W * V];
#pragma unroll
        for (int v = 0; v < W * V; ++v) acc[v] = s_zero(TC());
        op.row(i, [&](int64_t j, TC aij) {
            const uint32_t xa = xaddr(j);
#pragma unroll
            for (int w = 0; w < W; ++w) {
                const Slice<TS, TM> p = xslice(xa, j, w);
                if constexpr (kPacked) {
#pragma unroll
                    for (int v = 0; v < V; v += 2)
                        ffma2(aij, aij, p.v[v], p.v[v + 1], acc[w * V + v], acc[w * V + v + 1]);
                } else {
#pragma unroll
                    for (int v = 0; v < V; ++v) acc[w * V + v] = s_fma(aij, s_cvt<TC>(p.v[v]), acc[w * V + v]);
                }
            }
        });
        const uint32_t zrow = stage + (uint32_t)P.z_off + (uint32_t)li * rb + boff;
        const uint32_t srow = stage + (uint32_t)P.src_off + (uint32_t)li * rb + boff;
        const bool hz = a.z != nullptr;
        TM* yi = a.y + i * a.ld + off;
        const uint32_t xia = xaddr(i);
#pragma unroll
        for (int w = 0; w < W; ++w) {
            const Slice<TS, TM> xv = xslice(xia, i, w);
            Slice<TS, TM> out;
            if constexpr (SRC && kPacked) {
                const Slice<TS, TM> sv = slice_from<TS, TM>(lds128(srow + (uint32_t)w * bstride));
                const Slice<TS, TM> zv =
                    hz ? slice_from<TS, TM>(lds128(zrow + (uint32_t)w * bstride)) : Slice<TS, TM>{};
                const float* sgp = a.sig + off + w * wstride;
#pragma unroll
                for (int v = 0; v < V; v += 2) {
                    const float2 sg2 = __ldg(reinterpret_cast<const float2*>(sgp + v));
                    float r0f, r1f;
                    fmul2(a.alpha, a.alpha, acc[w * V + v], acc[w * V + v + 1], r0f, r1f);
                    ffma2(a.beta, a.beta, xv.v[v], xv.v[v + 1], r0f, r1f);
                    if (hz) ffma2(a.gamma, a.gamma, zv.v[v], zv.v[v + 1], r0f, r1f);
                    ffma2(sg2.x, sg2.y, sv.v[v], sv.v[v + 1], r0f, r1f);
                    out.v[v] = r0f;
                    out.v[v + 1] = r1f;
                }
            } else if constexpr (SRC) {
                const Slice<TS, TM> sv = slice_from<TS, TM>(lds128(srow + (uint32_t)w * bstride));
                const Slice<TS, TM> zv =
                    hz ? slice_from<TS, TM>(lds128(zrow + (uint32_t)w * bstride)) : Slice<TS, TM>{};
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    TC r = s_mul(a.alpha, acc[w * V + v]);
                    r = s_fma(a.beta, s_cvt<TC>(xv.v[v]), r);
                    if (hz) r = s_fma(a.gamma, s_cvt<TC>(zv.v[v]), r);
                    r = s_fma(s_from<TC>((double)__ldg(a.sig + off + w * wstride + v), 0.0), s_cvt<TC>(sv.v[v]), r);
                    out.v[v] = s_cvt<TS>(r);
                }
            } else if (hz) {
                const Slice<TS, TM> zv = slice_from<TS, TM>(lds128(zrow + (uint32_t)w * bstride));
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    TC r = s_mul(a.alpha, acc[w * V + v]);
                    r = s_fma(a.beta, s_cvt<TC>(xv.v[v]), r);
                    r = s_fma(a.gamma, s_cvt<TC>(zv.v[v]), r);
                    out.v[v] = s_cvt<TS>(r);
                }
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    TC r = s_mul(a.alpha, acc[w * V + v]);
                    r = s_fma(a.beta, s_cvt<TC>(xv.v[v]), r);
                    out.v[v] = s_cvt<TS>(r);
                }
            }
            stv<TS, TM>(yi + w * wstride, out);
        }
    }
}

}  // namespace rcb

namespace rcb {

// The staged step: two CTAs per SM (each with half the shared memory); the copies of chunk
// t + nstages - 1 are in flight while chunk t is computed. Pol: the stencil policy (unused for CSR,
// IsCsr = true).
template <class Pol, bool IsCsr, class TS, class TC, int W, bool SRC, class TM, class TA>
__global__ void __launch_bounds__(kStagedThreads, 2)
rm_staged_kernel(StagedPlan P, StagedArgs<TM, TC> a, Pol pol) {
    extern __shared__ __align__(128) unsigned char smem[];
    const uint32_t base = smem_u32(smem);
    const int64_t G = gridDim.x;
    const int ns = P.nstages;
    auto stage_of = [&](int64_t t) { return base + (uint32_t)(t % ns) * (uint32_t)P.stage_bytes; };
    auto krange = [&](int64_t c, int32_t& k0, int32_t& k1) {
        if (IsCsr && c < P.nchunks) {
            const int64_t r0 = c * P.R;
            k0 = __ldg(a.rowptr + r0);
            k1 = __ldg(a.rowptr + min(r0 + P.R, a.n));
        }
    };
    // prologue: the first nstages - 1 chunks (one copy group each, empty past the end)
    for (int t = 0; t < ns - 1; ++t) {
        const int64_t c = blockIdx.x + t * G;
        if (c < P.nchunks) {
            int32_t k0 = 0, k1 = 0;
            krange(c, k0, k1);
            staged_issue<TM, TC, TA>(P, a, c, stage_of(t), k0, k1);
        }
        cpasync_commit();
    }
    int32_t nk0 = 0, nk1 = 0;  // the row-pointer range of the next chunk to copy, loaded one chunk ahead
    krange(blockIdx.x + (ns - 1) * G, nk0, nk1);
    for (int64_t t = 0;; ++t) {
        const int64_t c = blockIdx.x + t * G;
        if (c >= P.nchunks) break;
        const int64_t cn = c + (ns - 1) * G;
        if (cn < P.nchunks) staged_issue<TM, TC, TA>(P, a, cn, stage_of(t + ns - 1), nk0, nk1);
        cpasync_commit();
        krange(cn + G, nk0, nk1);
        cpasync_wait(ns - 1);  // this thread's copies of chunk t have landed
        __syncthreads();       // everyone's
        const uint32_t stage = stage_of(t);
        const int64_t r0 = c * P.R;
        if constexpr (IsCsr) {
            const uint32_t rp = stage + (uint32_t)P.rp_off;
            StagedCsr<TA, TC> op{rp, stage + (uint32_t)P.ci_off, stage + (uint32_t)P.va_off, r0, lds32(rp) & ~3};
            staged_compute<StagedCsr<TA, TC>, TS, TC, W, SRC, TM>(P, a, op, r0, stage);
        } else {
            staged_compute<StagedStencil<Pol>, TS, TC, W, SRC, TM>(P, a, StagedStencil<Pol>{pol}, r0, stage);
        }
        __syncthreads();  // stage t % nstages is free for the copies of chunk t + nstages
    }
    cpasync_wait(0);
}

}  // namespace rcb
