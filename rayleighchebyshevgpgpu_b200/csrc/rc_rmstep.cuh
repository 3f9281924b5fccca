// rc_rmstep.cuh -- the degree-step and layout-change arithmetic of the row-major filter.
//
// Device functions shared by the single-solve kernels (rc_filter_rm.cu) and the batched kernels
// that serve several solves in one launch (rc_batch.cu), so both launch forms compute the same
// values in the same order.
#pragma once
#include <cuda_bf16.h>
#include <cstring>
#include <type_traits>
#include "rc_common.cuh"
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

// A 16-byte slice of a block stored as TM, unpacked to the storage type TS of the step arithmetic:
// TM == TS (16/sizeof(TS) values), TM bfloat16 with TS float (8 values; the correction filter's
// real blocks) or TM a bfloat16 pair with TS float2 (4 complex values, real and imaginary part
// each a bfloat16; its complex blocks), rounded to nearest even on store.
template <class TS, class TM = TS>
struct Slice {
    static constexpr int V = 16 / sizeof(TM);
    TS v[V];
};
__device__ __forceinline__ float bf_lo(uint32_t u) { return __uint_as_float(u << 16); }
__device__ __forceinline__ float bf_hi(uint32_t u) { return __uint_as_float(u & 0xffff0000u); }
__device__ __forceinline__ uint32_t bf2_pack(float lo, float hi) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    uint32_t u;
    memcpy(&u, &h, 4);
    return u;
}
template <class TS, class TM>
__device__ __forceinline__ Slice<TS, TM> slice_from(const uint4& u) {
    Slice<TS, TM> r;
    if constexpr (std::is_same<TM, TS>::value) {
        memcpy(&r, &u, 16);
    } else if constexpr (std::is_same<TM, __nv_bfloat162>::value) {
        static_assert(std::is_same<TS, float2>::value, "complex bfloat16 blocks feed c64 steps");
        r.v[0] = make_float2(bf_lo(u.x), bf_hi(u.x));
        r.v[1] = make_float2(bf_lo(u.y), bf_hi(u.y));
        r.v[2] = make_float2(bf_lo(u.z), bf_hi(u.z));
        r.v[3] = make_float2(bf_lo(u.w), bf_hi(u.w));
    } else {
        static_assert(std::is_same<TS, float>::value && std::is_same<TM, __nv_bfloat16>::value,
                      "bfloat16 blocks feed FP32 steps");
        r.v[0] = bf_lo(u.x);
        r.v[1] = bf_hi(u.x);
        r.v[2] = bf_lo(u.y);
        r.v[3] = bf_hi(u.y);
        r.v[4] = bf_lo(u.z);
        r.v[5] = bf_hi(u.z);
        r.v[6] = bf_lo(u.w);
        r.v[7] = bf_hi(u.w);
    }
    return r;
}
template <class TS, class TM>
__device__ __forceinline__ Slice<TS, TM> ldv_ro(const TM* p) {
    return slice_from<TS, TM>(__ldg(reinterpret_cast<const uint4*>(p)));
}
// The same through L2 only (ld.global.cg): for blocks that other CTAs write during the kernel.
template <class TS, class TM>
__device__ __forceinline__ Slice<TS, TM> ldv_cg(const TM* p) {
    return slice_from<TS, TM>(__ldcg(reinterpret_cast<const uint4*>(p)));
}
template <class TS, class TM>
__device__ __forceinline__ Slice<TS, TM> ldv(const TM* p) {
    return slice_from<TS, TM>(*reinterpret_cast<const uint4*>(p));
}
// Blocks that a step reads or writes once (x_{k-2}, the source block, the result) go through the
// caches with the evict-first policy (ld/st .cs), so that the L1 and L2 lines they take are the
// first to go and the rows of x_{k-1}, which the gathers of later rows read again, stay. Measured on
// the 128^3 7-point CSR operator with 96 FP64 columns: the step moves the same DRAM bytes either way
// (3.46 GB read, 1.6 GB written, its algorithmic traffic), but takes 1.04 ms instead of 1.45 ms.
// For bfloat16 blocks (the correction filter) the hints made the step about 1 % slower, so by
// default (RC_STREAM_HINTS 2) only blocks stored in FP64 take them; 1 hints every block, 0 none.
#ifndef RC_STREAM_HINTS
#define RC_STREAM_HINTS 2
#endif
template <class TS, class TM>
constexpr bool stream_hint() {
    return RC_STREAM_HINTS == 1 ||
           (RC_STREAM_HINTS == 2 && std::is_same<TS, TM>::value && sizeof(real_t<TS>) == 8);
}
template <class TS, class TM>
__device__ __forceinline__ Slice<TS, TM> ldv_once(const TM* p) {
    if constexpr (stream_hint<TS, TM>())
        return slice_from<TS, TM>(__ldcs(reinterpret_cast<const uint4*>(p)));
    else
        return slice_from<TS, TM>(*reinterpret_cast<const uint4*>(p));
}
template <class TS, class TM>
__device__ __forceinline__ uint4 slice_pack(const Slice<TS, TM>& v) {
    uint4 u;
    if constexpr (std::is_same<TM, TS>::value) {
        memcpy(&u, &v, 16);
    } else if constexpr (std::is_same<TM, __nv_bfloat162>::value) {
        u.x = bf2_pack(v.v[0].x, v.v[0].y);
        u.y = bf2_pack(v.v[1].x, v.v[1].y);
        u.z = bf2_pack(v.v[2].x, v.v[2].y);
        u.w = bf2_pack(v.v[3].x, v.v[3].y);
    } else {
        u.x = bf2_pack(v.v[0], v.v[1]);
        u.y = bf2_pack(v.v[2], v.v[3]);
        u.z = bf2_pack(v.v[4], v.v[5]);
        u.w = bf2_pack(v.v[6], v.v[7]);
    }
    return u;
}
template <class TS, class TM>
__device__ __forceinline__ void stv(TM* p, const Slice<TS, TM>& v) {
    *reinterpret_cast<uint4*>(p) = slice_pack<TS, TM>(v);
}
template <class TS, class TM>
__device__ __forceinline__ void stv_once(TM* p, const Slice<TS, TM>& v) {
    if constexpr (stream_hint<TS, TM>())
        __stcs(reinterpret_cast<uint4*>(p), slice_pack<TS, TM>(v));
    else
        *reinterpret_cast<uint4*>(p) = slice_pack<TS, TM>(v);
}
// Two FP32 fused multiply-adds in one packed instruction (sm_100 fma.rn.f32x2): c_q = a_q x_q + c_q
// rounded as two fmaf, so the packed and scalar forms give the same bits.
__device__ __forceinline__ void ffma2(float a0, float a1, float x0, float x1, float& c0, float& c1) {
    asm("{\n\t.reg .b64 ra, rx, rc;\n\t"
        "mov.b64 ra, {%2, %3};\n\t"
        "mov.b64 rx, {%4, %5};\n\t"
        "mov.b64 rc, {%0, %1};\n\t"
        "fma.rn.f32x2 rc, ra, rx, rc;\n\t"
        "mov.b64 {%0, %1}, rc;\n\t}"
        : "+f"(c0), "+f"(c1)
        : "f"(a0), "f"(a1), "f"(x0), "f"(x1));
}
__device__ __forceinline__ void fmul2(float a0, float a1, float x0, float x1, float& r0, float& r1) {
    asm("{\n\t.reg .b64 ra, rx, rr;\n\t"
        "mov.b64 ra, {%2, %3};\n\t"
        "mov.b64 rx, {%4, %5};\n\t"
        "mul.rn.f32x2 rr, ra, rx;\n\t"
        "mov.b64 {%0, %1}, rr;\n\t}"
        : "=f"(r0), "=f"(r1)
        : "f"(a0), "f"(a1), "f"(x0), "f"(x1));
}

__device__ __forceinline__ float elem_f(float v) { return v; }
__device__ __forceinline__ float elem_f(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float2 elem_f(float2 v) { return v; }
__device__ __forceinline__ float2 elem_f(__nv_bfloat162 v) { return __bfloat1622float2(v); }

constexpr int kRmThreads = 256;
// Resident CTAs per SM the register budget must allow: 8 (32 registers) for FP32 storage, 6 (40
// registers) for FP64 storage and for the correction step (rm_src_min_blocks), which spills at 32.
// Measured on 128^3 7-point CSR operators with 96 columns: the FP32 step takes 0.52 ms at 8 and
// 0.60 ms at 6; the correction step 0.75 ms at 8 and 0.66 ms at 6; the FP64 step is fastest at 6.
#ifndef RC_RM_MIN_BLOCKS_F32
#define RC_RM_MIN_BLOCKS_F32 8
#endif
#ifndef RC_RM_MIN_BLOCKS_SRC
#define RC_RM_MIN_BLOCKS_SRC 6
#endif
#ifndef RC_RM_MIN_BLOCKS_SRC_BF16
#define RC_RM_MIN_BLOCKS_SRC_BF16 0
#endif
// bfloat16 blocks (8 columns per thread, source coefficients re-read from L1): 6 resident CTAs
// with 32-bit offsets, 5 with 64-bit offsets (which spill at 6), unless the build sets the count.
// Several 16-byte slices per thread (W > 1, the CSR correction step) need more registers: 4 CTAs
// (64 registers), RC_RM_MIN_BLOCKS_SRC_WIDE.
#ifndef RC_RM_MIN_BLOCKS_SRC_WIDE
#define RC_RM_MIN_BLOCKS_SRC_WIDE 4
#endif
template <class TM, class IX, int W = 1>
constexpr int rm_src_min_blocks() {
    return W > 1                         ? RC_RM_MIN_BLOCKS_SRC_WIDE
           : sizeof(TM) != 2             ? RC_RM_MIN_BLOCKS_SRC
           : RC_RM_MIN_BLOCKS_SRC_BF16 > 0 ? RC_RM_MIN_BLOCKS_SRC_BF16
           : sizeof(IX) == 4             ? 6
                                         : 5;
}
#ifndef RC_RM_MIN_BLOCKS_F64
#define RC_RM_MIN_BLOCKS_F64 6
#endif
template <class TS>
constexpr int rm_min_blocks() {
    return sizeof(real_t<TS>) == 4 ? RC_RM_MIN_BLOCKS_F32 : RC_RM_MIN_BLOCKS_F64;
}

// Middle step. Row groups of rows_per_iter consecutive rows; CTA b takes the `groups`
// consecutive groups starting at group b*groups and walks them in order. CTAs are dispatched
// in index order, so the rows in flight at any moment form one contiguous band that moves down
// the block, and a row's far neighbours (i +- band) were read by the band shortly before (an L2
// hit). Thread (r, seg) of a group owns row r's W 16-byte slices seg, seg + nseg, ...,
// seg + (W-1)*nseg (V = 16/sizeof(TM) columns each), so one warp-wide load covers contiguous
// 16-byte slices and the row's index data serve W*V columns. Within a CTA the index data of
// a row are fetched ahead (Pol::fetch1 two groups early, Pol::fetch2 one group early), so
// only the gathers wait on memory.
// IX is the element-offset type: uint32_t when every offset of the block fits, else int64_t.
// pf_z > 0: each 128-byte line of row i + pf_z of x_{k-2} and of row i + pf_x of x_{k-1} (the
// rows first touched from DRAM that many rows later) is prefetched into L2.
// z == nullptr (the first step, gamma = 0): x_{k-2} is not read.
__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// The rows of virtual CTA `cta` (the kernel below passes blockIdx.x; the batched kernel of
// rc_batch.cu passes its own CTA numbering), so one arithmetic serves both launch forms.
// SRC (the correction filter): y also gets sig[c] * src(i, c), where src is a row-major block
// with the same leading dimension and sig holds one coefficient per column (ld entries).
// TM: element type of x, z, y and src in memory (TS, or bfloat16 for FP32 steps).
// ZCG: z is read through L2 only (ld.global.cg), so that no SM holds a line of it in L1 when other
// CTAs of the same kernel overwrite it (the first step of rm_corr2_kernel, whose result the second
// step gathers through the read-only path).
template <class Pol, class TS, class TC, int W, class IX, bool SRC = false, class TM = TS, bool ZCG = false>
__device__ __forceinline__ void rm_step_rows(const Pol& op, int64_t n, int nseg, int64_t ld, int groups, int64_t cta,
                                             const TM* __restrict__ x, const TM* z, TM* y, TC alpha, TC beta,
                                             TC gamma, int64_t pf_z, int64_t pf_x,
                                             const TM* __restrict__ src = nullptr,
                                             const float* __restrict__ sig = nullptr) {
    constexpr int V = Slice<TS, TM>::V;
    const int rows_per_iter = blockDim.x / nseg;
    const int rloc = threadIdx.x / nseg;
    if (rloc >= rows_per_iter) return;
    const IX off = (IX)(threadIdx.x - rloc * nseg) * (IX)V;
    const IX wstride = (IX)nseg * (IX)V;
    const IX ldx = (IX)ld;
    const int64_t stride = rows_per_iter;
    // source coefficients: held in registers, or (bfloat16 blocks, 8 columns per thread, and complex
    // blocks, where registers bound the resident CTAs) re-read from L1 per row
    constexpr bool kSigReg = sizeof(TM) != 2 && !IsComplex<TC>::value;
    // complex FP32 steps of the correction filter: every coefficient is real, so the epilogue
    // works on (re, im) pairs with real scalars (ffma2, fmul2)
    constexpr bool kCplxSrc = SRC && std::is_same<TC, float2>::value;
    // bfloat16 blocks (TS = TC = float): the FP32 arithmetic in packed pairs (ffma2, fmul2)
    constexpr bool kPacked = sizeof(TM) == 2;
    TC sg[SRC && kSigReg ? W * V : 1];
    if (SRC && kSigReg) {
#pragma unroll
        for (int w = 0; w < W; ++w)
#pragma unroll
            for (int v = 0; v < V; ++v) sg[w * V + v] = s_from<TC>((double)__ldg(sig + off + w * wstride + v), 0.0);
    }
    int64_t i = cta * groups * rows_per_iter + rloc;
    const int64_t i_end = min(n, (cta + 1) * groups * rows_per_iter);
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
        const IX oi = (IX)i * ldx + off;
        if (pf_z > 0) {
#pragma unroll
            for (int w = 0; w < W; ++w) {
                if ((((off + w * wstride) * (IX)sizeof(TM)) & 127) != 0) continue;  // one per 128-byte line
                if (z && i + pf_z < n) prefetch_l2(z + (IX)(i + pf_z) * ldx + off + w * wstride);
                if (SRC && i + pf_z < n) prefetch_l2(src + (IX)(i + pf_z) * ldx + off + w * wstride);
                if (i + pf_x < n) prefetch_l2(x + (IX)(i + pf_x) * ldx + off + w * wstride);
            }
        }
        TC acc[W * V];
#pragma unroll
        for (int v = 0; v < W * V; ++v) acc[v] = s_zero(TC());
        op.row(i, p0, [&](int64_t j, TC a) {
            const TM* xj = x + ((IX)j * ldx + off);
#pragma unroll
            for (int w = 0; w < W; ++w) {
                const Slice<TS, TM> p = ldv_ro<TS, TM>(xj + w * wstride);
                if constexpr (kPacked) {
#pragma unroll
                    for (int v = 0; v < V; v += 2)
                        ffma2(a, a, p.v[v], p.v[v + 1], acc[w * V + v], acc[w * V + v + 1]);
                } else {
#pragma unroll
                    for (int v = 0; v < V; ++v) acc[w * V + v] = s_fma(a, s_cvt<TC>(p.v[v]), acc[w * V + v]);
                }
            }
        });
#pragma unroll
        for (int w = 0; w < W; ++w) {
            const IX o = oi + w * wstride;
            const Slice<TS, TM> xi = ldv_ro<TS, TM>(x + o);
            Slice<TS, TM> out;
            if constexpr (SRC && kPacked) {
                const Slice<TS, TM> si = ldv_once<TS, TM>(src + o);
                const Slice<TS, TM> zi =
                    z ? (ZCG ? ldv_cg<TS, TM>(z + o) : ldv_once<TS, TM>(z + o)) : Slice<TS, TM>{};
                const float* sgp = sig + off + w * wstride;
#pragma unroll
                for (int v = 0; v < V; v += 2) {
                    const float2 sg2 = __ldg(reinterpret_cast<const float2*>(sgp + v));
                    float r0, r1;
                    fmul2(alpha, alpha, acc[w * V + v], acc[w * V + v + 1], r0, r1);
                    ffma2(beta, beta, xi.v[v], xi.v[v + 1], r0, r1);
                    if (z) ffma2(gamma, gamma, zi.v[v], zi.v[v + 1], r0, r1);
                    ffma2(sg2.x, sg2.y, si.v[v], si.v[v + 1], r0, r1);
                    out.v[v] = r0;
                    out.v[v + 1] = r1;
                }
            } else if constexpr (kCplxSrc) {
                const Slice<TS, TM> si = ldv_once<TS, TM>(src + o);
                const Slice<TS, TM> zi =
                    z ? (ZCG ? ldv_cg<TS, TM>(z + o) : ldv_once<TS, TM>(z + o)) : Slice<TS, TM>{};
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const float sgv = __ldg(sig + off + w * wstride + v);
                    float r0, r1;
                    fmul2(alpha.x, alpha.x, acc[w * V + v].x, acc[w * V + v].y, r0, r1);
                    ffma2(beta.x, beta.x, xi.v[v].x, xi.v[v].y, r0, r1);
                    if (z) ffma2(gamma.x, gamma.x, zi.v[v].x, zi.v[v].y, r0, r1);
                    ffma2(sgv, sgv, si.v[v].x, si.v[v].y, r0, r1);
                    out.v[v] = make_float2(r0, r1);
                }
            } else if (SRC) {
                const Slice<TS, TM> si = ldv_once<TS, TM>(src + o);
                const Slice<TS, TM> zi =
                    z ? (ZCG ? ldv_cg<TS, TM>(z + o) : ldv_once<TS, TM>(z + o)) : Slice<TS, TM>{};
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    TC r = s_mul(alpha, acc[w * V + v]);
                    r = s_fma(beta, s_cvt<TC>(xi.v[v]), r);
                    if (z) r = s_fma(gamma, s_cvt<TC>(zi.v[v]), r);
                    const TC sgv = kSigReg ? sg[kSigReg ? w * V + v : 0]
                                           : s_from<TC>((double)__ldg(sig + off + w * wstride + v), 0.0);
                    r = s_fma(sgv, s_cvt<TC>(si.v[v]), r);
                    out.v[v] = s_cvt<TS>(r);
                }
            } else if (z) {
                const Slice<TS, TM> zi = ldv_once<TS, TM>(z + o);
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    TC r = s_mul(alpha, acc[w * V + v]);
                    r = s_fma(beta, s_cvt<TC>(xi.v[v]), r);
                    r = s_fma(gamma, s_cvt<TC>(zi.v[v]), r);
                    out.v[v] = s_cvt<TS>(r);
                }
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    TC r = s_mul(alpha, acc[w * V + v]);
                    r = s_fma(beta, s_cvt<TC>(xi.v[v]), r);
                    out.v[v] = s_cvt<TS>(r);
                }
            }
            stv_once<TS, TM>(y + o, out);
        }
        p0 = p1;
        p1 = p2;
    }
}

// The 27-point stencil (every neighbour weight offd) with the box sum reused along x:
//   (A x)_i = (diag_i - offd) x_i + offd S_i,  S_i = Q(i-1) + Q(i) + Q(i+1),
// where Q(j) is the sum of x over the 3x3 cross-section (y, z neighbours, Dirichlet) of row j.
// Each thread walks `run` consecutive rows, so Q(i+1) is the only new cross-section per row:
// 9 gathers per row instead of 27 (the per-row form is bound by L1 throughput). Thread (r, seg)
// of a CTA takes rows cta*rows_per_iter*run + r*run .. + run, the CTA a contiguous range.
// The sums are formed in a different order than rm_step_rows (a rounding-level difference).
template <class TD, class TS, class TC, int W, class IX, bool SRC, class TM = TS>
__device__ __forceinline__ void rm_step_rows27(const StencilRows<TD, TC, 27>& op, int64_t n, int nseg, int64_t ld,
                                               int run, int64_t cta, const TM* __restrict__ x, const TM* z, TM* y,
                                               TC alpha, TC beta, TC gamma, int64_t pf_z, int64_t pf_x,
                                               const TM* __restrict__ src, const float* __restrict__ sig) {
    constexpr int V = Slice<TS, TM>::V;
    const int rows_per_iter = blockDim.x / nseg;
    const int rloc = threadIdx.x / nseg;
    if (rloc >= rows_per_iter) return;
    const IX off = (IX)(threadIdx.x - rloc * nseg) * (IX)V;
    const IX wstride = (IX)nseg * (IX)V;
    const IX ldx = (IX)ld;
    // source coefficients in registers, or (bfloat16 blocks, where registers bound the resident CTAs)
    // re-read from L1 per row
    constexpr bool kSigReg = sizeof(TM) != 2;
    TC sg[SRC && kSigReg ? W * V : 1];
    if (SRC && kSigReg) {
#pragma unroll
        for (int w = 0; w < W; ++w)
#pragma unroll
            for (int v = 0; v < V; ++v) sg[w * V + v] = s_from<TC>((double)__ldg(sig + off + w * wstride + v), 0.0);
    }
    const int64_t nx = op.nx, ny = op.ny, nz = op.nz, sy = nx, sz = nx * ny;
    const TC woff = s_from<TC>(op.offd, 0.0);
    const int64_t i0 = (cta * rows_per_iter + rloc) * (int64_t)run;
    const int64_t i1 = min(n, i0 + run);
    // cross-section sum of row j (same y, z as row i) for this thread's slices
    auto cross = [&](int64_t j, bool vym, bool vyp, bool vzm, bool vzp, TC (&q)[W * V]) {
#pragma unroll
        for (int v = 0; v < W * V; ++v) q[v] = s_zero(TC());
#pragma unroll
        for (int dz = -1; dz <= 1; ++dz) {
            const bool vz = dz < 0 ? vzm : (dz > 0 ? vzp : true);
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy) {
                const bool vy = dy < 0 ? vym : (dy > 0 ? vyp : true);
                if (vz && vy) {
                    const TM* xj = x + ((IX)(j + dy * sy + dz * sz) * ldx + off);
#pragma unroll
                    for (int w = 0; w < W; ++w) {
                        const Slice<TS, TM> pk = ldv_ro<TS, TM>(xj + w * wstride);
#pragma unroll
                        for (int v = 0; v < V; ++v) q[w * V + v] = s_add(q[w * V + v], s_cvt<TC>(pk.v[v]));
                    }
                }
            }
        }
    };
    TC qm[W * V], q0[W * V], qp[W * V];
    for (int64_t i = i0; i < i1; ++i) {
        int64_t ix, iy, iz;
        op.coords(i, ix, iy, iz);
        const bool vym = iy > 0, vyp = iy + 1 < ny, vzm = iz > 0, vzp = iz + 1 < nz;
        if (i == i0 || ix == 0) {  // (re)start the window at the run's first row or a new x-line
            if (ix > 0) cross(i - 1, vym, vyp, vzm, vzp, qm);
            else
#pragma unroll
                for (int v = 0; v < W * V; ++v) qm[v] = s_zero(TC());
            cross(i, vym, vyp, vzm, vzp, q0);
        }
        if (ix + 1 < nx) cross(i + 1, vym, vyp, vzm, vzp, qp);
        else
#pragma unroll
            for (int v = 0; v < W * V; ++v) qp[v] = s_zero(TC());
        const IX oi = (IX)i * ldx + off;
        if (pf_z > 0 && i + pf_z < n) {
#pragma unroll
            for (int w = 0; w < W; ++w) {
                if ((((off + w * wstride) * (IX)sizeof(TM)) & 127) != 0) continue;
                if (z) prefetch_l2(z + (IX)(i + pf_z) * ldx + off + w * wstride);
                if (SRC) prefetch_l2(src + (IX)(i + pf_z) * ldx + off + w * wstride);
                if (i + pf_x < n) prefetch_l2(x + (IX)(i + pf_x) * ldx + off + w * wstride);
            }
        }
        const TC dmw = s_sub(s_from<TC>((double)op.diag[i], 0.0), woff);
#pragma unroll
        for (int w = 0; w < W; ++w) {
            const IX o = oi + w * wstride;
            const Slice<TS, TM> xi = ldv_ro<TS, TM>(x + o);
            Slice<TS, TM> zi{}, si{};
            if (z) zi = ldv_once<TS, TM>(z + o);
            if (SRC) si = ldv_once<TS, TM>(src + o);
            Slice<TS, TM> out;
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int e = w * V + v;
                const TC xv = s_cvt<TC>(xi.v[v]);
                const TC ax = s_fma(woff, s_add(s_add(qm[e], q0[e]), qp[e]), s_mul(dmw, xv));
                TC r = s_mul(alpha, ax);
                r = s_fma(beta, xv, r);
                if (z) r = s_fma(gamma, s_cvt<TC>(zi.v[v]), r);
                if (SRC) {
                    const TC sgv = kSigReg ? sg[kSigReg ? e : 0]
                                           : s_from<TC>((double)__ldg(sig + off + w * wstride + v), 0.0);
                    r = s_fma(sgv, s_cvt<TC>(si.v[v]), r);
                }
                out.v[v] = s_cvt<TS>(r);
            }
            stv_once<TS, TM>(y + o, out);
        }
#pragma unroll
        for (int v = 0; v < W * V; ++v) {
            qm[v] = q0[v];
            q0[v] = qp[v];
        }
    }
}

template <class P> struct IsStencil27 {
    static constexpr bool value = false;
    using diag_t = float;
};
template <class TD, class TC> struct IsStencil27<StencilRows<TD, TC, 27>> {
    static constexpr bool value = true;
    using diag_t = TD;
};
// Consecutive rows per thread in rm_step_rows27 (and the 27-point residual walk). A run starts with
// two extra cross-section sums, so longer runs gather less; the values do not depend on it. Measured
// on the 256^3 27-point stencil with 48 columns (mixed solve): filter phase 3775 / 3633 / 3509 ms and
// Rayleigh-Ritz phase 4951 / 4553 / 4382 ms for runs of 16 / 32 / 64 rows.
#ifndef RC_RUN27
#define RC_RUN27 64
#endif
constexpr int kRun27 = RC_RUN27;

// The same 27-point step with the lanes of a warp on consecutive rows (rm_step27w_kernel), for rows
// of at most kMaxSeg27w 16-byte slices. With RW = 32 / nseg rows per step, lane l < RW * nseg takes
// slice l % nseg of row base + j * RW + l / nseg at step j, so one gather instruction of the warp
// reads RW consecutive rows (RW * nseg * 16 contiguous bytes) instead of rows a run apart. Each lane
// forms P = Q(row + 1), the cross-section sum of the next row with that row's boundary flags; row i
// then takes Q(i+1) from its own P, Q(i) from the lane nseg below and Q(i-1) from the lane 2 nseg
// below, by shuffles. The first two rows of a step take them from the last two rows of the previous
// step, which the warp keeps in shared memory; before the first step the warp forms Q(base) and
// Q(base - 1) itself. A warp walks kSteps27w steps (RW * kSteps27w consecutive rows), the warps of a
// CTA consecutive runs. The sums and their order are rm_step_rows27's, so both give the same bits.
constexpr int kMaxSeg27w = 10;
constexpr int kSteps27w = 16;

template <class TD, class TS, class TC, class IX, bool SRC, class TM = TS>
__device__ __forceinline__ void rm_step_rows27w(const StencilRows<TD, TC, 27>& op, int64_t n, int nseg, int64_t ld,
                                                const TM* __restrict__ x, const TM* z, TM* y, TC alpha, TC beta,
                                                TC gamma, int64_t pf_z, int64_t pf_x, const TM* __restrict__ src,
                                                const float* __restrict__ sig) {
    static_assert(!IsComplex<TC>::value, "the 27-point stencil is real");
    constexpr int V = Slice<TS, TM>::V;
    __shared__ TC carry[kRmThreads / 32][2][kMaxSeg27w][V];  // [warp][0: Q(first-1), 1: Q(first)][slice]
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int RW = 32 / nseg;
    const int rsub = lane / nseg, seg = lane - rsub * nseg;
    const bool act = rsub < RW;
    const IX off = (IX)seg * (IX)V;
    const IX ldx = (IX)ld;
    const int64_t nx = op.nx, ny = op.ny, nz = op.nz, sy = nx, sz = nx * ny;
    const TC woff = s_from<TC>(op.offd, 0.0);
    constexpr bool kSigReg = sizeof(TM) != 2;
    TC sg[SRC && kSigReg ? V : 1];
    if (SRC && kSigReg && act) {
#pragma unroll
        for (int v = 0; v < V; ++v) sg[v] = s_from<TC>((double)__ldg(sig + off + v), 0.0);
    }
    // cross-section sum of row j (over its y, z neighbours; flags of row j) for this lane's slice
    auto cross = [&](int64_t j, bool vym, bool vyp, bool vzm, bool vzp, TC (&q)[V]) {
#pragma unroll
        for (int v = 0; v < V; ++v) q[v] = s_zero(TC());
#pragma unroll
        for (int dz = -1; dz <= 1; ++dz) {
            const bool vz = dz < 0 ? vzm : (dz > 0 ? vzp : true);
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy) {
                const bool vy = dy < 0 ? vym : (dy > 0 ? vyp : true);
                if (vz && vy) {
                    const Slice<TS, TM> pk = ldv_ro<TS, TM>(x + ((IX)(j + dy * sy + dz * sz) * ldx + off));
#pragma unroll
                    for (int v = 0; v < V; ++v) q[v] = s_add(q[v], s_cvt<TC>(pk.v[v]));
                }
            }
        }
    };
    auto cross_at = [&](int64_t j, TC (&q)[V]) {
        int64_t jx, jy, jz;
        op.coords(j, jx, jy, jz);
        cross(j, jy > 0, jy + 1 < ny, jz > 0, jz + 1 < nz, q);
    };
    const int64_t base = ((int64_t)blockIdx.x * (kRmThreads / 32) + wib) * (int64_t)RW * kSteps27w;
    if (base >= n) return;  // the whole warp
    {
        TC q[V];
#pragma unroll
        for (int v = 0; v < V; ++v) q[v] = s_zero(TC());
        if (act && rsub == 0) cross_at(base, q);
        if (act && rsub == 1 && base > 0) cross_at(base - 1, q);
        if (act && rsub <= 1) {
#pragma unroll
            for (int v = 0; v < V; ++v) carry[wib][1 - rsub][seg][v] = q[v];
        }
    }
    __syncwarp();
    const int l1 = lane >= nseg ? lane - nseg : lane;
    const int l2 = lane >= 2 * nseg ? lane - 2 * nseg : lane;
    for (int j = 0; j < kSteps27w; ++j) {
        const int64_t row0 = base + (int64_t)j * RW;
        if (row0 >= n) break;  // the whole warp
        const int64_t i = row0 + rsub;
        const bool live = act && i < n;
        int64_t ix = 0, iy = 0, iz = 0;
        TC P[V];
#pragma unroll
        for (int v = 0; v < V; ++v) P[v] = s_zero(TC());
        if (live) {
            op.coords(i, ix, iy, iz);
            if (i + 1 < n) {
                int64_t jy = iy, jz = iz;
                if (ix + 1 == nx && ++jy == ny) {
                    jy = 0;
                    ++jz;
                }
                cross(i + 1, jy > 0, jy + 1 < ny, jz > 0, jz + 1 < nz, P);
            }
        }
        TC q0[V], qm[V];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            q0[v] = __shfl_sync(0xffffffffu, P[v], l1);
            qm[v] = __shfl_sync(0xffffffffu, P[v], l2);
        }
        if (rsub == 0 && act) {
#pragma unroll
            for (int v = 0; v < V; ++v) {
                q0[v] = carry[wib][1][seg][v];
                qm[v] = carry[wib][0][seg][v];
            }
        } else if (rsub == 1 && act) {
#pragma unroll
            for (int v = 0; v < V; ++v) qm[v] = carry[wib][1][seg][v];
        }
        __syncwarp();  // every lane has read the carries before they are replaced
        if (act && rsub >= RW - 2) {
#pragma unroll
            for (int v = 0; v < V; ++v) carry[wib][rsub - (RW - 2)][seg][v] = P[v];
        }
        __syncwarp();
        if (!live) continue;
        const IX oi = (IX)i * ldx + off;
        if (pf_z > 0 && i + pf_z < n && ((off * (IX)sizeof(TM)) & 127) == 0) {
            if (z) prefetch_l2(z + (IX)(i + pf_z) * ldx + off);
            if (SRC) prefetch_l2(src + (IX)(i + pf_z) * ldx + off);
            if (i + pf_x < n) prefetch_l2(x + (IX)(i + pf_x) * ldx + off);
        }
        const TC dmw = s_sub(s_from<TC>((double)op.diag[i], 0.0), woff);
        const bool hm = ix > 0, hp = ix + 1 < nx;
        const Slice<TS, TM> xi = ldv_ro<TS, TM>(x + oi);
        Slice<TS, TM> zi{}, si{};
        if (z) zi = ldv_once<TS, TM>(z + oi);
        if (SRC) si = ldv_once<TS, TM>(src + oi);
        Slice<TS, TM> out;
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const TC xv = s_cvt<TC>(xi.v[v]);
            const TC qmv = hm ? qm[v] : s_zero(TC()), qpv = hp ? P[v] : s_zero(TC());
            const TC ax = s_fma(woff, s_add(s_add(qmv, q0[v]), qpv), s_mul(dmw, xv));
            TC r = s_mul(alpha, ax);
            r = s_fma(beta, xv, r);
            if (z) r = s_fma(gamma, s_cvt<TC>(zi.v[v]), r);
            if (SRC) {
                const TC sgv = kSigReg ? sg[kSigReg ? v : 0] : s_from<TC>((double)__ldg(sig + off + v), 0.0);
                r = s_fma(sgv, s_cvt<TC>(si.v[v]), r);
            }
            out.v[v] = s_cvt<TS>(r);
        }
        stv_once<TS, TM>(y + oi, out);
    }
}

// Layout change between the caller's column-major FP64 block and the row-major scratch, through
// 32x32 shared-memory tiles (coalesced on both sides), converting precision and scaling.
//   to_rm:  R[i*ld + c] = (TS) V[i + c*ldv]
//   to_cm:  V[i + c*ldv] = scale * R[i*ld + c]
// One 32x32 tile with row origin r0 and column origin c0 (threads 32 x 8).
template <class TV, class TS>
__device__ __forceinline__ void to_rm_tile(int64_t n, int64_t s, const TV* __restrict__ Vc, int64_t ldv,
                                           TS* __restrict__ Rr, int64_t ld, int64_t r0, int64_t c0,
                                           TS (&tile)[32][33]) {
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
__device__ __forceinline__ void to_cm_tile(int64_t n, int64_t s, const TS* __restrict__ Rr, int64_t ld,
                                           TV* __restrict__ Vc, int64_t ldv, double scale, int64_t r0, int64_t c0,
                                           TS (&tile)[32][33]) {
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

// Last step of the correction filter: V[i + c*ldv] = coef[c] * V[i + c*ldv] + beta * E[i*ld + c]
// (x_m = c_m(lambda_c) v_c + a e_m, scaled by 1/(m+1)); one 32x32 tile, threads 32 x 8. Real
// blocks (TM bfloat16 or float, V double) or complex ones (TM a bfloat16 pair or float2, V double2;
// real and imaginary parts each formed as in the real case).
template <class TM>
using CorrTile = decltype(elem_f(TM()));
__device__ __forceinline__ double corr_fma(double c, double v, double b, float e) { return fma(c, v, b * (double)e); }
__device__ __forceinline__ double2 corr_fma(double c, double2 v, double b, float2 e) {
    return make_double2(fma(c, v.x, b * (double)e.x), fma(c, v.y, b * (double)e.y));
}
template <class TM, class TV>
__device__ __forceinline__ void corr_to_cm_tile(int64_t n, int64_t s, const TM* __restrict__ E, int64_t ld,
                                                TV* __restrict__ Vc, int64_t ldv, const double* __restrict__ coef,
                                                double beta, int64_t r0, int64_t c0, CorrTile<TM> (&tile)[32][33]) {
    const int tx = threadIdx.x, ty = threadIdx.y;
    using TT = CorrTile<TM>;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int64_t r = r0 + ty + 8 * j, c = c0 + tx;
        tile[ty + 8 * j][tx] = (r < n && c < s) ? elem_f(E[r * ld + c]) : s_zero(TT());
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int64_t c = c0 + ty + 8 * j, r = r0 + tx;
        if (r < n && c < s) {
            TV* vp = Vc + r + c * ldv;
            *vp = corr_fma(coef[c], *vp, beta, tile[tx][ty + 8 * j]);
        }
    }
}

}  // namespace rcb
