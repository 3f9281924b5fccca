// rc_common.cuh -- scalar traits and small device helpers shared by the kernels.
//
// Scalars: double (real FP64), float (real FP32 filter storage), double2 (c128, the layout of
// std::complex<double>) and float2 (c64). Complex values are interleaved (re, im).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define RC_HD __host__ __device__ __forceinline__

// ---- real part type ------------------------------------------------------------------
template <class T> struct RealOf;
template <> struct RealOf<double> { using type = double; };
template <> struct RealOf<float> { using type = float; };
template <> struct RealOf<double2> { using type = double; };
template <> struct RealOf<float2> { using type = float; };
template <class T> using real_t = typename RealOf<T>::type;

template <class T> struct IsComplex { static constexpr bool value = false; };
template <> struct IsComplex<double2> { static constexpr bool value = true; };
template <> struct IsComplex<float2> { static constexpr bool value = true; };

// ---- arithmetic ----------------------------------------------------------------------
RC_HD double s_zero(double) { return 0.0; }
RC_HD float s_zero(float) { return 0.0f; }
RC_HD double2 s_zero(double2) { return make_double2(0.0, 0.0); }
RC_HD float2 s_zero(float2) { return make_float2(0.0f, 0.0f); }

RC_HD double s_add(double a, double b) { return a + b; }
RC_HD float s_add(float a, float b) { return a + b; }
RC_HD double2 s_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
RC_HD float2 s_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }

RC_HD double s_sub(double a, double b) { return a - b; }
RC_HD float s_sub(float a, float b) { return a - b; }
RC_HD double2 s_sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
RC_HD float2 s_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

RC_HD double s_mul(double a, double b) { return a * b; }
RC_HD float s_mul(float a, float b) { return a * b; }
RC_HD double2 s_mul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
RC_HD float2 s_mul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }

// a*b + c
RC_HD double s_fma(double a, double b, double c) { return fma(a, b, c); }
RC_HD float s_fma(float a, float b, float c) { return fmaf(a, b, c); }
RC_HD double2 s_fma(double2 a, double2 b, double2 c) {
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
RC_HD float2 s_fma(float2 a, float2 b, float2 c) {
    return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
}
// conj(a)*b + c
RC_HD double s_cfma(double a, double b, double c) { return fma(a, b, c); }
RC_HD double2 s_cfma(double2 a, double2 b, double2 c) {
    return make_double2(fma(a.x, b.x, fma(a.y, b.y, c.x)), fma(a.x, b.y, fma(-a.y, b.x, c.y)));
}
// real * scalar
RC_HD double s_rscale(double r, double a) { return r * a; }
RC_HD float s_rscale(float r, float a) { return r * a; }
RC_HD double2 s_rscale(double r, double2 a) { return make_double2(r * a.x, r * a.y); }
RC_HD float2 s_rscale(float r, float2 a) { return make_float2(r * a.x, r * a.y); }

RC_HD double s_conj(double a) { return a; }
RC_HD double2 s_conj(double2 a) { return make_double2(a.x, -a.y); }
RC_HD float s_conj(float a) { return a; }
RC_HD float2 s_conj(float2 a) { return make_float2(a.x, -a.y); }
RC_HD double s_abs2(double a) { return a * a; }
RC_HD float s_abs2(float a) { return a * a; }
RC_HD double s_abs2(double2 a) { return a.x * a.x + a.y * a.y; }
RC_HD float s_abs2(float2 a) { return a.x * a.x + a.y * a.y; }
RC_HD double s_real(double a) { return a; }
RC_HD double s_real(double2 a) { return a.x; }
RC_HD double s_imag(double) { return 0.0; }
RC_HD double s_imag(double2 a) { return a.y; }

// ---- conversions between storage and compute types ----------------------------------
template <class To> RC_HD To s_cvt(double a);
template <class To> RC_HD To s_cvt(float a);
template <class To> RC_HD To s_cvt(double2 a);
template <class To> RC_HD To s_cvt(float2 a);
template <> RC_HD double s_cvt<double>(double a) { return a; }
template <> RC_HD float s_cvt<float>(double a) { return (float)a; }
template <> RC_HD double s_cvt<double>(float a) { return (double)a; }
template <> RC_HD float s_cvt<float>(float a) { return a; }
template <> RC_HD double2 s_cvt<double2>(double2 a) { return a; }
template <> RC_HD float2 s_cvt<float2>(double2 a) { return make_float2((float)a.x, (float)a.y); }
template <> RC_HD double2 s_cvt<double2>(float2 a) { return make_double2((double)a.x, (double)a.y); }
template <> RC_HD float2 s_cvt<float2>(float2 a) { return a; }

// scalar from (re, im) pair of doubles
template <class T> RC_HD T s_from(double re, double im);
template <> RC_HD double s_from<double>(double re, double) { return re; }
template <> RC_HD float s_from<float>(double re, double) { return (float)re; }
template <> RC_HD double2 s_from<double2>(double re, double im) { return make_double2(re, im); }
template <> RC_HD float2 s_from<float2>(double re, double im) { return make_float2((float)re, (float)im); }

// ---- division of row indices by a fixed grid extent ----------------------------------
// floor(i / d) for 0 <= i < 2^32 and 1 <= d < 2^32 as the high 64 bits of i * m, m = ceil(2^64 / d):
// with m d = 2^64 + e, 0 <= e < d, the product is i/d + i e / (d 2^64) and i e < 2^64, so the
// floor is exact. One 64-bit multiply-high instead of a 64-bit division per row.
struct RowDiv {
    uint64_t m = 0;  // 0 for d == 1
    RC_HD RowDiv() {}
    RC_HD explicit RowDiv(int64_t d) : m(d > 1 ? ~0ull / (uint64_t)d + 1 : 0) {}
    __device__ __forceinline__ int64_t div(int64_t i) const {
        return m ? (int64_t)__umul64hi((uint64_t)i, m) : i;
    }
};

// ---- reductions ----------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double2 warp_sum(double2 v) {
    v.x = warp_sum(v.x);
    v.y = warp_sum(v.y);
    return v;
}

// Block-wide sum (blockDim.x a multiple of 32, <= 1024). All threads get the result.
template <class T>
__device__ T block_sum(T v, T* scratch /* >= 32 entries */) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    T t = s_zero(T());
    if (wid == 0) {
        t = lane < nw ? scratch[lane] : s_zero(T());
        t = warp_sum(t);
        if (lane == 0) scratch[0] = t;
    }
    __syncthreads();
    t = scratch[0];
    __syncthreads();
    return t;
}

// Numbers of SMs of the B200 (2 dies x 74); grids are sized in multiples of it.
constexpr int kB200Sms = 148;
