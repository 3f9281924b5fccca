// rc_rowops.cuh -- row enumeration of the operators for the filter kernels.
//
// A policy's row(i, f) calls f(j, a_ij) for every stored entry of row i (diagonal included),
// so the same kernel body serves CSR matrices and matrix-free stencils.
#pragma once
#include "rc_common.cuh"

namespace rcb {

// gather<N>(i, js, as): the row's entries as N (column, value) pairs padded with (i, 0), for
// rows with at most N entries (the caller guarantees it). All loads are independent, so the
// kernel can issue the N gathers of a row back to back.
template <class TA, class TC>
struct CsrRows {
    const int32_t* __restrict__ rowptr;
    const int32_t* __restrict__ colind;
    const TA* __restrict__ vals;
    template <class F>
    __device__ __forceinline__ void row(int64_t i, F&& f) const {
        const int k0 = __ldg(rowptr + i), k1 = __ldg(rowptr + i + 1);
#pragma unroll 4
        for (int k = k0; k < k1; ++k) f((int64_t)__ldg(colind + k), s_cvt<TC>(vals[k]));
    }
    template <int N>
    __device__ __forceinline__ void gather(int64_t i, int64_t (&js)[N], TC (&as)[N]) const {
        const int k0 = __ldg(rowptr + i), cnt = __ldg(rowptr + i + 1) - k0;
#pragma unroll
        for (int r = 0; r < N; ++r) {
            const bool ok = r < cnt;
            js[r] = ok ? (int64_t)__ldg(colind + k0 + r) : i;
            as[r] = ok ? s_cvt<TC>(vals[k0 + r]) : s_zero(TC());
        }
    }
};

template <class TC> __device__ __forceinline__ TC unit_phase(double t, bool conj_);
template <> __device__ __forceinline__ double unit_phase<double>(double, bool) { return 1.0; }
template <> __device__ __forceinline__ float unit_phase<float>(double, bool) { return 1.0f; }
template <> __device__ __forceinline__ double2 unit_phase<double2>(double t, bool cj) {
    double sn, cs;
    sincos(t, &sn, &cs);
    return make_double2(cs, cj ? -sn : sn);
}
template <> __device__ __forceinline__ float2 unit_phase<float2>(double t, bool cj) {
    double sn, cs;
    sincos(t, &sn, &cs);
    return make_float2((float)cs, (float)(cj ? -sn : sn));
}

// Dirichlet stencil on nx*ny*nz, i = x + nx*(y + ny*z): diagonal diag[i], every neighbour offd;
// for complex TC the y-bonds carry exp(+i theta x) on (x,y)<-(x,y-1) and its conjugate on
// (x,y)<-(x,y+1). KIND 5 (2D), 7 (3D), 27 (3D, real).
template <class TD, class TC, int KIND>
struct StencilRows {
    int64_t nx, ny, nz;
    const TD* __restrict__ diag;
    double offd;
    double theta;
    template <class F>
    __device__ __forceinline__ void row(int64_t i, F&& f) const {
        const int64_t ix = i % nx;
        const int64_t t = i / nx;
        const int64_t iy = t % ny;
        const int64_t iz = t / ny;
        const int64_t sy = nx, sz = nx * ny;
        f(i, s_from<TC>((double)diag[i], 0.0));
        const TC w = s_from<TC>(offd, 0.0);
        if (KIND == 27) {
#pragma unroll
            for (int dz = -1; dz <= 1; ++dz) {
                const bool vz = dz < 0 ? iz > 0 : (dz > 0 ? iz + 1 < nz : true);
#pragma unroll
                for (int dy = -1; dy <= 1; ++dy) {
                    const bool vy = dy < 0 ? iy > 0 : (dy > 0 ? iy + 1 < ny : true);
#pragma unroll
                    for (int dx = -1; dx <= 1; ++dx) {
                        if (dx == 0 && dy == 0 && dz == 0) continue;
                        const bool vx = dx < 0 ? ix > 0 : (dx > 0 ? ix + 1 < nx : true);
                        if (vx && vy && vz) f(i + dx + dy * sy + dz * sz, w);
                    }
                }
            }
        } else {
            if (KIND == 7 && iz > 0) f(i - sz, w);
            if (IsComplex<TC>::value) {
                if (iy > 0) f(i - sy, s_mul(w, unit_phase<TC>(theta * (double)ix, false)));
            } else {
                if (iy > 0) f(i - sy, w);
            }
            if (ix > 0) f(i - 1, w);
            if (ix + 1 < nx) f(i + 1, w);
            if (IsComplex<TC>::value) {
                if (iy + 1 < ny) f(i + sy, s_mul(w, unit_phase<TC>(theta * (double)ix, true)));
            } else {
                if (iy + 1 < ny) f(i + sy, w);
            }
            if (KIND == 7 && iz + 1 < nz) f(i + sz, w);
        }
    }
    // All entries of row i as N = KIND pairs (diagonal first), invalid neighbours as (i, 0).
    template <int N>
    __device__ __forceinline__ void gather(int64_t i, int64_t (&js)[N], TC (&as)[N]) const {
        static_assert(N == KIND, "stencil gather width must equal its point count");
        const int64_t ix = i % nx;
        const int64_t t = i / nx;
        const int64_t iy = t % ny;
        const int64_t iz = t / ny;
        const int64_t sy = nx, sz = nx * ny;
        const TC w = s_from<TC>(offd, 0.0);
        const TC zero = s_zero(TC());
        js[0] = i;
        as[0] = s_from<TC>((double)diag[i], 0.0);
        if (KIND == 27) {
            int r = 1;
#pragma unroll
            for (int dz = -1; dz <= 1; ++dz) {
                const bool vz = dz < 0 ? iz > 0 : (dz > 0 ? iz + 1 < nz : true);
#pragma unroll
                for (int dy = -1; dy <= 1; ++dy) {
                    const bool vy = dy < 0 ? iy > 0 : (dy > 0 ? iy + 1 < ny : true);
#pragma unroll
                    for (int dx = -1; dx <= 1; ++dx) {
                        if (dx == 0 && dy == 0 && dz == 0) continue;
                        const bool vx = dx < 0 ? ix > 0 : (dx > 0 ? ix + 1 < nx : true);
                        const bool ok = vx && vy && vz;
                        js[r] = ok ? i + dx + dy * sy + dz * sz : i;
                        as[r] = ok ? w : zero;
                        ++r;
                    }
                }
            }
        } else {
            TC wym = w, wyp = w;
            if (IsComplex<TC>::value) {
                wym = s_mul(w, unit_phase<TC>(theta * (double)ix, false));
                wyp = s_mul(w, unit_phase<TC>(theta * (double)ix, true));
            }
            js[1] = ix > 0 ? i - 1 : i;            as[1] = ix > 0 ? w : zero;
            js[2] = ix + 1 < nx ? i + 1 : i;       as[2] = ix + 1 < nx ? w : zero;
            js[3] = iy > 0 ? i - sy : i;           as[3] = iy > 0 ? wym : zero;
            js[4] = iy + 1 < ny ? i + sy : i;      as[4] = iy + 1 < ny ? wyp : zero;
            if (KIND == 7) {
                js[5 % N] = iz > 0 ? i - sz : i;           as[5 % N] = iz > 0 ? w : zero;
                js[6 % N] = iz + 1 < nz ? i + sz : i;      as[6 % N] = iz + 1 < nz ? w : zero;
            }
        }
    }
};

}  // namespace rcb
