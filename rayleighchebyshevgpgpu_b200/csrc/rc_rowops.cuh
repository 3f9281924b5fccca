// rc_rowops.cuh -- row enumeration of the operators for the filter kernels.
//
// A policy's row(i, f) calls f(j, a_ij) for every stored entry of row i (diagonal included),
// so the same kernel body serves CSR matrices and matrix-free stencils.
#pragma once
#include "rc_common.cuh"

namespace rcb {

// Index data fetched ahead of use. A kernel that walks rows calls fetch1 for a row two
// iterations before it is processed and fetch2 one iteration before, so loads that feed the
// gather addresses are off the critical path:
//   fetch1(i, p): loads that need only i (CSR: the row's extent from rowptr)
//   fetch2(i, p): loads that need fetch1's result (none for the policies here)
//   row(i, p, f): f(j, a_ij) for every entry (CSR: column indices and values loaded here, four
//                 entries unrolled so their gathers overlap)
template <class TA, class TC>
struct CsrRows {
    static constexpr bool kIsCsr = true;
    using value_t = TA;
    const int32_t* __restrict__ rowptr;
    const int32_t* __restrict__ colind;
    const TA* __restrict__ vals;
    struct Pre {
        int k0, k1;
    };
    __device__ __forceinline__ void fetch1(int64_t i, Pre& p) const {
        p.k0 = __ldg(rowptr + i);
        p.k1 = __ldg(rowptr + i + 1);
    }
    __device__ __forceinline__ void fetch2(int64_t, Pre&) const {}
    template <class F>
    __device__ __forceinline__ void row(int64_t, const Pre& p, F&& f) const {
#pragma unroll 4
        for (int k = p.k0; k < p.k1; ++k) f((int64_t)__ldg(colind + k), s_cvt<TC>(__ldg(vals + k)));
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
    static constexpr bool kIsCsr = false;
    int64_t nx, ny, nz;
    const TD* __restrict__ diag;
    double offd;
    double theta;
    const TC* ph = nullptr;  // complex: phase table exp(i theta x), x < nx (else evaluated per row)
    RowDiv dx, dy;           // division by nx and ny (grids of fewer than 2^32 points)
    RC_HD StencilRows(int64_t nx_, int64_t ny_, int64_t nz_, const TD* diag_, double offd_, double theta_)
        : nx(nx_), ny(ny_), nz(nz_), diag(diag_), offd(offd_), theta(theta_), dx(nx_), dy(ny_) {}
    // grid coordinates of row i
    __device__ __forceinline__ void coords(int64_t i, int64_t& ix, int64_t& iy, int64_t& iz) const {
        const int64_t t = dx.div(i);
        ix = i - t * nx;
        iz = dy.div(t);
        iy = t - iz * ny;
    }
    template <class F>
    __device__ __forceinline__ void row(int64_t i, F&& f) const {
        int64_t ix, iy, iz;
        coords(i, ix, iy, iz);
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
            TC p = s_zero(TC());
            if (IsComplex<TC>::value) p = ph ? ph[ix] : unit_phase<TC>(theta * (double)ix, false);
            if (IsComplex<TC>::value) {
                if (iy > 0) f(i - sy, s_mul(w, p));
            } else {
                if (iy > 0) f(i - sy, w);
            }
            if (ix > 0) f(i - 1, w);
            if (ix + 1 < nx) f(i + 1, w);
            if (IsComplex<TC>::value) {
                if (iy + 1 < ny) f(i + sy, s_mul(w, s_conj(p)));
            } else {
                if (iy + 1 < ny) f(i + sy, w);
            }
            if (KIND == 7 && iz + 1 < nz) f(i + sz, w);
        }
    }
    struct Pre {};
    __device__ __forceinline__ void fetch1(int64_t, Pre&) const {}
    __device__ __forceinline__ void fetch2(int64_t, Pre&) const {}
    template <class F>
    __device__ __forceinline__ void row(int64_t i, const Pre&, F&& f) const {
        row(i, f);
    }
};

}  // namespace rcb
