// The per-vector drop-in interface (include/rc_b200_rc.h) driven the way a caller of the reference's
// CPU RayleighChebyshev<Vtype, Otype, VRandomizeOpType> drives it: a vector class with the reference's
// Vtype members (RayleighChebyshev.h:26-40), a randomize op, eigenvectors returned as
// std::vector<Vtype>, and three operators on one 2D 5-point problem:
//   stencil  rcb200::StencilOperator (fused kernels)
//   csr      rcb200::CsrOperator<double> (fused kernels)
//   host     an operator with only the reference's in-place host apply(Vtype&)
// Host C++ only: it links against the library and never includes CUDA code of its own.
// Prints one JSON line per operator with the eigenvalues, residuals and counters.
#include <cmath>
#include <cstdio>
#include <random>
#include <string>
#include <vector>
#include "rc_b200_rc.h"

struct Vec {  // the Vtype contract of RayleighChebyshev.h, values in the public std::vector vData
    std::vector<double> vData;
    Vec() = default;
    explicit Vec(long n) : vData((size_t)n) {}
    Vec(const Vec&) = default;
    void initialize() { vData.clear(); }
    void initialize(const Vec& v) { vData = v.vData; }
    Vec& operator=(const Vec&) = default;
    Vec& operator+=(const Vec& v) {
        for (size_t i = 0; i < vData.size(); ++i) vData[i] += v.vData[i];
        return *this;
    }
    Vec& operator-=(const Vec& v) {
        for (size_t i = 0; i < vData.size(); ++i) vData[i] -= v.vData[i];
        return *this;
    }
    Vec& operator*=(double a) {
        for (auto& x : vData) x *= a;
        return *this;
    }
    double dot(const Vec& v) const {
        double s = 0.0;
        for (size_t i = 0; i < vData.size(); ++i) s += vData[i] * v.vData[i];
        return s;
    }
    long getDimension() const { return (long)vData.size(); }
};

struct Rand {  // uniform [-1, 1] draws
    std::mt19937_64 g{3141592};
    std::uniform_real_distribution<double> u{-1.0, 1.0};
    void randomize(Vec& v) {
        for (auto& x : v.vData) x = u(g);
    }
};

struct HostLaplacian {  // only the reference's in-place host apply: v <- A v
    long nx = 0, ny = 0;
    const std::vector<double>* diag = nullptr;
    std::vector<double> tmp;
    void apply(Vec& v) {
        const long n = nx * ny;
        tmp.assign(v.vData.begin(), v.vData.end());
        for (long i = 0; i < n; ++i) {
            const long x = i % nx, y = i / nx;
            double r = (*diag)[i] * tmp[i];
            if (y > 0) r -= tmp[i - nx];
            if (x > 0) r -= tmp[i - 1];
            if (x + 1 < nx) r -= tmp[i + 1];
            if (y + 1 < ny) r -= tmp[i + nx];
            v.vData[i] = r;
        }
    }
};

template <class Op>
static void run(const char* name, Op& op, long n, int k) {
    rcb200::RayleighChebyshev<Vec, Op, Rand, double> rc;
    rc.setStopCondition("residual_only");
    rc.setStopCondition(rcb200::RC_Types::RESIDUAL_ONLY);  // the enum form, same condition
    rc.setUseJacobi(true);                                  // CPU-implementation switches: no effect
    rc.setVerboseSubspaceFlag(false);
    rc.setEigDiagnosticsFlag(false);
    rc.setIntervalStopCondition(false);
    Vec vStart(n);
    Rand rnd;
    std::vector<double> evals;
    std::vector<Vec> evecs;
    const long found = rc.getMinEigenSystem(k, 1.0e-10, k, 8, vStart, op, rnd, evals, evecs);
    const auto res = rc.getEigVectorResiduals();
    const auto counts = rc.getCountData();
    double orth = 0.0;  // largest |<v_i, v_j> - delta_ij| over the returned vectors
    for (long i = 0; i < found; ++i)
        for (long j = 0; j < found; ++j) orth = std::fmax(orth, std::fabs(evecs[i].dot(evecs[j]) - (i == j)));
    std::printf("{\"op\": \"%s\", \"found\": %ld, \"vectors\": %zu, \"dim\": %ld, \"evals\": [", name, found,
                evecs.size(), found > 0 ? evecs[0].getDimension() : 0L);
    for (long i = 0; i < found; ++i) std::printf("%s%.17g", i ? ", " : "", evals[i]);
    std::printf("], \"residuals\": [");
    for (long i = 0; i < found; ++i) std::printf("%s%.6g", i ? ", " : "", res[i]);
    std::printf("], \"orth\": %.3g, \"opapply\": %ld, \"bounds\": [%.17g, %.17g], \"lanczos\": %ld}\n", orth,
                (long)counts.at("OpApply"), rc.getMinEigValueEst(), rc.getMaxEigValueEst(),
                rc.getSpectralBoundsIterCount());
}

int main() {
    const long nx = 48, ny = 40, n = nx * ny;
    const int k = 8;
    std::vector<double> diag((size_t)n);
    for (long i = 0; i < n; ++i) diag[i] = 4.0 + 0.5 * (1.0 + std::sin(0.7 * (double)i));
    rcb200::CsrOperator<double> csr;
    csr.n = n;
    csr.rowptr.push_back(0);
    for (long i = 0; i < n; ++i) {
        const long x = i % nx, y = i / nx;
        auto add = [&](long j, double a) {
            csr.colind.push_back((int)j);
            csr.vals.push_back(a);
        };
        if (y > 0) add(i - nx, -1.0);
        if (x > 0) add(i - 1, -1.0);
        add(i, diag[i]);
        if (x + 1 < nx) add(i + 1, -1.0);
        if (y + 1 < ny) add(i + nx, -1.0);
        csr.rowptr.push_back((int)csr.colind.size());
    }
    rcb200::StencilOperator st;
    st.kind = RC_STENCIL_5PT_2D;
    st.nx = nx;
    st.ny = ny;
    st.nz = 1;
    st.diag = diag;
    st.offdiag = -1.0;
    HostLaplacian host;
    host.nx = nx;
    host.ny = ny;
    host.diag = &diag;
    try {
        run("stencil", st, n, k);
        run("csr", csr, n, k);
        run("host", host, n, k);
    } catch (const std::exception& e) {
        std::printf("{\"error\": \"%s\"}\n", e.what());
        return 1;
    }
    return 0;
}
