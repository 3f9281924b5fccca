// The templated drop-in interface (include/rc_b200_lmcuda.h) driven the way a caller of the
// reference's RayleighChebyshevLMCuda drives it: own vector and matrix containers with the
// reference's members, a randomize op, and three operators on one 2D 5-point problem:
//   stencil  rcb200::StencilOperator (fused kernels)
//   csr      rcb200::CsrOperator<double> (fused kernels)
//   foreign  an operator with only a device block apply(in, out, alpha, beta) on the containers
// Prints one JSON line per operator with the eigenvalues, residuals and solver counters.
#include <cmath>
#include <cstdio>
#include <random>
#include <string>
#include <vector>
#include "rc_b200_lmcuda.h"

template <class T>
struct Vec {  // the members of AvectorClassLMCuda the interface uses
    std::vector<T> vData;
    Vec() = default;
    explicit Vec(long n) : vData((size_t)n) {}
    long getDimension() const { return (long)vData.size(); }
};

template <class T>
struct Mat {  // the members of AmatrixClassLMCuda the interface uses (column-major m x n)
    long m = 0, n = 0;
    std::vector<T> mData;
    T* mData_d = nullptr;
    void resize(long r, long c) {
        m = r;
        n = c;
        mData.assign((size_t)r * c, T());
    }
    long getColSize() const { return n; }
};

struct Rand {  // uniform [-1, 1] draws, like ArandomizeOpClassLMCuda
    std::mt19937_64 g{3141592};
    std::uniform_real_distribution<double> u{-1.0, 1.0};
    void randomize(Vec<double>& v) {
        for (auto& x : v.vData) x = u(g);
    }
    void randomize(Mat<double>& M) {
        for (auto& x : M.mData) x = u(g);
    }
};

__global__ void csr_block_apply(long n, long s, const int* rp, const int* ci, const double* v, const double* x,
                                double* y, double alpha, double beta) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (long c = 0; c < s; ++c) {
        double acc = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) acc += v[k] * x[ci[k] + c * n];
        y[i + c * n] = alpha * acc + beta * y[i + c * n];
    }
}

struct ForeignCsr {  // only the reference's device block apply
    long n = 0;
    int *rp = nullptr, *ci = nullptr;
    double* v = nullptr;
    void apply(Mat<double>& in, Mat<double>& out, double alpha, double beta) {
        csr_block_apply<<<(unsigned)((n + 255) / 256), 256>>>(n, in.n, rp, ci, v, in.mData_d, out.mData_d, alpha,
                                                               beta);
    }
};

template <class Op>
static void run(const char* name, Op& op, long n, int k) {
    rcb200::RayleighChebyshevLMCuda<Mat<double>, Vec<double>, Op, Rand, double> rc;
    rc.setStopCondition("RESIDUAL_ONLY");
    rc.setStopCondition(rcb200::RC_Types::RESIDUAL_ONLY);  // the enum form, same condition
    rc.setUseJacobi(true);                                  // host-implementation switches: no effect
    rc.setVerboseSubspaceFlag(false);
    rc.setEigDiagnosticsFlag(false);
    rc.setFixedIterationCount(false);
    Vec<double> vStart(n);
    Rand rnd;
    std::vector<double> evals;
    Mat<double> evecs;
    const long found = rc.getMinEigenSystem(k, 1.0e-10, k, 8, vStart, op, rnd, evals, evecs);
    const auto res = rc.getEigVectorResiduals();
    const auto counts = rc.getCountData();
    std::printf("{\"op\": \"%s\", \"found\": %ld, \"cols\": %ld, \"evals\": [", name, found, evecs.n);
    for (long i = 0; i < found; ++i) std::printf("%s%.17g", i ? ", " : "", evals[i]);
    std::printf("], \"residuals\": [");
    for (long i = 0; i < found; ++i) std::printf("%s%.6g", i ? ", " : "", res[i]);
    std::printf("], \"opapply\": %ld, \"evec0\": [%.17g, %.17g], \"bounds\": [%.17g, %.17g], \"lanczos\": %ld}\n",
                (long)counts.at("OpApply"), evecs.mData[0], evecs.mData[1], rc.getMinEigValueEst(),
                rc.getMaxEigValueEst(), (long)rc.getSpectralBoundsIterCount());
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
    ForeignCsr fo;
    fo.n = n;
    cudaMalloc(&fo.rp, csr.rowptr.size() * sizeof(int));
    cudaMalloc(&fo.ci, csr.colind.size() * sizeof(int));
    cudaMalloc(&fo.v, csr.vals.size() * sizeof(double));
    cudaMemcpy(fo.rp, csr.rowptr.data(), csr.rowptr.size() * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(fo.ci, csr.colind.data(), csr.colind.size() * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(fo.v, csr.vals.data(), csr.vals.size() * sizeof(double), cudaMemcpyHostToDevice);
    try {
        run("stencil", st, n, k);
        run("csr", csr, n, k);
        run("foreign", fo, n, k);
    } catch (const std::exception& e) {
        std::printf("{\"error\": \"%s\"}\n", e.what());
        return 1;
    }
    cudaFree(fo.rp);
    cudaFree(fo.ci);
    cudaFree(fo.v);
    return 0;
}
