// The templated drop-in interface (include/rc_b200_lmcuda.h) instantiated with the reference's own
// containers and randomize op, compiled from the reference's headers (test infrastructure: built
// into oracle/_ref by oracle/Makefile, never part of the library):
//   rcb200::RayleighChebyshevLMCuda<AmatrixClassLMCuda<double>, AvectorClassLMCuda<double>,
//                                   CusparseCsrOp, ArandomizeOpClassLMCuda<double>, double>
// CusparseCsrOp is an operator of the shape the reference's GPU solver calls: a host single-vector
// apply(AvectorClassLMCuda&) (LanczosMaxMinFinder.h:341) and a device block
// apply(AmatrixClassLMCuda& in, AmatrixClassLMCuda& out, alpha, beta), out = alpha*A*in + beta*out, by
// cuSPARSE SpMM on the containers' own dense-matrix descriptors (AmatrixClassLMCuda.h:82-107;
// LanczosCpolyOperatorLMCuda.h:245). The library reaches it through views of its device blocks
// (BlockAccess: attach mData_d, create_cuda_descriptor, detach).
//
//   lmcuda_reference_containers <problem.bin> k incr buffer tol
// problem.bin: int64 n, int64 nnz, int32 rowptr[n+1], int32 colind[nnz], double vals[nnz].
// Prints one JSON line: eigenvalues, the library's residuals, residuals and orthonormality of the
// returned eigVectors (host mData) recomputed here, and whether mData_d holds the same values.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include <cusparse.h>

#include "AvectorClassLMCuda.h"
#include "AmatrixClassLMCuda.h"
#include "ArandomizeOpClassLMCuda.h"
#include "cusparse_csr_op.h"
#include "rc_b200_lmcuda.h"

using Vec = AvectorClassLMCuda<double>;
using Mat = AmatrixClassLMCuda<double>;

using CusparseCsrOp = CusparseCsrOpT<Vec, Mat>;

static void print_vec(const char* name, const std::vector<double>& x) {
    std::printf("\"%s\": [", name);
    for (size_t i = 0; i < x.size(); ++i) std::printf("%s%.17g", i ? ", " : "", x[i]);
    std::printf("], ");
}

int main(int argc, char** argv) {
    if (argc < 6) {
        std::fprintf(stderr, "usage: %s problem.bin k incr buffer tol\n", argv[0]);
        return 2;
    }
    CusparseCsrOp op;
    {
        FILE* f = std::fopen(argv[1], "rb");
        if (!f) return 3;
        int64_t hdr[2];
        if (std::fread(hdr, 8, 2, f) != 2) return 3;
        op.n = (long)hdr[0];
        op.rp.resize(op.n + 1);
        op.ci.resize(hdr[1]);
        op.v.resize(hdr[1]);
        bool ok = std::fread(op.rp.data(), 4, op.n + 1, f) == (size_t)(op.n + 1);
        ok = ok && std::fread(op.ci.data(), 4, hdr[1], f) == (size_t)hdr[1];
        ok = ok && std::fread(op.v.data(), 8, hdr[1], f) == (size_t)hdr[1];
        std::fclose(f);
        if (!ok) return 3;
    }
    const long k = std::atol(argv[2]), incr = std::atol(argv[3]), buffer = std::atol(argv[4]);
    const double tol = std::atof(argv[5]);
    try {
        op.setup();
        Vec vStart(op.n);
        ArandomizeOpClassLMCuda<double> randOp;
        std::vector<double> evals;
        Mat evecs;
        rcb200::RayleighChebyshevLMCuda<Mat, Vec, CusparseCsrOp, ArandomizeOpClassLMCuda<double>, double> rc;
        rc.setStopCondition("RESIDUAL_ONLY");
        const long found = rc.getMinEigenSystem(k, tol, incr, buffer, vStart, op, randOp, evals, evecs);
        // the returned host block: residuals and orthonormality, recomputed here on the host
        std::vector<double> res(found), col(op.n);
        double orth = 0.0;
        for (long c = 0; c < found; ++c) {
            Vec x(op.n);
            for (long i = 0; i < op.n; ++i) x.vData[i] = evecs(i, c);
            op.apply(x);
            double r2 = 0.0;
            for (long i = 0; i < op.n; ++i) {
                const double d = x.vData[i] - evals[c] * evecs(i, c);
                r2 += d * d;
            }
            res[c] = std::sqrt(r2);
            for (long c2 = 0; c2 <= c; ++c2) {
                double g = 0.0;
                for (long i = 0; i < op.n; ++i) g += evecs(i, c) * evecs(i, c2);
                orth = std::max(orth, std::fabs(g - (c == c2 ? 1.0 : 0.0)));
            }
        }
        // the device copy the container holds after the solve
        std::vector<double> host_copy = evecs.mData;
        bool device_same = evecs.mData_d != nullptr;
        if (device_same) {
            evecs.device_to_host();
            device_same = evecs.mData == host_copy;
        }
        std::printf("{\"found\": %ld, \"rows\": %ld, \"cols\": %ld, ", found, evecs.getRowSize(), evecs.getColSize());
        print_vec("evals", evals);
        print_vec("residuals", rc.getEigVectorResiduals());
        print_vec("host_residuals", res);
        std::printf("\"orthonormality\": %.3e, \"device_copy_matches\": %s, \"apply_calls\": %ld, "
                    "\"lanczos\": %ld, \"bounds\": [%.17g, %.17g]}\n",
                    orth, device_same ? "true" : "false", op.calls, (long)rc.getSpectralBoundsIterCount(),
                    rc.getMinEigValueEst(), rc.getMaxEigValueEst());
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
