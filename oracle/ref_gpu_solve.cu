// The reference's own FP64 GPU solver, RayleighChebyshevLMCuda (RayleighChebyshevLMCuda.h:220-2472),
// timed on one problem: built by oracle/Makefile from the reference's headers and cuda_kernels.cu where
// they lie, with -DRAY_INT=long -DTIMING_, the SCC LapackInterface stand-in of oracle/shim (LAPACK
// dsyev / zhpevx from scipy's OpenBLAS) and the cuSPARSE CSR operator of tests/cpp/cusparse_csr_op.h.
// Test infrastructure (a baseline): the library never links or runs it.
//
//   ref_gpu_solve <problem.bin> k incr buffer tol [repeats]
// problem.bin: the RCPB file of oracle/ref_io.write_problem (CSR, start block, optional Lanczos
// vector, unused here: the reference's bounds start from its own randomize op). The start block is
// passed as eigVectors with setNonRandomStartFlag (RayleighChebyshevLMCuda.h:1044-1070). Prints one
// JSON line: found, eigenvalues, the wall time of each solve (device synchronised before and after),
// and the reference's own TIMING_ buckets and count data of the last solve.
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <map>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <cusparse.h>

// the reference's headers rely on the standard headers above being included first
#include "AvectorClassLMCuda.h"
#include "AmatrixClassLMCuda.h"
#include "ArandomizeOpClassLMCuda.h"
#include "RayleighChebyshevLMCuda.h"
#include "cusparse_csr_op.h"

using Vec = AvectorClassLMCuda<double>;
using Mat = AmatrixClassLMCuda<double>;
using Op = CusparseCsrOpT<Vec, Mat>;

struct ProblemFile {
    int64_t n = 0, nnz = 0, s = 0, has_lz0 = 0;
    std::vector<int> rp, ci;
    std::vector<double> v, start;
};

static bool read_problem(const char* path, ProblemFile& P) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    char magic[4];
    int32_t ver = 0;
    int64_t hdr[4];
    bool ok = std::fread(magic, 1, 4, f) == 4 && std::memcmp(magic, "RCPB", 4) == 0 && std::fread(&ver, 4, 1, f) == 1 &&
              ver == 1 && std::fread(hdr, 8, 4, f) == 4;
    if (ok) {
        P.n = hdr[0];
        P.nnz = hdr[1];
        P.s = hdr[2];
        P.has_lz0 = hdr[3];
        P.rp.resize(P.n + 1);
        P.ci.resize(P.nnz);
        P.v.resize(P.nnz);
        P.start.resize((size_t)P.n * P.s);
        ok = std::fread(P.rp.data(), 4, P.n + 1, f) == (size_t)(P.n + 1) &&
             std::fread(P.ci.data(), 4, P.nnz, f) == (size_t)P.nnz && std::fread(P.v.data(), 8, P.nnz, f) == (size_t)P.nnz &&
             std::fread(P.start.data(), 8, P.start.size(), f) == P.start.size();
    }
    std::fclose(f);
    return ok;
}

int main(int argc, char** argv) {
    if (argc < 6) {
        std::fprintf(stderr, "usage: %s problem.bin k incr buffer tol [repeats]\n", argv[0]);
        return 2;
    }
    ProblemFile P;
    if (!read_problem(argv[1], P)) {
        std::fprintf(stderr, "cannot read %s\n", argv[1]);
        return 3;
    }
    const long k = std::atol(argv[2]), incr = std::atol(argv[3]), buffer = std::atol(argv[4]);
    const double tol = std::atof(argv[5]);
    const int repeats = argc > 6 ? std::atoi(argv[6]) : 1;
    const long s = incr + buffer;
    if (P.s < s) {
        std::fprintf(stderr, "the problem file holds %ld start columns, the block needs %ld\n", (long)P.s, s);
        return 3;
    }
    try {
        Op op;
        op.n = (long)P.n;
        op.rp = P.rp;
        op.ci = P.ci;
        op.v = P.v;
        op.setup();
        std::vector<double> walls, evals;
        std::map<std::string, double> timing;
        std::map<std::string, RAY_INT> counts;
        long found = 0;
        for (int r = 0; r < repeats; ++r) {
            Vec vStart(op.n);
            ArandomizeOpClassLMCuda<double> randOp;
            Mat ev;
            ev.resize(op.n, s);
            for (long j = 0; j < s; ++j)
                for (long i = 0; i < op.n; ++i) ev(i, j) = P.start[(size_t)j * op.n + i];
            ev.host_to_device();
            RayleighChebyshevLMCuda<Mat, Vec, Op, ArandomizeOpClassLMCuda<double>, double> rc;
            rc.setStopCondition("RESIDUAL_ONLY");
            rc.setNonRandomStartFlag(true);
            evals.clear();
            cudaDeviceSynchronize();
            const auto t0 = std::chrono::steady_clock::now();
            found = (long)rc.getMinEigenSystem(k, tol, incr, buffer, vStart, op, randOp, evals, ev);
            cudaDeviceSynchronize();
            const auto t1 = std::chrono::steady_clock::now();
            walls.push_back(std::chrono::duration<double>(t1 - t0).count());
            timing = rc.getTimingData();
            counts = rc.getCountData();
        }
        std::printf("{\"found\": %ld, \"evals\": [", found);
        for (size_t i = 0; i < evals.size(); ++i) std::printf("%s%.17g", i ? ", " : "", evals[i]);
        std::printf("], \"wall_s\": [");
        for (size_t i = 0; i < walls.size(); ++i) std::printf("%s%.6f", i ? ", " : "", walls[i]);
        std::printf("], \"timing\": {");
        bool first = true;
        for (auto& kv : timing) {
            std::printf("%s\"%s\": %.6f", first ? "" : ", ", kv.first.c_str(), kv.second);
            first = false;
        }
        std::printf("}, \"counts\": {");
        first = true;
        for (auto& kv : counts) {
            std::printf("%s\"%s\": %ld", first ? "" : ", ", kv.first.c_str(), (long)kv.second);
            first = false;
        }
        std::printf("}, \"apply_calls\": %ld}\n", op.calls);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
