// Stand-in for SCC::ZHPEVX (see SCC_LapackMatrix.h): all eigenpairs of a complex Hermitian matrix by
// LAPACK zhpevx on its packed upper triangle (jobz = 'V', range = 'A'), eigenvalues ascending,
// eigenvectors as columns, the call the reference makes at RayleighChebyshevLMCuda.h:618.
#pragma once
#include <complex>
#include <stdexcept>
#include <vector>
#include "SCC_LapackMatrixCmplx16.h"

extern "C" void scipy_zhpevx_(const char* jobz, const char* range, const char* uplo, const int* n,
                              std::complex<double>* ap, const double* vl, const double* vu, const int* il,
                              const int* iu, const double* abstol, int* m, double* w, std::complex<double>* z,
                              const int* ldz, std::complex<double>* work, double* rwork, int* iwork, int* ifail,
                              int* info, size_t, size_t, size_t);

namespace SCC {

class ZHPEVX {
public:
    void createEigensystem(LapackMatrixCmplx16& A, std::vector<double>& evals, LapackMatrixCmplx16& evecs) {
        const int n = (int)A.getRowDimension();
        std::vector<std::complex<double>> ap((size_t)n * (n + 1) / 2);
        size_t p = 0;
        for (int j = 0; j < n; ++j)
            for (int i = 0; i <= j; ++i) ap[p++] = A(i, j);
        evecs.initialize(n, n);
        evals.assign(n, 0.0);
        std::vector<std::complex<double>> work(2 * (size_t)n);
        std::vector<double> rwork(7 * (size_t)n);
        std::vector<int> iwork(5 * (size_t)n), ifail(n);
        const double vl = 0.0, vu = 0.0, abstol = 0.0;
        const int il = 1, iu = n;
        int m = 0, info = 0;
        scipy_zhpevx_("V", "A", "U", &n, ap.data(), &vl, &vu, &il, &iu, &abstol, &m, evals.data(),
                      evecs.getDataPointer(), &n, work.data(), rwork.data(), iwork.data(), ifail.data(), &info, 1, 1,
                      1);
        if (info != 0 || m != n) throw std::runtime_error("zhpevx failed");
    }
};

}  // namespace SCC
