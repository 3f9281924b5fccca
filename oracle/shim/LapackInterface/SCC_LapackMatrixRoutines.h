// Stand-in for SCC::DSYEV (see SCC_LapackMatrix.h): all eigenpairs of a real symmetric matrix by
// LAPACK dsyev (jobz = 'V', uplo = 'U'), eigenvalues ascending, eigenvectors as columns, the call
// the reference makes at RayleighChebyshevLMCuda.h:614. LAPACK comes from the OpenBLAS that scipy
// bundles (its exported routines carry a scipy_ prefix); oracle/Makefile links it.
#pragma once
#include <stdexcept>
#include <vector>
#include "SCC_LapackMatrix.h"

extern "C" void scipy_dsyev_(const char* jobz, const char* uplo, const int* n, double* a, const int* lda, double* w,
                             double* work, const int* lwork, int* info, size_t, size_t);

namespace SCC {

class DSYEV {
public:
    void computeEigensystem(LapackMatrix& A, std::vector<double>& evals, LapackMatrix& evecs) {
        const int n = (int)A.getRowDimension();
        evecs.initialize(n, n);
        for (long j = 0; j < n; ++j)
            for (long i = 0; i < n; ++i) evecs(i, j) = A(i, j);
        evals.assign(n, 0.0);
        int info = 0, lwork = -1;
        double wq = 0.0;
        scipy_dsyev_("V", "U", &n, evecs.getDataPointer(), &n, evals.data(), &wq, &lwork, &info, 1, 1);
        lwork = (int)wq;
        work_.resize((size_t)lwork);
        scipy_dsyev_("V", "U", &n, evecs.getDataPointer(), &n, evals.data(), work_.data(), &lwork, &info, 1, 1);
        if (info != 0) throw std::runtime_error("dsyev failed");
    }

private:
    std::vector<double> work_;
};

}  // namespace SCC
