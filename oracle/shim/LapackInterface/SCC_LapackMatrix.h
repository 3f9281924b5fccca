// Stand-in for the un-vendored SCC LapackInterface component the reference's GPU solver includes
// (RayleighChebyshevLMCuda.h:171-177): the column-major dense matrix it uses in
// computeVtVeigensystem (:585-627). Test infrastructure: built only into oracle/_ref/ by
// oracle/Makefile, never part of the library. Our own code; the SCC library is not vendored here.
#pragma once
#include <vector>

namespace SCC {

class LapackMatrix {
public:
    void initialize(long rows, long cols) {
        rows_ = rows;
        cols_ = cols;
        data_.assign((size_t)rows * cols, 0.0);
    }
    double& operator()(long i, long j) { return data_[(size_t)i + (size_t)j * rows_]; }
    const double& operator()(long i, long j) const { return data_[(size_t)i + (size_t)j * rows_]; }
    long getRowDimension() const { return rows_; }
    long getColDimension() const { return cols_; }
    double* getDataPointer() { return data_.data(); }

private:
    long rows_ = 0, cols_ = 0;
    std::vector<double> data_;
};

}  // namespace SCC
