// Stand-in for SCC::LapackMatrixCmplx16 (see SCC_LapackMatrix.h): column-major complex<double>.
#pragma once
#include <complex>
#include <vector>

namespace SCC {

class LapackMatrixCmplx16 {
public:
    void initialize(long rows, long cols) {
        rows_ = rows;
        cols_ = cols;
        data_.assign((size_t)rows * cols, std::complex<double>(0.0, 0.0));
    }
    std::complex<double>& operator()(long i, long j) { return data_[(size_t)i + (size_t)j * rows_]; }
    const std::complex<double>& operator()(long i, long j) const { return data_[(size_t)i + (size_t)j * rows_]; }
    long getRowDimension() const { return rows_; }
    long getColDimension() const { return cols_; }
    std::complex<double>* getDataPointer() { return data_.data(); }

private:
    long rows_ = 0, cols_ = 0;
    std::vector<std::complex<double>> data_;
};

}  // namespace SCC
