// A CSR operator of the shape the reference's GPU solver calls (test infrastructure): a host
// single-vector apply(Vec&) (LanczosMaxMinFinder.h:341) and a device block apply(Mat& in, Mat& out,
// alpha, beta), out = alpha*A*in + beta*out, by cuSPARSE SpMM on the containers' own dense-matrix
// descriptors (AmatrixClassLMCuda.h:82-107; LanczosCpolyOperatorLMCuda.h:245). Vec and Mat are the
// reference's AvectorClassLMCuda<double> / AmatrixClassLMCuda<double> (or any containers with their
// vData, matrix_desc members). Used by tests/cpp/lmcuda_reference_containers.cu and
// oracle/ref_gpu_solve.cu.
#pragma once
#include <stdexcept>
#include <vector>

#include <cuda_runtime.h>
#include <cusparse.h>

template <class Vec, class Mat>
struct CusparseCsrOpT {
    long n = 0;
    std::vector<int> rp, ci;
    std::vector<double> v;
    int *d_rp = nullptr, *d_ci = nullptr;
    double* d_v = nullptr;
    cusparseHandle_t h = nullptr;
    cusparseSpMatDescr_t A = nullptr;
    void* buf = nullptr;
    size_t buf_bytes = 0;
    long calls = 0;

    void setup() {
        const long nnz = (long)ci.size();
        cudaMalloc(&d_rp, (n + 1) * sizeof(int));
        cudaMalloc(&d_ci, nnz * sizeof(int));
        cudaMalloc(&d_v, nnz * sizeof(double));
        cudaMemcpy(d_rp, rp.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice);
        cudaMemcpy(d_ci, ci.data(), nnz * sizeof(int), cudaMemcpyHostToDevice);
        cudaMemcpy(d_v, v.data(), nnz * sizeof(double), cudaMemcpyHostToDevice);
        if (cusparseCreate(&h) != CUSPARSE_STATUS_SUCCESS) throw std::runtime_error("cusparseCreate");
        cusparseCreateCsr(&A, n, n, nnz, d_rp, d_ci, d_v, CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I,
                          CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F);
    }
    ~CusparseCsrOpT() {
        if (A) cusparseDestroySpMat(A);
        if (h) cusparseDestroy(h);
        cudaFree(buf);
        cudaFree(d_rp);
        cudaFree(d_ci);
        cudaFree(d_v);
    }
    // host single-vector apply (the Lanczos bounds of the reference)
    void apply(Vec& x) {
        std::vector<double> y((size_t)n);
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
        for (long i = 0; i < n; ++i) {
            double s = 0.0;
            for (int k = rp[i]; k < rp[i + 1]; ++k) s += v[k] * x.vData[ci[k]];
            y[i] = s;
        }
        x.vData.swap(y);
    }
    // device block apply out = alpha*A*in + beta*out on the containers' cuSPARSE descriptors
    void apply(Mat& in, Mat& out, double alpha, double beta) {
        ++calls;
        size_t need = 0;
        if (cusparseSpMM_bufferSize(h, CUSPARSE_OPERATION_NON_TRANSPOSE, CUSPARSE_OPERATION_NON_TRANSPOSE, &alpha, A,
                                    in.matrix_desc, &beta, out.matrix_desc, CUDA_R_64F, CUSPARSE_SPMM_ALG_DEFAULT,
                                    &need) != CUSPARSE_STATUS_SUCCESS)
            throw std::runtime_error("cusparseSpMM_bufferSize");
        if (need > buf_bytes) {
            cudaFree(buf);
            cudaMalloc(&buf, need);
            buf_bytes = need;
        }
        if (cusparseSpMM(h, CUSPARSE_OPERATION_NON_TRANSPOSE, CUSPARSE_OPERATION_NON_TRANSPOSE, &alpha, A,
                         in.matrix_desc, &beta, out.matrix_desc, CUDA_R_64F, CUSPARSE_SPMM_ALG_DEFAULT,
                         buf) != CUSPARSE_STATUS_SUCCESS)
            throw std::runtime_error("cusparseSpMM");
    }
};

