// rc_batch.h -- batched filter applications of concurrent solves (rc_batch.cu), used by the
// request server (rc_serve.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include "rc_internal.h"

namespace rcb {

constexpr int kMaxBatchJobs = 64;   // filter applications per batch
constexpr int kBatchSlots = 4;      // device tables in flight (ring)
constexpr int64_t kMaxGraphDepth = 256;  // deeper batches launch without a graph
constexpr int32_t kBatchCorr = 2;        // BatchJob::prec of a correction-filter application

// One solve's filter application X <- P_m(A')X as the batched kernels read it.
struct BatchJob {
    int32_t kind;     // 0 CSR, 5 / 7 / 27 stencil (real)
    int32_t prec;     // P32 or P64 (storage and compute), or kBatchCorr (rc_corr_t storage, FP32)
    int32_t nseg;     // 16-byte slices per row-major row / slices per thread
    int32_t groups;   // consecutive row groups per virtual CTA
    int64_t n, ld, ldv, s, degree;
    int64_t vcta0, vcta1;  // virtual CTAs of the degree steps
    int64_t tile0, tile1;  // virtual 32x32 tiles of the layout changes
    int64_t tiles_x;       // row tiles, ceil(n / 32)
    const int32_t* rowptr;
    const int32_t* colind;
    const void* vals;      // CSR values in the storage precision
    const void* diag;      // stencil diagonal in the storage precision
    double offd;
    int64_t nx, ny, nz;
    double* V;             // the solve's column-major FP64 block (x0 in, x_m / (m+1) out)
    void* bufA;            // row-major intermediates
    void* bufB;
    double a, b;           // x_k = a A x_{k-1} + b x_{k-1} - x_{k-2}
    int64_t pf_z, pf_x;    // L2 prefetch distances (rows)
    const void* R;         // kBatchCorr: the residual block (e_1), row-major rc_corr_t
    const float* sig;      // kBatchCorr: source coefficients, (degree + 1) x ld
    const double* coef;    // kBatchCorr: weight of V in the result, one per column
};

struct BatchTable {
    int32_t njobs;
    int32_t pad;
    int64_t total_vctas;
    int64_t total_tiles;
    BatchJob jobs[kMaxBatchJobs];
};

struct BatchCounters {
    int64_t batches = 0;
    int64_t jobs = 0;
    int64_t kernel_launches = 0;
    int64_t graph_launches = 0;
    int64_t graphs_built = 0;
    int64_t max_jobs = 0;
};

struct BatchRunner;

// Describe a filter application for the batched kernels; false when it needs the single-solve
// path (callback or complex operator, degree < 2, 64-bit offsets, scratch too small, or a
// slice count forced by the context that the batched kernels do not use). The FP32 copy of the
// operator must already exist for prec == RC_PREC_MIXED.
bool batch_job_describe(const rc_ctx* ctx, const rc_op* op, void* V, int64_t ldv, int64_t s, int64_t degree,
                        double a, double b, int prec, void* bufA, void* bufB, size_t buf_bytes, BatchJob* J);

// The same for a correction-filter application (rm_filter_corr): V holds the Ritz vectors, R their
// residual block, sig and coef the tables corr_coef_kernel wrote. CSR and 5/7-point stencils with
// 32-bit offsets; the 27-point stencil keeps the single-solve run form (rm_step_rows27).
bool batch_job_describe_corr(const rc_ctx* ctx, const rc_op* op, double* V, int64_t ldv, int64_t s, int64_t degree,
                             double a, double b, const rc_corr_t* R, const float* sig, const double* coef,
                             void* bufA, void* bufB, BatchJob* J);

rc_status batch_runner_create(int device, int sm_count, bool use_graphs, BatchRunner** out, std::string* err);
void batch_runner_destroy(BatchRunner* R);
cudaStream_t batch_runner_stream(BatchRunner* R);
BatchCounters batch_runner_counters(const BatchRunner* R);
// Launch one batch on the runner's stream (the caller has made that stream wait for every job's
// inputs). *done is recorded after the batch; jobs' streams wait on it before reading V.
rc_status batch_run(BatchRunner* R, const BatchJob* jobs, int njobs, cudaEvent_t* done, std::string* err);

}  // namespace rcb
