// rc_noalloc.cu -- the small Hermitian eigensolver without any device allocation.
//
// rc_small_eigh stages H, Q and the eigenvalues in device scratch taken from the context's
// allocator, and the Jacobi kernel needs global work memory whenever its working copies do not
// fit in shared memory. Some callers cannot allocate device memory at the point where they need
// this result: code running inside a CUDA stream capture (a cudaMalloc there breaks the capture),
// code that runs under a fixed device-memory budget negotiated at start-up, and callbacks invoked
// from another library's allocator or from an operator apply(). For them,
// rc_small_eigh_noalloc uses one file-scope device array of fixed size instead (about 1 MiB on
// every GPU that loads this library, held until the process exits) and calls no cudaMalloc or
// cudaFree.
#include <cstring>
#include <mutex>
#include "rc_common.cuh"
#include "rc_internal.h"

namespace {

constexpr int64_t kNoAllocMaxS = 128;                                      // largest s accepted
constexpr size_t kEsz = 16;                                                // complex double (the wider scalar)
constexpr size_t kMat = (size_t)kNoAllocMaxS * kNoAllocMaxS * kEsz;       // staging for H and for Q
constexpr size_t kEvals = (size_t)kNoAllocMaxS * sizeof(double) + 256;     // eigenvalues + sweep count
constexpr size_t kWork = 2 * (size_t)kNoAllocMaxS * (kNoAllocMaxS + 1) * kEsz;  // Jacobi working copies
constexpr size_t kScratchBytes = 2 * kMat + kEvals + kWork;

// Shared by every call on a device; calls whose work overlaps on the GPU race on it.
static __device__ __align__(256) unsigned char rc_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
constexpr int kMaxDevices = 128;
void* g_scratch[kMaxDevices] = {};

}  // namespace

extern "C" rc_status rc_small_eigh_noalloc(rc_ctx* ctx, int dtype, int64_t s, const void* H, double* evals,
                                           void* Q) {
    if (!ctx) return RC_ERR_INVALID;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return rc_fail(ctx, RC_ERR_CUDA, "cudaSetDevice failed");
    if (!H || !evals || (dtype != RC_REAL64 && dtype != RC_COMPLEX128))
        return rc_fail(ctx, RC_ERR_INVALID, "rc_small_eigh_noalloc: bad arguments");
    if (s < 1 || s > kNoAllocMaxS)
        return rc_fail(ctx, RC_ERR_INVALID, "rc_small_eigh_noalloc: s must be in [1, 128] (fixed scratch size)");
    if (ctx->device < 0 || ctx->device >= kMaxDevices)
        return rc_fail(ctx, RC_ERR_UNSUPPORTED, "rc_small_eigh_noalloc: device index out of range");
    // Set-up, once per device with that device current: the array's name is only a host-side
    // handle, so the kernel must be given the device address of the array.
    unsigned char* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_scratch[ctx->device]) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, rc_noalloc_scratch);
            if (e != cudaSuccess || !p)
                return rc_fail(ctx, RC_ERR_CUDA,
                               std::string("cudaGetSymbolAddress(rc_noalloc_scratch): ") + cudaGetErrorString(e));
            g_scratch[ctx->device] = p;
        }
        base = (unsigned char*)g_scratch[ctx->device];
    }
    const size_t mat = (size_t)s * s * elem_bytes(dtype, P64);
    void* Hd = base;
    void* Qd = base + kMat;
    double* dl = (double*)(base + 2 * kMat);
    int* di = (int*)(dl + kNoAllocMaxS);
    void* work = base + 2 * kMat + kEvals;
    RC_CU(ctx, cudaMemcpyAsync(Hd, H, mat, cudaMemcpyHostToDevice, ctx->stream));
    // every entry the kernel reads is written first (H staged above, its working copies
    // initialised by the kernel), so nothing left over from an earlier call is used
    RC_TRY(rcb::small_eigh_work(ctx, dtype, s, Hd, Qd, dl, di, work));
    RC_CU(ctx, cudaMemcpyAsync(evals, dl, (size_t)s * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (Q) RC_CU(ctx, cudaMemcpyAsync(Q, Qd, mat, cudaMemcpyDeviceToHost, ctx->stream));
    RC_CU(ctx, cudaStreamSynchronize(ctx->stream));
    return RC_OK;
}
