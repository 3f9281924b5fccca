// rc_noalloc.cu -- the small Hermitian eigensolver without any device allocation.
//
// rc_small_eigh stages H, Q and the eigenvalues in device scratch taken from the context's
// allocator, and the Jacobi kernel needs global work memory whenever its working copies do not
// fit in shared memory. Some callers cannot allocate device memory at the point where they need
// this result: code that runs under a fixed device-memory budget negotiated at start-up (a
// cudaMalloc there can fail or push another tenant of the GPU out of memory), and callbacks
// invoked from another library's allocator or from an operator apply(), where allocating again
// would re-enter that library. For them, rc_small_eigh_noalloc uses one file-scope device array
// of fixed size instead (about 1.3 MiB on every GPU that loads this library, held until the
// process exits) and calls no cudaMalloc or cudaFree.
//
// Set-up: the first call on a device (and the first after that device's CUDA context was
// re-created, for example by cudaDeviceReset) looks up the array's device address with
// cudaGetSymbolAddress, which may also load this library's module on the device; make that first
// call before any stream capture. Later calls in the same context do no set-up.
#include <cstring>
#include <mutex>
#include "rc_common.cuh"
#include "rc_internal.h"

namespace {

constexpr int64_t kNoAllocMaxS = 128;                                      // largest s accepted
constexpr size_t kEsz = 16;                                                // complex double (the wider scalar)
constexpr size_t kMat = (size_t)kNoAllocMaxS * kNoAllocMaxS * kEsz;       // staging for H and for Q
constexpr size_t kEvals = (size_t)kNoAllocMaxS * sizeof(double) + 256;     // eigenvalues + sweep count
constexpr size_t kWork = 3 * (size_t)kNoAllocMaxS * (kNoAllocMaxS + 1) * kEsz;  // Jacobi working copies (A twice, Q)
constexpr size_t kScratchBytes = 2 * kMat + kEvals + kWork;

// Shared by every call on a device; calls whose work overlaps on the GPU race on it.
static __device__ __align__(256) unsigned char rc_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
constexpr int kMaxDevices = 128;
// The array's device address per device, and the CUDA context it belongs to: a symbol's address is
// valid only in the context that resolved it, so a re-created context resolves it again.
struct ScratchAddr {
    void* ctx = nullptr;
    void* ptr = nullptr;
};
ScratchAddr g_scratch[kMaxDevices];

// cuCtxGetCurrent through the runtime's driver entry point (no link-time dependency on libcuda).
typedef int (*CtxGetCurrentFn)(void**);
CtxGetCurrentFn ctx_get_current() {
    static CtxGetCurrentFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return (CtxGetCurrentFn)f;
    }();
    return fn;
}

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
    // Set-up, once per device (per CUDA context) with that device current: the array's name is
    // only a host-side handle, so the kernel must be given the device address of the array.
    unsigned char* base = nullptr;
    {
        // the current context exists once a runtime call has made the device current (cudaSetDevice
        // above initialises it)
        void* cur = nullptr;
        CtxGetCurrentFn get = ctx_get_current();
        if (!get || get(&cur) != 0 || !cur)
            return rc_fail(ctx, RC_ERR_CUDA, "rc_small_eigh_noalloc: no current CUDA context");
        std::lock_guard<std::mutex> lock(g_mu);
        ScratchAddr& sa = g_scratch[ctx->device];
        if (!sa.ptr || sa.ctx != cur) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, rc_noalloc_scratch);
            if (e != cudaSuccess || !p)
                return rc_fail(ctx, RC_ERR_CUDA,
                               std::string("cudaGetSymbolAddress(rc_noalloc_scratch): ") + cudaGetErrorString(e));
            sa.ctx = cur;
            sa.ptr = p;
        }
        base = (unsigned char*)sa.ptr;
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
