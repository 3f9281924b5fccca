// rc_batch.cu -- the filter applications of several concurrent solves in one set of launches.
//
// A batch holds up to kMaxBatchJobs filter applications X_j <- P_{m_j}(A_j') X_j, each with its
// own operator (CSR or 5/7/27-point stencil, real), block width, degree, recurrence coefficients
// and storage precision (FP32 or FP64). The whole batch runs as
//   batch_to_rm  -> batch_step(k = 1) -> ... -> batch_step(k = D) -> batch_to_cm,   D = max m_j,
// one launch per stage for all solves: each launch walks one virtual CTA numbering that
// concatenates the solves' own CTA ranges, and a solve whose degree is below k skips its range.
// The per-solve arithmetic is the single-solve row-major filter's (rc_rmstep.cuh), so a solve
// gets the same values whether it runs alone, in a batch, or outside the server.
// A batch also carries correction-filter applications (prec kBatchCorr, the MIXED refinement of
// rc_filter_rm.cu): they skip the entry layout change, run their steps k = 2..m in a third step
// kernel (bfloat16 blocks, the residual block as the source term) and form V = coef v + a e_m/(m+1)
// in the exit layout change.
//
// The batch description lives in a device table that a memcpy node refreshes from pinned host
// memory at the start of the batch, so one captured CUDA graph per (D, table slot) serves every
// batch of that depth: the server replays a graph instead of issuing D + 3 launches.
#include <algorithm>
#include <cstring>
#include <map>
#include <utility>
#include "rc_batch.h"
#include "rc_common.cuh"
#include "rc_rmstep.cuh"

namespace rcb {

// Grids of the batched kernels: the step kernels' resident CTAs per SM (rm_min_blocks, as the
// single-solve kernels) and the transposes'.
constexpr int kBatchTileBlocksPerSm = 8;

template <class TS, class TC, class Pol, int W>
__device__ __noinline__ void batch_step_typed(const Pol pol, const BatchJob& J, int k, int64_t cta) {
    constexpr int VEC = Pack16<TS>::V;
    (void)VEC;
    TS* A = (TS*)J.bufA;
    TS* B = (TS*)J.bufB;
    const TS* xk1 = (k - 1) % 2 ? B : A;  // x_{k-1}
    TS* y = k % 2 ? B : A;                // x_k overwrites x_{k-2}
    const TS* z = k >= 2 ? y : nullptr;
    const TC ta = s_from<TC>(J.a, 0.0), tb = s_from<TC>(J.b, 0.0);
    const TC tg = k >= 2 ? s_from<TC>(-1.0, 0.0) : s_zero(TC());
    rm_step_rows<Pol, TS, TC, W, uint32_t>(pol, J.n, J.nseg, J.ld, J.groups, cta, xk1, z, y, ta, tb, tg, J.pf_z,
                                           J.pf_x);
}

template <class TS>
__device__ __forceinline__ void batch_step_job(const BatchJob& J, int k, int64_t cta) {
    using TD = TS;
    const TD* dg = (const TD*)J.diag;
    if (J.kind == 0) {
        CsrRows<TS, TS> pol{J.rowptr, J.colind, (const TS*)J.vals};
        if (sizeof(TS) == 8) batch_step_typed<TS, TS, CsrRows<TS, TS>, 2>(pol, J, k, cta);
        else batch_step_typed<TS, TS, CsrRows<TS, TS>, 1>(pol, J, k, cta);
    } else if (J.kind == 7) {
        StencilRows<TD, TS, 7> pol{J.nx, J.ny, J.nz, dg, J.offd, 0.0};
        batch_step_typed<TS, TS, StencilRows<TD, TS, 7>, 1>(pol, J, k, cta);
    } else if (J.kind == 5) {
        StencilRows<TD, TS, 5> pol{J.nx, J.ny, J.nz, dg, J.offd, 0.0};
        batch_step_typed<TS, TS, StencilRows<TD, TS, 5>, 1>(pol, J, k, cta);
    } else {
        StencilRows<TD, TS, 27> pol{J.nx, J.ny, J.nz, dg, J.offd, 0.0};
        batch_step_typed<TS, TS, StencilRows<TD, TS, 27>, 1>(pol, J, k, cta);
    }
}

// Degree-step k of every solve of the batch whose storage precision is TS (one kernel per
// precision, so each keeps the single-solve kernel's register budget). Virtual CTA v belongs to
// the job whose [vcta0, vcta1) holds it; each CTA walks v = blockIdx.x, blockIdx.x + gridDim.x,
// ... so the job index only moves forward.
template <class TS>
__global__ void __launch_bounds__(kRmThreads, rm_min_blocks<TS>())
batch_step_kernel(const BatchTable* __restrict__ T, int k) {
    __shared__ int64_t ends[kMaxBatchJobs];
    const int nj = T->njobs;
    for (int j = threadIdx.x; j < nj; j += blockDim.x) ends[j] = T->jobs[j].vcta1;
    __syncthreads();
    const int64_t total = T->total_vctas;
    constexpr int kPrec = sizeof(TS) == 4 ? P32 : P64;
    int j = 0;
    for (int64_t v = blockIdx.x; v < total; v += gridDim.x) {
        while (j < nj && ends[j] <= v) ++j;
        if (j >= nj) break;
        const BatchJob& J = T->jobs[j];
        if (J.prec != kPrec || k > J.degree) continue;
        batch_step_job<TS>(J, k, v - J.vcta0);
    }
}

// Degree-step k (2 <= k <= m) of every correction-filter application of the batch, with the
// single-solve correction filter's buffer rotation (run_rm_corr): e_1 = R, e_k over e_{k-2}.
template <class Pol>
__device__ __noinline__ void batch_corr_step_typed(const Pol pol, const BatchJob& J, int k, int64_t cta) {
    using TM = rc_corr_t;
    const TM* R = (const TM*)J.R;
    TM* A = (TM*)J.bufA;
    TM* B = (TM*)J.bufB;
    const TM* xk1 = k == 2 ? R : ((k - 1) % 2 == 0 ? A : B);  // e_{k-1}
    TM* y = k % 2 == 0 ? A : B;                                 // e_k
    const TM* z = k == 2 ? nullptr : (k == 3 ? R : y);          // e_{k-2}
    const float ta = s_from<float>(J.a, 0.0), tb = s_from<float>(J.b, 0.0);
    const float tg = k == 2 ? s_zero(float()) : s_from<float>(-1.0, 0.0);
    rm_step_rows<Pol, float, float, 1, uint32_t, true, TM>(pol, J.n, J.nseg, J.ld, J.groups, cta, xk1, z, y, ta, tb,
                                                           tg, J.pf_z, J.pf_x, R, J.sig + k * J.ld);
}

// 4 resident CTAs per SM: the out-of-line per-operator step (which keeps each operator's code
// apart, as batch_step_typed does) spills at the single-solve kernel's 6.
constexpr int kBatchCorrBlocksPerSm = 4;

__global__ void __launch_bounds__(kRmThreads, kBatchCorrBlocksPerSm)
batch_corr_step_kernel(const BatchTable* __restrict__ T, int k) {
    __shared__ int64_t ends[kMaxBatchJobs];
    const int nj = T->njobs;
    for (int j = threadIdx.x; j < nj; j += blockDim.x) ends[j] = T->jobs[j].vcta1;
    __syncthreads();
    const int64_t total = T->total_vctas;
    int j = 0;
    for (int64_t v = blockIdx.x; v < total; v += gridDim.x) {
        while (j < nj && ends[j] <= v) ++j;
        if (j >= nj) break;
        const BatchJob& J = T->jobs[j];
        if (J.prec != kBatchCorr || k < 2 || k > J.degree) continue;
        const int64_t cta = v - J.vcta0;
        if (J.kind == 0) {
            CsrRows<float, float> pol{J.rowptr, J.colind, (const float*)J.vals};
            batch_corr_step_typed(pol, J, k, cta);
        } else if (J.kind == 7) {
            StencilRows<float, float, 7> pol{J.nx, J.ny, J.nz, (const float*)J.diag, J.offd, 0.0};
            batch_corr_step_typed(pol, J, k, cta);
        } else {
            StencilRows<float, float, 5> pol{J.nx, J.ny, J.nz, (const float*)J.diag, J.offd, 0.0};
            batch_corr_step_typed(pol, J, k, cta);
        }
    }
}

// Layout changes of every solve: to_rm (x0 = X, column-major FP64 -> row-major storage) and
// to_cm (X = x_m / (m+1)). Virtual tiles as above; a barrier closes each tile because the
// shared tile is reused by the next one.
template <bool TO_RM>
__global__ void __launch_bounds__(256, kBatchTileBlocksPerSm)
batch_transpose_kernel(const BatchTable* __restrict__ T) {
    __shared__ double tile64[32][33];
    float(&tile32)[32][33] = *reinterpret_cast<float(*)[32][33]>(&tile64[0][0]);
    __shared__ int64_t ends[kMaxBatchJobs];
    const int nj = T->njobs;
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    for (int j = tid; j < nj; j += blockDim.x * blockDim.y) ends[j] = T->jobs[j].tile1;
    __syncthreads();
    const int64_t total = T->total_tiles;
    int j = 0;
    for (int64_t v = blockIdx.x; v < total; v += gridDim.x) {
        while (j < nj && ends[j] <= v) ++j;
        if (j >= nj) break;
        const BatchJob& J = T->jobs[j];
        const int64_t t = v - J.tile0;
        const int64_t r0 = (t % J.tiles_x) * 32, c0 = (t / J.tiles_x) * 32;
        if (J.prec == kBatchCorr) {  // no entry layout change; the exit forms coef v + a e_m / (m+1)
            if (TO_RM) continue;
            const void* em = J.degree == 1 ? J.R : (J.degree % 2 == 0 ? J.bufA : J.bufB);
            corr_to_cm_tile<rc_corr_t>(J.n, J.s, (const rc_corr_t*)em, J.ld, J.V, J.ldv, J.coef,
                                       J.a / (double)(J.degree + 1), r0, c0, tile32);
        } else if (TO_RM) {
            if (J.prec == P32) to_rm_tile<double, float>(J.n, J.s, J.V, J.ldv, (float*)J.bufA, J.ld, r0, c0, tile32);
            else to_rm_tile<double, double>(J.n, J.s, J.V, J.ldv, (double*)J.bufA, J.ld, r0, c0, tile64);
        } else {
            const void* xm = J.degree % 2 ? J.bufB : J.bufA;
            const double scale = 1.0 / (double)(J.degree + 1);
            if (J.prec == P32)
                to_cm_tile<float, double>(J.n, J.s, (const float*)xm, J.ld, J.V, J.ldv, scale, r0, c0, tile32);
            else
                to_cm_tile<double, double>(J.n, J.s, (const double*)xm, J.ld, J.V, J.ldv, scale, r0, c0, tile64);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------
int64_t rm_leading_dim(int dtype, int prec, int64_t s);

bool batch_job_describe(const rc_ctx* ctx, const rc_op* op, void* V, int64_t ldv, int64_t s, int64_t degree,
                        double a, double b, int prec, void* bufA, void* bufB, size_t buf_bytes, BatchJob* J) {
    if (op->kind == 2 || op->dtype != RC_REAL64 || degree < 2 || s < 1) return false;
    if (op->kind == 1 && op->skind != 5 && op->skind != 7 && op->skind != 27) return false;
    const int p = prec == RC_PREC_MIXED ? P32 : P64;
    const int64_t ld = rm_leading_dim(op->dtype, p, s);
    const size_t esz = elem_bytes(op->dtype, p);
    if (!bufA || !bufB || buf_bytes < (size_t)op->n * ld * esz) return false;
    // 32-bit element offsets only, and the single-solve choices of slices (two for FP64 CSR)
    if ((op->n + 1) * ld >= ((int64_t)1 << 32)) return false;
    if (ctx->rm_slices != 0 && ctx->rm_slices != ((op->kind == 0 && p == P64) ? 2 : 1)) return false;
    const int W = (op->kind == 0 && p == P64) ? 2 : 1;
    const int vec = (int)(16 / esz);
    if (ld % (vec * W) != 0) return false;
    const int nseg = (int)(ld / (vec * W));
    if (nseg > kRmThreads) return false;
    const bool csr = op->kind == 0, f32 = p == P32;
    const int groups = ctx->rm_groups > 0 ? ctx->rm_groups : (csr ? (f32 ? 4 : 2) : (f32 ? 8 : 4));
    const int64_t rows_per_cta = (int64_t)groups * (kRmThreads / nseg);
    if (p == P32) {
        if (csr ? op->vals32 == nullptr : op->diag32 == nullptr) return false;
    }
    std::memset(J, 0, sizeof(*J));
    J->kind = csr ? 0 : op->skind;
    J->prec = p;
    J->nseg = nseg;
    J->groups = groups;
    J->n = op->n;
    J->ld = ld;
    J->ldv = ldv;
    J->s = s;
    J->degree = degree;
    J->vcta1 = (op->n + rows_per_cta - 1) / rows_per_cta;  // local count; offsets added by batch_run
    J->tiles_x = (op->n + 31) / 32;
    J->tile1 = J->tiles_x * ((s + 31) / 32);
    J->rowptr = op->rowptr;
    J->colind = op->colind;
    J->vals = f32 ? op->vals32 : op->vals64;
    J->diag = f32 ? (const void*)op->diag32 : (const void*)op->diag64;
    J->offd = op->offdiag;
    J->nx = op->nx;
    J->ny = op->ny;
    J->nz = op->nz;
    J->V = (double*)V;
    J->bufA = bufA;
    J->bufB = bufB;
    J->a = a;
    J->b = b;
    const int64_t band = csr ? op->band : (op->skind == 5 ? op->nx : op->nx * op->ny);
    J->pf_z = ctx->pf_rows;
    J->pf_x = ctx->pf_rows > 0 ? ctx->pf_rows + band : 0;
    return true;
}

bool batch_job_describe_corr(const rc_ctx* ctx, const rc_op* op, double* V, int64_t ldv, int64_t s, int64_t degree,
                             double a, double b, const rc_corr_t* R, const float* sig, const double* coef,
                             void* bufA, void* bufB, BatchJob* J) {
    if (op->kind == 2 || op->dtype != RC_REAL64 || degree < 1 || s < 1) return false;
    if (op->kind == 1 && op->skind != 5 && op->skind != 7) return false;
    const int64_t ld = rm_leading_dim(RC_REAL64, P32, s);
    if ((op->n + 1) * ld >= ((int64_t)1 << 32)) return false;
    const int vec = (int)(16 / sizeof(rc_corr_t));
    if (ld % vec != 0) return false;
    const int nseg = (int)(ld / vec);
    if (nseg > kRmThreads) return false;
    const bool csr = op->kind == 0;
    if (csr ? op->vals32 == nullptr : op->diag32 == nullptr) return false;
    // the single-solve correction filter's choices (run_rm_corr)
    const int groups = ctx->rm_groups > 0 ? ctx->rm_groups : (csr ? 4 : 8);
    const int64_t rows_per_cta = (int64_t)groups * (kRmThreads / nseg);
    std::memset(J, 0, sizeof(*J));
    J->kind = csr ? 0 : op->skind;
    J->prec = kBatchCorr;
    J->nseg = nseg;
    J->groups = groups;
    J->n = op->n;
    J->ld = ld;
    J->ldv = ldv;
    J->s = s;
    J->degree = degree;
    J->vcta1 = (op->n + rows_per_cta - 1) / rows_per_cta;
    J->tiles_x = (op->n + 31) / 32;
    J->tile1 = J->tiles_x * ((s + 31) / 32);
    J->rowptr = op->rowptr;
    J->colind = op->colind;
    J->vals = op->vals32;
    J->diag = op->diag32;
    J->offd = op->offdiag;
    J->nx = op->nx;
    J->ny = op->ny;
    J->nz = op->nz;
    J->V = V;
    J->bufA = bufA;
    J->bufB = bufB;
    J->a = a;
    J->b = b;
    const int64_t band = csr ? op->band : (op->skind == 5 ? op->nx : op->nx * op->ny);
    J->pf_z = ctx->pf_rows;
    J->pf_x = ctx->pf_rows > 0 ? ctx->pf_rows + band : 0;
    J->R = R;
    J->sig = sig;
    J->coef = coef;
    return true;
}

struct BatchRunner {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    bool use_graphs = true;
    BatchTable* host[kBatchSlots] = {};
    BatchTable* dev[kBatchSlots] = {};
    cudaEvent_t done[kBatchSlots] = {};
    bool used[kBatchSlots] = {};
    int next = 0;
    std::map<std::pair<int64_t, int>, cudaGraphExec_t> graphs;
    BatchCounters counters;
};

rc_status batch_runner_create(int device, int sm_count, bool use_graphs, BatchRunner** out, std::string* err) {
    *out = nullptr;
    BatchRunner* R = new BatchRunner();
    R->device = device;
    R->sm_count = sm_count;
    R->use_graphs = use_graphs;
    auto fail = [&](const char* what) {
        *err = std::string("batch runner: ") + what;
        batch_runner_destroy(R);
        return RC_ERR_CUDA;
    };
    if (cudaStreamCreateWithFlags(&R->stream, cudaStreamNonBlocking) != cudaSuccess) return fail("stream");
    for (int i = 0; i < kBatchSlots; ++i) {
        if (cudaMallocHost((void**)&R->host[i], sizeof(BatchTable)) != cudaSuccess) return fail("pinned table");
        if (cudaMalloc((void**)&R->dev[i], sizeof(BatchTable)) != cudaSuccess) return fail("device table");
        if (cudaEventCreateWithFlags(&R->done[i], cudaEventDisableTiming) != cudaSuccess) return fail("event");
        std::memset(R->host[i], 0, sizeof(BatchTable));
    }
    *out = R;
    return RC_OK;
}

void batch_runner_destroy(BatchRunner* R) {
    if (!R) return;
    if (R->stream) cudaStreamSynchronize(R->stream);
    for (auto& g : R->graphs) cudaGraphExecDestroy(g.second);
    for (int i = 0; i < kBatchSlots; ++i) {
        if (R->host[i]) cudaFreeHost(R->host[i]);
        if (R->dev[i]) cudaFree(R->dev[i]);
        if (R->done[i]) cudaEventDestroy(R->done[i]);
    }
    if (R->stream) cudaStreamDestroy(R->stream);
    delete R;
}

cudaStream_t batch_runner_stream(BatchRunner* R) { return R->stream; }
BatchCounters batch_runner_counters(const BatchRunner* R) { return R->counters; }

// The batch's launches on R->stream, reading table `tab` (device).
static int64_t batch_launches(int64_t depth, bool has32, bool has64, bool hasC) {
    return depth * ((has32 ? 1 : 0) + (has64 ? 1 : 0)) + (hasC ? std::max<int64_t>(depth - 1, 0) : 0) + 2;
}

static cudaError_t issue(BatchRunner* R, int slot, int64_t depth, bool has32, bool has64, bool hasC,
                         int64_t* launches) {
    const unsigned gs = (unsigned)(R->sm_count * rm_min_blocks<float>());
    const unsigned gt = (unsigned)(R->sm_count * kBatchTileBlocksPerSm);
    const dim3 tblk(32, 8);
    cudaError_t e = cudaMemcpyAsync(R->dev[slot], R->host[slot], sizeof(BatchTable), cudaMemcpyHostToDevice, R->stream);
    if (e != cudaSuccess) return e;
    batch_transpose_kernel<true><<<gt, tblk, 0, R->stream>>>(R->dev[slot]);
    const unsigned gs64 = (unsigned)(R->sm_count * rm_min_blocks<double>());
    const unsigned gsc = (unsigned)(R->sm_count * kBatchCorrBlocksPerSm);
    for (int64_t k = 1; k <= depth; ++k) {
        if (has32) batch_step_kernel<float><<<gs, kRmThreads, 0, R->stream>>>(R->dev[slot], (int)k);
        if (has64) batch_step_kernel<double><<<gs64, kRmThreads, 0, R->stream>>>(R->dev[slot], (int)k);
        if (hasC && k >= 2) batch_corr_step_kernel<<<gsc, kRmThreads, 0, R->stream>>>(R->dev[slot], (int)k);
    }
    batch_transpose_kernel<false><<<gt, tblk, 0, R->stream>>>(R->dev[slot]);
    *launches = batch_launches(depth, has32, has64, hasC);
    return cudaGetLastError();
}

rc_status batch_run(BatchRunner* R, const BatchJob* jobs, int njobs, cudaEvent_t* done, std::string* err) {
    if (njobs < 1 || njobs > kMaxBatchJobs) {
        *err = "batch_run: bad job count";
        return RC_ERR_INVALID;
    }
    const int slot = R->next;
    R->next = (R->next + 1) % kBatchSlots;
    if (R->used[slot] && cudaEventSynchronize(R->done[slot]) != cudaSuccess) {
        *err = "batch_run: waiting for an earlier batch failed";
        return RC_ERR_CUDA;
    }
    BatchTable* T = R->host[slot];
    T->njobs = njobs;
    int64_t vc = 0, tc = 0, depth = 0;
    bool has32 = false, has64 = false, hasC = false;
    for (int j = 0; j < njobs; ++j) {
        BatchJob J = jobs[j];
        const int64_t nv = J.vcta1, nt = J.tile1;  // local counts from batch_job_describe
        J.vcta0 = vc;
        J.vcta1 = vc + nv;
        J.tile0 = tc;
        J.tile1 = tc + nt;
        vc += nv;
        tc += nt;
        depth = std::max(depth, J.degree);
        (J.prec == kBatchCorr ? hasC : (J.prec == P32 ? has32 : has64)) = true;
        T->jobs[j] = J;
    }
    T->total_vctas = vc;
    T->total_tiles = tc;
    int64_t launches = 0;
    cudaError_t e = cudaSuccess;
    if (R->use_graphs && depth <= kMaxGraphDepth) {
        // graph key: depth, table slot and which precisions have step kernels
        const int64_t kind = depth * 8 + (has32 ? 1 : 0) + (has64 ? 2 : 0) + (hasC ? 4 : 0);
        const auto key = std::make_pair(kind, slot);
        auto it = R->graphs.find(key);
        if (it == R->graphs.end()) {
            cudaGraph_t g = nullptr;
            cudaGraphExec_t ge = nullptr;
            e = cudaStreamBeginCapture(R->stream, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                cudaError_t ei = issue(R, slot, depth, has32, has64, hasC, &launches);
                e = cudaStreamEndCapture(R->stream, &g);
                if (ei != cudaSuccess) e = ei;
            }
            if (e == cudaSuccess) e = cudaGraphInstantiate(&ge, g, 0);
            if (g) cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                cudaGetLastError();
                *err = std::string("batch graph capture: ") + cudaGetErrorString(e);
                return RC_ERR_CUDA;
            }
            it = R->graphs.emplace(key, ge).first;
            R->counters.graphs_built++;
        }
        e = cudaGraphLaunch(it->second, R->stream);
        launches = batch_launches(depth, has32, has64, hasC);
        R->counters.graph_launches++;
    } else {
        e = issue(R, slot, depth, has32, has64, hasC, &launches);
    }
    if (e == cudaSuccess) e = cudaEventRecord(R->done[slot], R->stream);
    if (e != cudaSuccess) {
        *err = std::string("batch launch: ") + cudaGetErrorString(e);
        return RC_ERR_CUDA;
    }
    R->used[slot] = true;
    R->counters.batches++;
    R->counters.jobs += njobs;
    R->counters.kernel_launches += launches;
    R->counters.max_jobs = std::max<int64_t>(R->counters.max_jobs, njobs);
    *done = R->done[slot];
    return RC_OK;
}

}  // namespace rcb
