// rc_capi.cu -- the extern "C" boundary (include/rc_b200.h).
//
// Every entry point validates its arguments, makes the context's device current, and
// returns a status code; nothing here terminates the process (the reference's error macros
// call exit(), cudaErrchk.h:8-51).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <vector>
#include <new>
#include <string>
#include "rc_common.cuh"
#include "rc_cpoly.h"
#include "rc_internal.h"

namespace rcb {
rc_status solve(rc_ctx* ctx, rc_op* op, const rc_solve_params& p, const void* v0, double* evals_out, void* evecs_out,
                double* resid_out, rc_solve_info* info);
}

rc_status rc_fail(rc_ctx* ctx, rc_status st, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return st;
}

rc_status rc_slot(rc_ctx* ctx, int slot, size_t bytes, void** out) {
    if ((int)ctx->slots.size() < S_COUNT) ctx->slots.resize(S_COUNT);
    DevBuf& b = ctx->slots[slot];
    if (b.bytes < bytes) {
        if (b.ptr) {
            if (ctx->pool) {
                cudaFreeAsync(b.ptr, ctx->stream);
            } else {
                cudaStreamSynchronize(ctx->stream);
                cudaFree(b.ptr);
            }
            b.ptr = nullptr;
            b.bytes = 0;
        }
        // round up to 2 MiB so repeated small growth does not thrash the allocator
        const size_t want = ((bytes + (2u << 20) - 1) / (2u << 20)) * (2u << 20);
        const cudaError_t e = ctx->pool ? cudaMallocFromPoolAsync(&b.ptr, want, ctx->pool, ctx->stream)
                                        : cudaMalloc(&b.ptr, want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            b.ptr = nullptr;
            return rc_fail(ctx, RC_ERR_NOMEM, "cudaMalloc of " + std::to_string(want) + " bytes failed");
        }
        b.bytes = want;
    }
    *out = b.ptr;
    return RC_OK;
}

void rc_release_slots(rc_ctx* ctx) {
    for (auto& b : ctx->slots) {
        if (b.ptr) {
            if (ctx->pool) {
                cudaFreeAsync(b.ptr, ctx->stream);
            } else {
                cudaStreamSynchronize(ctx->stream);
                cudaFree(b.ptr);
            }
        }
        b.ptr = nullptr;
        b.bytes = 0;
    }
}

rc_status rc_host_small(rc_ctx* ctx, size_t bytes, double** out) {
    if (ctx->host_small_bytes < bytes) {
        if (ctx->host_small) {
            cudaStreamSynchronize(ctx->stream);
            cudaFreeHost(ctx->host_small);
        }
        ctx->host_small = nullptr;
        ctx->host_small_bytes = 0;
        const size_t want = bytes < 4096 ? 4096 : bytes;
        if (cudaMallocHost((void**)&ctx->host_small, want) != cudaSuccess)
            return rc_fail(ctx, RC_ERR_NOMEM, "cudaMallocHost failed");
        ctx->host_small_bytes = want;
    }
    *out = ctx->host_small;
    return RC_OK;
}

#define RC_CHECK_CTX(ctx)                                    \
    do {                                                     \
        if (!(ctx)) return RC_ERR_INVALID;                   \
        if (cudaSetDevice((ctx)->device) != cudaSuccess)     \
            return rc_fail((ctx), RC_ERR_CUDA, "cudaSetDevice failed"); \
    } while (0)

static void op_release(rc_op* op) {
    if (op->rowptr) cudaFree(op->rowptr);
    if (op->colind) cudaFree(op->colind);
    if (op->vals64) cudaFree(op->vals64);
    if (op->vals32) cudaFree(op->vals32);
    if (op->diag64) cudaFree(op->diag64);
    if (op->diag32) cudaFree(op->diag32);
    if (op->phase64) cudaFree(op->phase64);
    if (op->phase32) cudaFree(op->phase32);
    delete op;
}

extern "C" {

int rc_abi_version(void) { return RC_B200_ABI_VERSION; }

rc_status rc_ctx_create(int device, rc_ctx** out) {
    if (!out) return RC_ERR_INVALID;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return RC_ERR_CUDA;
    }
    if (device < 0 || device >= count) return RC_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return RC_ERR_CUDA;
    rc_ctx* c = new (std::nothrow) rc_ctx();
    if (!c) return RC_ERR_NOMEM;
    c->device = device;
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return RC_ERR_CUDA;
    }
    c->stream = c->own_stream;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) {
        c->sm_count = prop.multiProcessorCount;
        c->smem_optin = prop.sharedMemPerBlockOptin;
    }
    c->slots.resize(S_COUNT);
    if (const char* v = std::getenv("RCB200_CM_CPT")) c->cm_cpt = std::max(0, std::atoi(v));
    if (const char* v = std::getenv("RCB200_CM_ORDER")) c->cm_order = std::atoi(v) == 1 ? 1 : 0;
    if (const char* v = std::getenv("RCB200_CSR_KERNEL")) {
        if (!std::strcmp(v, "loop")) c->csr_variant = 1;
        else if (!std::strcmp(v, "reg")) c->csr_variant = 2;
    }
    if (const char* v = std::getenv("RCB200_STAGED")) c->staged = std::atoi(v) != 0 ? 1 : 0;
    if (const char* v = std::getenv("RCB200_JACOBI_CTAS")) c->jacobi_ctas = std::max(0, std::atoi(v));
    if (const char* v = std::getenv("RCB200_JACOBI_THREADS")) {
        // whole warps, 64 to 1024
        const int t = std::atoi(v) / 32 * 32;
        c->jacobi_threads = t >= 64 && t <= 1024 ? t : 0;
    }
    if (const char* v = std::getenv("RCB200_RM_RR")) c->rm_rr = std::atoi(v) != 0 ? 1 : 0;
    if (const char* v = std::getenv("RCB200_GRAM_C")) c->gram_c = std::atoi(v) != 0 ? 1 : 0;
    if (const char* v = std::getenv("RCB200_ROWS27W")) c->rows27w = std::atoi(v) != 0 ? 1 : 0;
    if (const char* v = std::getenv("RCB200_CORR_PAIR")) c->corr_pair = std::atoi(v) != 0 ? 1 : 0;
    if (const char* v = std::getenv("RCB200_STAGED_ROWS")) c->staged_rows = std::max(0, std::atoi(v) / 4 * 4);
    if (const char* v = std::getenv("RCB200_STAGED_STAGES")) c->staged_stages = std::max(0, std::min(4, std::atoi(v)));
    c->pf_rows = 4096;
    if (const char* v = std::getenv("RCB200_PF_ROWS")) c->pf_rows = std::max<int64_t>(0, std::atoll(v));
    if (const char* v = std::getenv("RCB200_RM_SLICES")) c->rm_slices = std::atoi(v) == 1 ? 1 : 2;
    if (const char* v = std::getenv("RCB200_RM_GROUPS")) c->rm_groups = std::max(1, std::min(64, std::atoi(v)));
    *out = c;
    return RC_OK;
}

rc_status rc_ctx_destroy(rc_ctx* ctx) {
    if (!ctx) return RC_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (rc_op* op : ctx->ops) op_release(op);
    ctx->ops.clear();
    rc_release_slots(ctx);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->host_small) cudaFreeHost(ctx->host_small);
    for (cudaEvent_t e : ctx->step_events) cudaEventDestroy(e);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return RC_OK;
}

const char* rc_ctx_last_error(const rc_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

rc_status rc_ctx_set_stream(rc_ctx* ctx, void* stream) {
    RC_CHECK_CTX(ctx);
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return RC_OK;
}

rc_status rc_ctx_synchronize(rc_ctx* ctx) {
    RC_CHECK_CTX(ctx);
    RC_CU(ctx, cudaStreamSynchronize(ctx->stream));
    return RC_OK;
}

rc_status rc_ctx_launch_count(rc_ctx* ctx, int64_t* launches, int reset) {
    if (!ctx || !launches) return RC_ERR_INVALID;
    *launches = ctx->launches;
    if (reset) ctx->launches = 0;
    return RC_OK;
}

rc_status rc_ctx_counter(rc_ctx* ctx, const char* name, int64_t* value) {
    if (!ctx || !name || !value) return RC_ERR_INVALID;
    if (!std::strcmp(name, "launches")) *value = ctx->launches;
    else if (!std::strcmp(name, "staged_launches")) *value = ctx->staged_launches;
    else if (!std::strcmp(name, "pair_launches")) *value = ctx->pair_launches;
    else if (!std::strcmp(name, "jacobi_sweeps")) *value = ctx->jacobi_sweeps;
    else return rc_fail(ctx, RC_ERR_INVALID, std::string("rc_ctx_counter: unknown counter ") + name);
    return RC_OK;
}

rc_status rc_ctx_device_bytes(rc_ctx* ctx, int64_t* bytes) {
    if (!ctx || !bytes) return RC_ERR_INVALID;
    int64_t t = ctx->op_bytes;
    for (auto& b : ctx->slots) t += (int64_t)b.bytes;
    *bytes = t;
    return RC_OK;
}

// ---------------------------------------------------------------------------------------
// Operators
// ---------------------------------------------------------------------------------------
// Operator arrays carry 64 bytes of tail padding: the staged step kernels copy 16-byte aligned
// spans of them, which may reach up to 15 bytes past the last element.
static rc_status dev_copy(rc_ctx* ctx, void** dst, const void* src, size_t bytes, rc_op* op) {
    if (cudaMalloc(dst, bytes + 64) != cudaSuccess) {
        cudaGetLastError();
        return rc_fail(ctx, RC_ERR_NOMEM, "cudaMalloc for operator storage failed");
    }
    if (bytes) RC_CU(ctx, cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
    op->bytes += (int64_t)bytes;
    ctx->op_bytes += (int64_t)bytes;
    return RC_OK;
}

rc_status rc_op_csr_create(rc_ctx* ctx, int dtype, int64_t n, int64_t nnz, const int32_t* rowptr,
                           const int32_t* colind, const void* vals, rc_op** out) {
    RC_CHECK_CTX(ctx);
    if (!out || n <= 0 || nnz < 0 || !rowptr || (nnz > 0 && (!colind || !vals)))
        return rc_fail(ctx, RC_ERR_INVALID, "rc_op_csr_create: bad arguments");
    if (dtype != RC_REAL64 && dtype != RC_COMPLEX128) return rc_fail(ctx, RC_ERR_INVALID, "bad dtype");
    if (n > 2147483647LL || nnz > 2147483647LL) return rc_fail(ctx, RC_ERR_INVALID, "CSR indices are int32");
    // structural checks on the host (the kernels do not bounds-check colind)
    if (rowptr[0] != 0 || rowptr[n] != nnz) return rc_fail(ctx, RC_ERR_INVALID, "rowptr[0] != 0 or rowptr[n] != nnz");
    int64_t max_row = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (rowptr[i + 1] < rowptr[i]) return rc_fail(ctx, RC_ERR_INVALID, "rowptr not non-decreasing");
        max_row = std::max<int64_t>(max_row, rowptr[i + 1] - rowptr[i]);
    }
    for (int64_t k = 0; k < nnz; ++k)
        if (colind[k] < 0 || colind[k] >= n) return rc_fail(ctx, RC_ERR_INVALID, "column index out of range");
    int64_t band = 0;
    std::vector<int64_t> offs;  // distinct column offsets, while there are few
    bool few = true;
    for (int64_t i = 0; i < n; ++i)
        for (int32_t k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            const int64_t o = (int64_t)colind[k] - i;
            band = std::max<int64_t>(band, o);
            if (few && std::find(offs.begin(), offs.end(), o) == offs.end()) {
                offs.push_back(o);
                few = (int)offs.size() <= rc_op::kMaxOffsets;
            }
        }
    rc_op* op = new (std::nothrow) rc_op();
    if (!op) return RC_ERR_NOMEM;
    op->ctx = ctx;
    op->dtype = dtype;
    op->kind = 0;
    op->n = n;
    op->nnz = nnz;
    op->max_row_nnz = max_row;
    op->band = band;
    if (few) {
        std::sort(offs.begin(), offs.end());
        op->n_offsets = (int)offs.size();
        for (size_t q = 0; q < offs.size(); ++q) op->offsets[q] = offs[q];
    }
    const size_t vsz = (dtype == RC_COMPLEX128 ? 16 : 8);
    rc_status st = dev_copy(ctx, (void**)&op->rowptr, rowptr, (size_t)(n + 1) * 4, op);
    if (st == RC_OK) st = dev_copy(ctx, (void**)&op->colind, colind, (size_t)nnz * 4, op);
    if (st == RC_OK) st = dev_copy(ctx, &op->vals64, vals, (size_t)nnz * vsz, op);
    if (st != RC_OK) {
        rc_op_destroy(op);
        return st;
    }
    ctx->ops.push_back(op);
    *out = op;
    return RC_OK;
}

rc_status rc_op_stencil_create(rc_ctx* ctx, int dtype, int kind, int64_t nx, int64_t ny, int64_t nz,
                               const double* diag, double offdiag, double flux, rc_op** out) {
    RC_CHECK_CTX(ctx);
    if (!out || !diag || nx < 1 || ny < 1 || nz < 1) return rc_fail(ctx, RC_ERR_INVALID, "bad stencil arguments");
    if (dtype != RC_REAL64 && dtype != RC_COMPLEX128) return rc_fail(ctx, RC_ERR_INVALID, "bad dtype");
    if (kind != RC_STENCIL_5PT_2D && kind != RC_STENCIL_7PT_3D && kind != RC_STENCIL_27PT_3D)
        return rc_fail(ctx, RC_ERR_INVALID, "stencil kind must be 5, 7 or 27");
    if (kind == RC_STENCIL_5PT_2D && nz != 1) return rc_fail(ctx, RC_ERR_INVALID, "5-point stencil needs nz == 1");
    if (kind == RC_STENCIL_27PT_3D && dtype == RC_COMPLEX128)
        return rc_fail(ctx, RC_ERR_UNSUPPORTED, "27-point stencil is real only");
    // the kernels divide row indices by nx and ny with a multiply-high (RowDiv): grids below 2^32 points
    if (nx > INT32_MAX || ny > INT32_MAX || nz > INT32_MAX || (double)nx * (double)ny * (double)nz >= 4294967296.0)
        return rc_fail(ctx, RC_ERR_UNSUPPORTED, "stencil grids must have fewer than 2^32 points");
    rc_op* op = new (std::nothrow) rc_op();
    if (!op) return RC_ERR_NOMEM;
    op->ctx = ctx;
    op->dtype = dtype;
    op->kind = 1;
    op->skind = kind;
    op->nx = nx;
    op->ny = ny;
    op->nz = nz;
    op->n = nx * ny * nz;
    op->offdiag = offdiag;
    op->flux = dtype == RC_COMPLEX128 ? flux : 0.0;
    rc_status st = dev_copy(ctx, (void**)&op->diag64, diag, (size_t)op->n * 8, op);
    if (st == RC_OK && dtype == RC_COMPLEX128) {
        std::vector<double> p64((size_t)2 * nx);
        std::vector<float> p32((size_t)2 * nx);
        const double theta = 2.0 * 3.14159265358979323846 * op->flux;
        for (int64_t x = 0; x < nx; ++x) {
            p64[2 * x] = std::cos(theta * (double)x);
            p64[2 * x + 1] = std::sin(theta * (double)x);
            p32[2 * x] = (float)p64[2 * x];
            p32[2 * x + 1] = (float)p64[2 * x + 1];
        }
        st = dev_copy(ctx, &op->phase64, p64.data(), p64.size() * sizeof(double), op);
        if (st == RC_OK) st = dev_copy(ctx, &op->phase32, p32.data(), p32.size() * sizeof(float), op);
    }
    if (st != RC_OK) {
        rc_op_destroy(op);
        return st;
    }
    ctx->ops.push_back(op);
    *out = op;
    return RC_OK;
}

rc_status rc_op_callback_create(rc_ctx* ctx, int dtype, int64_t n, rc_block_apply_fn fn, void* user, rc_op** out) {
    RC_CHECK_CTX(ctx);
    if (!out || !fn || n <= 0) return rc_fail(ctx, RC_ERR_INVALID, "bad callback operator arguments");
    if (dtype != RC_REAL64 && dtype != RC_COMPLEX128) return rc_fail(ctx, RC_ERR_INVALID, "bad dtype");
    rc_op* op = new (std::nothrow) rc_op();
    if (!op) return RC_ERR_NOMEM;
    op->ctx = ctx;
    op->dtype = dtype;
    op->kind = 2;
    op->n = n;
    op->fn = fn;
    op->user = user;
    ctx->ops.push_back(op);
    *out = op;
    return RC_OK;
}

rc_status rc_op_destroy(rc_op* op) {
    if (!op) return RC_OK;
    rc_ctx* ctx = op->ctx;
    if (ctx) {
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        ctx->op_bytes -= op->bytes;
        for (size_t i = 0; i < ctx->ops.size(); ++i)
            if (ctx->ops[i] == op) {
                ctx->ops.erase(ctx->ops.begin() + i);
                break;
            }
    }
    op_release(op);
    return RC_OK;
}

rc_status rc_op_dim(const rc_op* op, int64_t* n, int* dtype) {
    if (!op) return RC_ERR_INVALID;
    if (n) *n = op->n;
    if (dtype) *dtype = op->dtype;
    return RC_OK;
}

// ---------------------------------------------------------------------------------------
// Filter-polynomial design
// ---------------------------------------------------------------------------------------
rc_status rc_cpoly_xstar(int64_t m, double* xstar, double* upper_xstar) {
    if (m < 0) return RC_ERR_INVALID;
    rcb::CPoly cp;
    if (xstar) *xstar = cp.xstar((long)m);
    if (upper_xstar) *upper_xstar = cp.upper_xstar((long)m);
    return RC_OK;
}

rc_status rc_cpoly_star_degree(double shift, double lambda_bound, double lambda_star, int64_t degree_max,
                               int64_t* star_degree, double* star_bound) {
    if (!star_degree || !star_bound || degree_max < 1) return RC_ERR_INVALID;
    rcb::CPoly cp;
    long d = 0;
    double b = 0.0;
    cp.star_degree_and_bound(shift, lambda_bound, lambda_star, (long)degree_max, d, b);
    *star_degree = d;
    *star_bound = b;
    return RC_OK;
}

rc_status rc_cpoly_gammas(int64_t m, double lambda_max, double shift, double* gamma1, double* gamma2) {
    if (m < 0 || !gamma1 || !gamma2) return RC_ERR_INVALID;
    rcb::CPoly cp;
    const double ux = cp.upper_xstar((long)m);
    const double rhoB = lambda_max / ux + shift / ux;
    *gamma1 = -2.0 / (rhoB - 2.0 * shift);
    *gamma2 = 2.0 - (4.0 * shift) / rhoB;
    return RC_OK;
}

double rc_cpoly_pm(int64_t m, double x) { return rcb::CPoly::pm((long)m, x); }

// ---------------------------------------------------------------------------------------
// Kernel-level entry points
// ---------------------------------------------------------------------------------------
rc_status rc_spmm(rc_ctx* ctx, const rc_op* op_c, const void* X, int64_t ldx, void* Y, int64_t ldy, int64_t s,
                  const double* alpha, const double* beta) {
    RC_CHECK_CTX(ctx);
    rc_op* op = const_cast<rc_op*>(op_c);
    if (!op || !X || !Y || s < 0 || ldx < op->n || ldy < op->n || !alpha || !beta)
        return rc_fail(ctx, RC_ERR_INVALID, "rc_spmm: bad arguments");
    if (X == Y) return rc_fail(ctx, RC_ERR_INVALID, "rc_spmm: X and Y must not alias");
    rcb::StepArgs a;
    a.s = s;
    a.x = X; a.xp = P64; a.ldx = ldx;
    a.y = Y; a.yp = P64; a.ldy = ldy;
    a.alpha[0] = alpha[0];
    a.alpha[1] = op->dtype == RC_COMPLEX128 ? alpha[1] : 0.0;
    // out = alpha*A*X + beta*Y: beta*Y enters as gamma*z with z = y (in place)
    if (beta[0] != 0.0 || (op->dtype == RC_COMPLEX128 && beta[1] != 0.0)) {
        a.z = Y; a.zp = P64; a.ldz = ldy;
        a.gamma[0] = beta[0];
        a.gamma[1] = op->dtype == RC_COMPLEX128 ? beta[1] : 0.0;
    }
    a.cp = P64;
    return rcb::op_step(ctx, op, a);
}

rc_status rc_filter(rc_ctx* ctx, const rc_op* op_c, void* X, int64_t ld, int64_t s, int64_t degree,
                    int64_t repetition, double gamma1, double gamma2, int precision) {
    RC_CHECK_CTX(ctx);
    rc_op* op = const_cast<rc_op*>(op_c);
    if (!op || !X || s < 0 || ld < op->n || degree < 0 || repetition < 0)
        return rc_fail(ctx, RC_ERR_INVALID, "rc_filter: bad arguments");
    if (precision != RC_PREC_FP64 && precision != RC_PREC_MIXED)
        return rc_fail(ctx, RC_ERR_INVALID, "rc_filter: bad precision");
    void* tmp = nullptr;
    RC_TRY(rc_slot(ctx, S_T1, (size_t)op->n * (s > 0 ? s : 1) * elem_bytes(op->dtype, P64), &tmp));
    int64_t steps = 0;
    return rcb::filter_apply(ctx, op, X, ld, s, degree, repetition, gamma2 * gamma1, gamma2, precision, tmp, nullptr,
                             (size_t)op->n * (s > 0 ? s : 1) * elem_bytes(op->dtype, P64), &steps);
}

int64_t rc_rm_leading_dim(int dtype, int precision, int64_t s) {
    if ((dtype != RC_REAL64 && dtype != RC_COMPLEX128) || (precision != RC_PREC_FP64 && precision != RC_PREC_MIXED) ||
        s < 1)
        return 0;
    return rcb::rm_leading_dim(dtype, precision == RC_PREC_MIXED ? P32 : P64, s);
}

rc_status rc_filter_step_rm(rc_ctx* ctx, const rc_op* op_c, const void* x, const void* z, void* y, int64_t ld,
                            int64_t s, const double* alpha, const double* beta, const double* gamma, int precision) {
    RC_CHECK_CTX(ctx);
    rc_op* op = const_cast<rc_op*>(op_c);
    if (!op || !x || !y || s < 1 || !alpha || !beta || (z && !gamma))
        return rc_fail(ctx, RC_ERR_INVALID, "rc_filter_step_rm: bad arguments");
    if (x == y) return rc_fail(ctx, RC_ERR_INVALID, "rc_filter_step_rm: y must not alias x");
    if (precision != RC_PREC_FP64 && precision != RC_PREC_MIXED)
        return rc_fail(ctx, RC_ERR_INVALID, "rc_filter_step_rm: bad precision");
    double a[2] = {alpha[0], op->dtype == RC_COMPLEX128 ? alpha[1] : 0.0};
    double b[2] = {beta[0], op->dtype == RC_COMPLEX128 ? beta[1] : 0.0};
    double g[2] = {z ? gamma[0] : 0.0, z && op->dtype == RC_COMPLEX128 ? gamma[1] : 0.0};
    return rcb::rm_step(ctx, op, x, z, y, ld, s, a, b, g, precision);
}

rc_status rc_lanczos_bounds(rc_ctx* ctx, const rc_op* op_c, const void* v0, uint64_t seed, double tol, int which,
                            int64_t max_iter, double* lmin, double* lmax, int64_t* iters) {
    RC_CHECK_CTX(ctx);
    rc_op* op = const_cast<rc_op*>(op_c);
    if (!op || !lmin || !lmax || which < 0 || which > 2) return rc_fail(ctx, RC_ERR_INVALID, "rc_lanczos_bounds: bad arguments");
    rcb::LanczosResult r;
    RC_TRY(rcb::lanczos_bounds(ctx, op, v0, seed, tol, which, max_iter > 0 ? max_iter : 10000, &r));
    *lmin = r.lmin;
    *lmax = r.lmax;
    if (iters) *iters = r.iters;
    return RC_OK;
}

rc_status rc_cholqr(rc_ctx* ctx, int dtype, void* V, int64_t ld, int64_t n, int64_t s, int* passes) {
    RC_CHECK_CTX(ctx);
    if (!V || n < 1 || s < 1 || ld < n || (dtype != RC_REAL64 && dtype != RC_COMPLEX128))
        return rc_fail(ctx, RC_ERR_INVALID, "rc_cholqr: bad arguments");
    if (s > n) return rc_fail(ctx, RC_ERR_INVALID, "rc_cholqr: more columns than rows");
    void* tmp = nullptr;
    RC_TRY(rc_slot(ctx, S_T1, (size_t)n * s * elem_bytes(dtype, P64), &tmp));
    bool swapped = false;
    int np = 0;
    RC_TRY(rcb::cholqr(ctx, dtype, V, ld, n, s, tmp, &swapped, &np));
    if (swapped) RC_TRY(rcb::copy_cols(ctx, dtype, tmp, n, V, ld, n, s));
    if (passes) *passes = np;
    RC_CU(ctx, cudaStreamSynchronize(ctx->stream));
    return RC_OK;
}

rc_status rc_rayleigh_ritz(rc_ctx* ctx, const rc_op* op_c, void* V, void* W, int64_t ld, int64_t s, int64_t res_count,
                           double* evals, double* residuals, void* Q) {
    RC_CHECK_CTX(ctx);
    rc_op* op = const_cast<rc_op*>(op_c);
    if (!op || !V || !W || s < 1 || ld < op->n || res_count < 0 || res_count > s || !evals)
        return rc_fail(ctx, RC_ERR_INVALID, "rc_rayleigh_ritz: bad arguments");
    const int dt = op->dtype;
    const size_t esz = elem_bytes(dt, P64);
    const int64_t n = op->n;
    void *T1 = nullptr, *T2 = nullptr, *sm = nullptr;
    RC_TRY(rc_slot(ctx, S_T1, (size_t)n * s * esz, &T1));
    RC_TRY(rc_slot(ctx, S_T2, (size_t)n * s * esz, &T2));
    const size_t mat = (size_t)s * s * esz;
    RC_TRY(rc_slot(ctx, S_IO, 3 * mat + (size_t)s * 16 + 256, &sm));
    void* H = sm;
    void* Qd = (char*)sm + mat;
    double* dlam = (double*)((char*)sm + 3 * mat);
    double* dres = dlam + s;
    int* dinfo = (int*)(dres + s);
    rcb::StepArgs st;
    st.s = s;
    st.x = V; st.xp = P64; st.ldx = ld;
    st.y = W; st.yp = P64; st.ldy = ld;
    RC_TRY(rcb::op_step(ctx, op, st));
    RC_TRY(rcb::gram(ctx, dt, n, s, s, V, ld, W, ld, H, true));
    RC_TRY(rcb::small_eigh(ctx, dt, s, H, Qd, dlam, dinfo));
    rcb::XtArgs a;
    a.n = n; a.k = s; a.nc = s;
    a.X = V; a.ldx = ld;
    a.T = Qd; a.ldt = s;
    a.Y = T1; a.ldy = n;
    a.X2 = W; a.ldx2 = ld;
    a.Y2 = T2; a.ldy2 = n;
    a.lam = dlam; a.res_count = res_count; a.res = dres;
    RC_TRY(rcb::xt(ctx, dt, a));
    RC_TRY(rcb::copy_cols(ctx, dt, T1, n, V, ld, n, s));
    RC_TRY(rcb::copy_cols(ctx, dt, T2, n, W, ld, n, s));
    RC_CU(ctx, cudaMemcpyAsync(evals, dlam, s * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (residuals && res_count > 0)
        RC_CU(ctx, cudaMemcpyAsync(residuals, dres, res_count * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (Q) RC_CU(ctx, cudaMemcpyAsync(Q, Qd, mat, cudaMemcpyDeviceToHost, ctx->stream));
    RC_CU(ctx, cudaStreamSynchronize(ctx->stream));
    return RC_OK;
}

rc_status rc_small_eigh(rc_ctx* ctx, int dtype, int64_t s, const void* H, double* evals, void* Q) {
    RC_CHECK_CTX(ctx);
    if (s < 1 || !H || !evals || (dtype != RC_REAL64 && dtype != RC_COMPLEX128))
        return rc_fail(ctx, RC_ERR_INVALID, "rc_small_eigh: bad arguments");
    const size_t mat = (size_t)s * s * elem_bytes(dtype, P64);
    void* sm = nullptr;
    RC_TRY(rc_slot(ctx, S_SMALL, 3 * mat + (size_t)s * 8 + 256, &sm));
    void* Hd = sm;
    void* Qd = (char*)sm + mat;
    double* dl = (double*)((char*)sm + 3 * mat);
    int* di = (int*)(dl + s);
    RC_CU(ctx, cudaMemcpyAsync(Hd, H, mat, cudaMemcpyHostToDevice, ctx->stream));
    RC_TRY(rcb::small_eigh(ctx, dtype, s, Hd, Qd, dl, di));
    RC_CU(ctx, cudaMemcpyAsync(evals, dl, s * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (Q) RC_CU(ctx, cudaMemcpyAsync(Q, Qd, mat, cudaMemcpyDeviceToHost, ctx->stream));
    int sweeps = 0;
    RC_CU(ctx, cudaMemcpyAsync(&sweeps, di, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    RC_CU(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->jacobi_sweeps = sweeps;
    return RC_OK;
}

void rc_solve_params_default(rc_solve_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->struct_size = sizeof(rc_solve_params);
    p->eig_count = 1;
    p->tol = 1e-10;
    p->subspace_increment = 1;
    p->buffer_size = 8;
    p->stop_condition = RC_STOP_COMBINATION;
    p->precision = RC_PREC_FP64;
    p->poly_degree_max = 200;
    p->filter_repetition = 1;
    p->max_inner_loop = 10000;
    p->max_min_tol = 1e-6;
    p->lanczos_max_iter = 10000;
    p->mode = 0;
    p->seed = 3141592;
    p->mixed_switch_tol = 0.0;  // by operator: correction filter at once, FP64 filter at 1e-6
}

rc_status rc_solve(rc_ctx* ctx, const rc_op* op_c, const rc_solve_params* params, const void* v0, double* evals_out,
                   void* evecs_out, double* residuals_out, rc_solve_info* info) {
    RC_CHECK_CTX(ctx);
    rc_op* op = const_cast<rc_op*>(op_c);
    if (!op || !params) return rc_fail(ctx, RC_ERR_INVALID, "rc_solve: null operator or params");
    rc_solve_params p;
    rc_solve_params_default(&p);
    const size_t sz = params->struct_size ? params->struct_size : sizeof(rc_solve_params);
    std::memcpy(&p, params, sz < sizeof(p) ? sz : sizeof(p));
    if (!(p.tol > 0.0)) return rc_fail(ctx, RC_ERR_INVALID, "rc_solve: tol must be positive");
    if (p.precision != RC_PREC_FP64 && p.precision != RC_PREC_MIXED)
        return rc_fail(ctx, RC_ERR_INVALID, "rc_solve: bad precision");
    if (p.stop_condition < 0 || p.stop_condition > 3) return rc_fail(ctx, RC_ERR_INVALID, "rc_solve: bad stop condition");
    return rcb::solve(ctx, op, p, v0, evals_out, evecs_out, residuals_out, info);
}

}  // extern "C"
