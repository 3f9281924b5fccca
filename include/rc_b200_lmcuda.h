/* rc_b200_lmcuda.h -- the templated solver interface of RayleighChebyshevLMCuda
 * (RayleighChebyshevLMCuda.h:220-564 of almaeder/RayleighChebyshevGPGPU) over the C ABI of rc_b200.h.
 *
 * A caller of the reference replaces
 *     #include "RayleighChebyshevLMCuda.h"
 *     RayleighChebyshevLMCuda<Atype, Vtype, Otype, VRandomizeOpType, Dtype> rc;
 * with
 *     #include "rc_b200_lmcuda.h"
 *     rcb200::RayleighChebyshevLMCuda<Atype, Vtype, Otype, VRandomizeOpType, Dtype> rc;
 * and keeps its containers (AmatrixClassLMCuda / AvectorClassLMCuda or its own), its operator and its
 * randomize op. The entry points, setters and getters keep the reference's names, argument order and
 * meaning (getMinEigenSystem :775, :794; getMinIntervalEigenSystem :827, :876; setters :340-532;
 * getters :534-560). Results are returned in host eigVectors.mData (and on the device when the
 * container has host_to_device()), as in the reference.
 *
 * Operators:
 *   - rcb200::CsrOperator<Dtype> and rcb200::StencilOperator are seen by the fused sm_100a kernels;
 *   - any other Otype is called through its device block apply(Atype& in, Atype& out, Dtype alpha,
 *     Dtype beta), out = alpha*A*in + beta*out (LanczosCpolyOperatorLMCuda.h:245), on views of the
 *     library's column-major device blocks (BlockAccess below). The library synchronises the device
 *     around each call, so the operator may use any stream. The spectral bounds use the same block
 *     apply on one column, where the reference calls the operator's host apply(Vtype&).
 * Randomize op: randomize(Atype&) fills the start and refresh blocks on the host (RayleighChebyshevLMCuda.h
 * :1046, :1178), randomize(Vtype&) the Lanczos start vector (LanczosMaxMinFinder.h:272).
 *
 * Errors throw std::runtime_error (the reference throws, or exits on CUDA errors).
 */
#pragma once

#include <algorithm>
#include <complex>
#include <cstdint>
#include <cstring>
#include <iosfwd>
#include <map>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include <cuda_runtime.h>
#if __has_include(<cusparse.h>)
#include <cusparse.h>
#define RCB200_HAVE_CUSPARSE 1
#endif

#include "rc_b200.h"

#ifndef RAY_INT
#define RAY_INT long
#endif

namespace rcb200 {

/* The stop-condition names of the reference's RC_Types.h, in the order of RC_STOP_*. */
struct RC_Types {
    enum StopCondition { DEFAULT, COMBINATION, EIGENVALUE_ONLY, RESIDUAL_ONLY };
};

/* The RC_STOP_* value of a StopCondition enumerator (this header's RC_Types, or the reference's
 * global RC_Types when the caller still includes RC_Types.h): DEFAULT means COMBINATION. */
template <class E>
inline int stop_condition_value(E e) {
    static_assert(std::is_enum<E>::value, "a StopCondition enumerator");
    const int v = (int)e;
    if (v < RC_STOP_DEFAULT || v > RC_STOP_RESIDUAL_ONLY) throw std::runtime_error("setStopCondition: unknown stop condition");
    return v == RC_STOP_DEFAULT ? RC_STOP_COMBINATION : v;
}

template <class D> struct dtype_of;
template <> struct dtype_of<double> { static constexpr int value = RC_REAL64; };
template <> struct dtype_of<std::complex<double>> { static constexpr int value = RC_COMPLEX128; };

/* A CSR matrix held on the host (rows rowptr[i]..rowptr[i+1]-1), Hermitian. */
template <typename Dtype = double>
struct CsrOperator {
    RAY_INT n = 0;
    std::vector<int32_t> rowptr, colind;
    std::vector<Dtype> vals;
};

/* The matrix-free Dirichlet stencil of rc_op_stencil_create (kind 5, 7 or 27). */
struct StencilOperator {
    int kind = RC_STENCIL_7PT_3D;
    RAY_INT nx = 1, ny = 1, nz = 1;
    std::vector<double> diag;
    double offdiag = -1.0;
    double flux = 0.0;
};

namespace detail {
template <class T, class = void> struct has_vData : std::false_type {};
template <class T> struct has_vData<T, std::void_t<decltype(std::declval<T&>().vData)>> : std::true_type {};
template <class T, class = void> struct has_matrix_desc : std::false_type {};
template <class T> struct has_matrix_desc<T, std::void_t<decltype(std::declval<T&>().matrix_desc)>> : std::true_type {};
template <class T, class = void> struct has_create_desc : std::false_type {};
template <class T>
struct has_create_desc<T, std::void_t<decltype(std::declval<T&>().create_cuda_descriptor())>> : std::true_type {};
template <class T, class = void> struct has_host_to_device : std::false_type {};
template <class T>
struct has_host_to_device<T, std::void_t<decltype(std::declval<T&>().host_to_device())>> : std::true_type {};
}  // namespace detail

/* Access to a vector container: AvectorClassLMCuda keeps its values in the public std::vector vData.
 * Specialise for other containers. */
template <class Vtype>
struct VectorAccess {
    static void* data(Vtype& v) {
        if constexpr (detail::has_vData<Vtype>::value) return (void*)v.vData.data();
        else return (void*)v.data();
    }
};

/* Access to a block container: AmatrixClassLMCuda is column-major with public m (rows), n (columns),
 * host values mData and device values mData_d, and a cuSPARSE dense-matrix descriptor matrix_desc
 * that its users' operators read. attach() makes a container a view of a device block, detach()
 * releases the view without freeing the block. Specialise for other containers. */
template <class Atype>
struct BlockAccess {
    static void attach(Atype& a, void* dptr, RAY_INT rows, RAY_INT cols) {
        a.m = rows;
        a.n = cols;
        a.mData_d = static_cast<decltype(a.mData_d)>(dptr);
        if constexpr (detail::has_create_desc<Atype>::value) a.create_cuda_descriptor();
    }
    static void detach(Atype& a) {
        if constexpr (detail::has_matrix_desc<Atype>::value) {
#ifdef RCB200_HAVE_CUSPARSE
            if (a.matrix_desc != nullptr) cusparseDestroyDnMat(a.matrix_desc);
#endif
            a.matrix_desc = nullptr;
        }
        a.mData_d = nullptr;
    }
    static void host_resize(Atype& a, RAY_INT rows, RAY_INT cols) { a.resize(rows, cols); }
    static void* host_data(Atype& a) { return (void*)a.mData.data(); }
    static void to_device(Atype& a) {
        if constexpr (detail::has_host_to_device<Atype>::value) a.host_to_device();
    }
};

template <class Atype, class Vtype, class Otype, class VRandomizeOpType, typename Dtype = double>
class RayleighChebyshevLMCuda {
public:
    explicit RayleighChebyshevLMCuda(int device = 0) {
        if (rc_ctx_create(device, &ctx_) != RC_OK) throw std::runtime_error("rc_ctx_create failed");
        rc_solve_params_default(&p_);
        p_.stop_condition = RC_STOP_COMBINATION;
    }
    ~RayleighChebyshevLMCuda() {
        if (ctx_) rc_ctx_destroy(ctx_);
    }
    RayleighChebyshevLMCuda(const RayleighChebyshevLMCuda&) = delete;
    RayleighChebyshevLMCuda& operator=(const RayleighChebyshevLMCuda&) = delete;

    // ---- setters (RayleighChebyshevLMCuda.h:340-532) ----
    void setStopCondition(const std::string& s) {
        if (s == "COMBINATION" || s == "DEFAULT") p_.stop_condition = RC_STOP_COMBINATION;
        else if (s == "EIGENVALUE_ONLY") p_.stop_condition = RC_STOP_EIGENVALUE_ONLY;
        else if (s == "RESIDUAL_ONLY") p_.stop_condition = RC_STOP_RESIDUAL_ONLY;
        else throw std::runtime_error("setStopCondition: unknown stop condition " + s);
    }
    // the enum form (:370-395)
    template <class E, typename std::enable_if<std::is_enum<E>::value, int>::type = 0>
    void setStopCondition(E e) { p_.stop_condition = stop_condition_value(e); }
    void setMaxMinTolerance(double val = 1.0e-6) { p_.max_min_tol = val; }
    void setMaxInnerLoopCount(RAY_INT val) { p_.max_inner_loop = val; }
    // a fixed inner iteration count (:419) is not offered by the GPU solver
    void setFixedIterationCount(bool val) {
        if (val) throw std::runtime_error("setFixedIterationCount: fixed iteration counts are not supported");
    }
    void setNonRandomStartFlag(bool val = true) { nonRandomStart_ = val; }
    void setVerboseFlag(bool val = true) { p_.verbose = val ? 1 : 0; }
    void setMinIntervalPolyDegreeMax(RAY_INT polyDegMax) { p_.poly_degree_max = polyDegMax; }
    void setFilterRepetitionCount(RAY_INT repetitionCount) { p_.filter_repetition = repetitionCount; }
    void setMaxSpectralBoundsIter(RAY_INT iterCount) { p_.lanczos_max_iter = iterCount; }
    // Host-implementation switches, accepted for source compatibility: the small eigensolve is always
    // the GPU Jacobi, verbose lines go to stdout, and there is no per-subspace or eigen-diagnostic output.
    void setVerboseSubspaceFlag(bool = true) {}
    void setEigDiagnosticsFlag(bool = true) {}
    void setUseJacobi(bool) {}
    void setResultsStream(std::ostream&) {}
    // The interval stop rules (:494-512): each entry point here selects its own, as the reference's
    // entry points set them (getMinEigenSystem: hard stop at the bound; getMinIntervalEigenSystem: the
    // guard-eigenvalue test), so the toggles are accepted and have no effect.
    void setIntervalStopCondition(bool = true) {}
    void clearIntervalStopCondition() {}
    void setHardIntervalStop(bool = true) {}
    void clearHardIntervalStop() {}
    // no reference counterpart: FP32 filter with FP64 Rayleigh-Ritz (RC_PREC_MIXED), and the
    // per-phase CUDA-event timing behind getTimingData
    void setMixedPrecision(bool val = true) { p_.precision = val ? RC_PREC_MIXED : RC_PREC_FP64; }
    void setTimingFlag(bool val = true) { p_.phase_timing = val ? 1 : 0; }

    // ---- entry points ----
    // getMinEigenSystem(eigCount, subspaceTol, ...) (RayleighChebyshevLMCuda.h:794)
    RAY_INT getMinEigenSystem(RAY_INT eigCount, double subspaceTol, RAY_INT subspaceIncrementSize, RAY_INT bufferSize,
                              Vtype& vStart, Otype& oP, VRandomizeOpType& randOp, std::vector<double>& eigValues,
                              Atype& eigVectors) {
        return run(0, eigCount, 0.0, 0.0, 0.0, subspaceTol, subspaceIncrementSize, bufferSize, vStart, oP, randOp,
                   eigValues, eigVectors);
    }
    // getMinEigenSystem(eigCount, minEigValueEst, maxEigValueBound, ...) (:775)
    RAY_INT getMinEigenSystem(RAY_INT eigCount, double minEigValueEst, double maxEigValueBound, double subspaceTol,
                              RAY_INT subspaceIncrementSize, RAY_INT bufferSize, Vtype& vStart, Otype& oP,
                              VRandomizeOpType& randOp, std::vector<double>& eigValues, Atype& eigVectors) {
        return run(1, eigCount, minEigValueEst, maxEigValueBound, 0.0, subspaceTol, subspaceIncrementSize, bufferSize,
                   vStart, oP, randOp, eigValues, eigVectors);
    }
    // getMinIntervalEigenSystem(lambdaMax, ...) (:827)
    RAY_INT getMinIntervalEigenSystem(double lambdaMax, double subspaceTol, RAY_INT subspaceIncrementSize,
                                      RAY_INT bufferSize, RAY_INT maxEigensystemDim, Vtype& vStart, Otype& oP,
                                      VRandomizeOpType& randOp, std::vector<double>& eigValues, Atype& eigVectors) {
        return run(2, maxEigensystemDim, 0.0, 0.0, lambdaMax, subspaceTol, subspaceIncrementSize, bufferSize, vStart,
                   oP, randOp, eigValues, eigVectors);
    }
    // getMinIntervalEigenSystem(minEigValueEst, lambdaMax, maxEigValueBound, ...) (:876)
    RAY_INT getMinIntervalEigenSystem(double minEigValueEst, double lambdaMax, double maxEigValueBound,
                                      double subspaceTol, RAY_INT subspaceIncrementSize, RAY_INT bufferSize,
                                      RAY_INT maxEigensystemDim, Vtype& vStart, Otype& oP, VRandomizeOpType& randOp,
                                      std::vector<double>& eigValues, Atype& eigVectors) {
        return run(3, maxEigensystemDim, minEigValueEst, maxEigValueBound, lambdaMax, subspaceTol,
                   subspaceIncrementSize, bufferSize, vStart, oP, randOp, eigValues, eigVectors);
    }

    // ---- getters (:469-478, :489, :519, :534-560) ----
    double getMinEigValueEst() const { return info_.min_eig_est; }
    double getMaxEigValueEst() const { return info_.max_eig_est; }
    RAY_INT getSpectralBoundsIterCount() const { return (RAY_INT)info_.lanczos_iterations; }
    double getGuardEigenvalue() const { return info_.guard_value; }
    std::vector<double> getEigVectorResiduals() const { return residuals_; }
    std::map<std::string, double> getFinalData() const {
        return {{"maxResidual", info_.max_residual},
                {"maxEigValueDifference", info_.max_eig_diff},
                {"maxRelEigValueGap", info_.max_rel_gap}};
    }
    std::map<std::string, RAY_INT> getCountData() const {
        return {{"ortho", (RAY_INT)info_.count_ortho},
                {"OpApply", (RAY_INT)info_.count_opapply},
                {"eigenvalue", (RAY_INT)info_.count_eigenvalue}};
    }
    // CUDA-event milliseconds per phase (setTimingFlag), where the reference reports wall-clock
    // seconds under TIMING_ (:2342-2381)
    std::map<std::string, double> getTimingData() const {
        return {{"ortho", info_.time_ortho_ms},
                {"OpApply", info_.time_filter_ms},
                {"eigenvalue", info_.time_eigenvalue_ms},
                {"totalTime", info_.time_total_ms}};
    }
    const rc_solve_info& getSolveInfo() const { return info_; }

private:
    struct Binding {
        Otype* op;
        VRandomizeOpType* rand;
        RAY_INT n;
    };

    static Dtype scalar(const double* v) {
        if constexpr (std::is_same<Dtype, double>::value) return v[0];
        else return Dtype(v[0], v[1]);
    }

    static int apply_tramp(void* user, const void* in, void* out, int64_t n, int64_t s, int64_t ld,
                           const double* alpha, const double* beta, void* stream) {
        auto* b = static_cast<Binding*>(user);
        if (ld != n) return 1;
        if (cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) != cudaSuccess) return 1;
        int rc = 0;
        Atype vin, vout;
        BlockAccess<Atype>::attach(vin, const_cast<void*>(in), (RAY_INT)n, (RAY_INT)s);
        BlockAccess<Atype>::attach(vout, out, (RAY_INT)n, (RAY_INT)s);
        try {
            b->op->apply(vin, vout, scalar(alpha), scalar(beta));
        } catch (...) {
            rc = 1;
        }
        BlockAccess<Atype>::detach(vin);
        BlockAccess<Atype>::detach(vout);
        if (cudaDeviceSynchronize() != cudaSuccess) rc = 1;
        return rc;
    }

    static void randomize_tramp(void* user, void* host_block, int64_t n, int64_t s) {
        auto* b = static_cast<Binding*>(user);
        Atype tmp;
        BlockAccess<Atype>::host_resize(tmp, (RAY_INT)n, (RAY_INT)s);
        b->rand->randomize(tmp);
        std::memcpy(host_block, BlockAccess<Atype>::host_data(tmp), (size_t)n * s * sizeof(Dtype));
    }

    void check(rc_status st, const char* what) const {
        if (st != RC_OK) throw std::runtime_error(std::string(what) + ": " + rc_ctx_last_error(ctx_));
    }

    rc_op* make_op(Otype& oP, RAY_INT n, Binding* bind) {
        rc_op* op = nullptr;
        constexpr int dt = dtype_of<Dtype>::value;
        if constexpr (std::is_same<Otype, CsrOperator<Dtype>>::value) {
            check(rc_op_csr_create(ctx_, dt, oP.n, (int64_t)oP.colind.size(), oP.rowptr.data(), oP.colind.data(),
                                   oP.vals.data(), &op),
                  "rc_op_csr_create");
        } else if constexpr (std::is_same<Otype, StencilOperator>::value) {
            check(rc_op_stencil_create(ctx_, dt, oP.kind, oP.nx, oP.ny, oP.nz, oP.diag.data(), oP.offdiag, oP.flux,
                                       &op),
                  "rc_op_stencil_create");
        } else {
            check(rc_op_callback_create(ctx_, dt, n, &apply_tramp, bind, &op), "rc_op_callback_create");
        }
        return op;
    }

    RAY_INT run(int mode, RAY_INT count, double minEst, double maxBound, double lambdaMax, double tol, RAY_INT incr,
                RAY_INT buffer, Vtype& vStart, Otype& oP, VRandomizeOpType& randOp, std::vector<double>& eigValues,
                Atype& eigVectors) {
        Vtype lz(vStart);
        randOp.randomize(lz);  // the Lanczos start vector, as LanczosMaxMinFinder.h:272
        const RAY_INT n = [&] {
            if constexpr (std::is_same<Otype, CsrOperator<Dtype>>::value) return (RAY_INT)oP.n;
            else if constexpr (std::is_same<Otype, StencilOperator>::value) return (RAY_INT)(oP.nx * oP.ny * oP.nz);
            else return (RAY_INT)vStart.getDimension();
        }();
        Binding bind{&oP, &randOp, n};
        rc_op* op = make_op(oP, n, &bind);
        rc_solve_params p = p_;
        p.mode = mode;
        p.eig_count = count;
        p.min_eig_est = minEst;
        p.max_eig_bound = maxBound;
        p.lambda_max = lambdaMax;
        p.tol = tol;
        p.subspace_increment = incr;
        p.buffer_size = buffer;
        p.host_buffers = 1;
        p.randomize_fn = &randomize_tramp;
        p.randomize_user = &bind;
        p.lanczos_v0 = VectorAccess<Vtype>::data(lz);
        std::vector<Dtype> start;
        if (nonRandomStart_) {  // the columns of eigVectors start the subspace (:1048-1070)
            const RAY_INT cols = std::min<RAY_INT>((RAY_INT)eigVectors.getColSize(), incr + buffer);
            if (cols > 0) {
                start.resize((size_t)n * cols);
                std::memcpy(start.data(), BlockAccess<Atype>::host_data(eigVectors), start.size() * sizeof(Dtype));
                p.non_random_start = 1;
                p.v0_cols = cols;
            }
        }
        const RAY_INT cap = std::max<RAY_INT>(count > 0 ? count : n, 1);
        std::vector<double> evals((size_t)cap), res((size_t)cap);
        std::vector<Dtype> evecs((size_t)n * cap);
        info_ = rc_solve_info();
        info_.struct_size = sizeof(rc_solve_info);
        const rc_status st = rc_solve(ctx_, op, &p, start.empty() ? nullptr : start.data(), evals.data(),
                                      evecs.data(), res.data(), &info_);
        rc_op_destroy(op);
        check(st, "rc_solve");
        const RAY_INT found = (RAY_INT)info_.found;
        eigValues.assign(evals.begin(), evals.begin() + found);
        residuals_.assign(res.begin(), res.begin() + found);
        BlockAccess<Atype>::host_resize(eigVectors, n, found);
        if (found > 0) {
            std::memcpy(BlockAccess<Atype>::host_data(eigVectors), evecs.data(), (size_t)n * found * sizeof(Dtype));
            BlockAccess<Atype>::to_device(eigVectors);
        }
        return found;
    }

    rc_ctx* ctx_ = nullptr;
    rc_solve_params p_;
    rc_solve_info info_{};
    bool nonRandomStart_ = false;
    std::vector<double> residuals_;
};

}  // namespace rcb200
