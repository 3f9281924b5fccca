/* rc_b200_rc.h -- the per-vector solver interface of RayleighChebyshev
 * (RayleighChebyshev.h:210-833 of almaeder/RayleighChebyshevGPGPU) over the C ABI of rc_b200.h, so a
 * caller of the CPU template is served by the GPU solver.
 *
 * A caller of the reference replaces
 *     #include "RayleighChebyshev.h"
 *     RayleighChebyshev<Vtype, Otype, VRandomizeOpType, Dtype> rc;
 * with
 *     #include "rc_b200_rc.h"
 *     rcb200::RayleighChebyshev<Vtype, Otype, VRandomizeOpType, Dtype> rc;
 * and keeps its vector class, operator and randomize op. The entry points keep the reference's names,
 * argument order and meaning, with the eigenvectors returned as std::vector<Vtype>:
 * getMinEigenSystem (:709, :728) and getMinIntervalEigenSystem (:761, :812). The setters and getters
 * are those of :279-470; the ones that only steer the CPU implementation are accepted and ignored.
 *
 * The vector class must hold its n values contiguously: VectorAccess<Vtype>::data (rc_b200_lmcuda.h)
 * reads the public std::vector vData of AvectorClassLMCuda or data() of a std::vector-like class;
 * specialise it for other layouts. Vtype is otherwise used through its copy constructor, as the
 * reference's own std::vector<Vtype> storage does, and getDimension().
 *
 * Operators:
 *   - rcb200::CsrOperator<Dtype> and rcb200::StencilOperator (rc_b200_lmcuda.h) are seen by the fused
 *     sm_100a kernels;
 *   - any other Otype is called through its host apply(Vtype& v), v <- A v (RayleighChebyshev.h:59),
 *     once per column: the library copies each filter step's block to the host, applies the operator
 *     column by column and copies the result back. This keeps any operator working, at host speed.
 * Randomize op: randomize(Vtype&) fills every start, refresh and Lanczos vector
 * (RayleighChebyshev.h:69).
 *
 * Errors throw std::runtime_error, as the reference does.
 */
#pragma once

#include "rc_b200_lmcuda.h"

#include <algorithm>
#include <cctype>
#include <cstring>
#include <iosfwd>
#include <map>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

namespace rcb200 {

template <class Vtype, class Otype, class VRandomizeOpType, typename Dtype = double>
class RayleighChebyshev {
public:
    explicit RayleighChebyshev(int device = 0) {
        if (rc_ctx_create(device, &ctx_) != RC_OK) throw std::runtime_error("rc_ctx_create failed");
        rc_solve_params_default(&p_);
        p_.stop_condition = RC_STOP_COMBINATION;
    }
    ~RayleighChebyshev() {
        if (ctx_) rc_ctx_destroy(ctx_);
    }
    RayleighChebyshev(const RayleighChebyshev&) = delete;
    RayleighChebyshev& operator=(const RayleighChebyshev&) = delete;

    // ---- setters (RayleighChebyshev.h:279-440) ----
    // stop condition names are case-insensitive, as in the reference (:279-307)
    void setStopCondition(std::string s) {
        std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return (char)std::toupper(c); });
        if (s == "COMBINATION" || s == "DEFAULT") p_.stop_condition = RC_STOP_COMBINATION;
        else if (s == "EIGENVALUE_ONLY") p_.stop_condition = RC_STOP_EIGENVALUE_ONLY;
        else if (s == "RESIDUAL_ONLY") p_.stop_condition = RC_STOP_RESIDUAL_ONLY;
        else throw std::runtime_error("RayleighChebyshev: unknown stopping condition " + s);
    }
    // the enum form (:309-338)
    template <class E, typename std::enable_if<std::is_enum<E>::value, int>::type = 0>
    void setStopCondition(E e) { p_.stop_condition = stop_condition_value(e); }
    void setMaxMinTolerance(double val = 1.0e-6) { p_.max_min_tol = val; }
    void setMaxInnerLoopCount(long val) { p_.max_inner_loop = val; }
    void setNonRandomStartFlag(bool val = true) { nonRandomStart_ = val; }
    void setVerboseFlag(bool val = true) { p_.verbose = val ? 1 : 0; }
    void setMinIntervalPolyDegreeMax(long polyDegMax) { p_.poly_degree_max = polyDegMax; }
    void setFilterRepetitionCount(long repetitionCount) { p_.filter_repetition = repetitionCount; }
    void setMaxSpectralBoundsIter(long iterCount) { p_.lanczos_max_iter = iterCount; }
    // a fixed inner iteration count (:352, :1083) is not offered by the GPU solver
    void setFixedIterationCount(bool val) {
        if (val) throw std::runtime_error("RayleighChebyshev: fixed iteration counts are not supported");
    }
    // CPU-implementation switches, accepted for source compatibility: the GPU solver has one small
    // eigensolver (Jacobi on the device), prints its verbose lines to stdout and keeps no per-subspace
    // or eigen-diagnostic output
    void setVerboseSubspaceFlag(bool = true) {}
    void setEigDiagnosticsFlag(bool = true) {}
    void setUseJacobi(bool) {}
    void setResultsStream(std::ostream&) {}
    // the interval stop rules (:402-420): each entry point selects its own, as the reference's entry
    // points set them, so the toggles are accepted and have no effect
    void setIntervalStopCondition(bool = true) {}
    void clearIntervalStopCondition() {}
    void setHardIntervalStop(bool = true) {}
    void clearHardIntervalStop() {}
    // no reference counterpart: FP32 / bfloat16 filter with FP64 Rayleigh-Ritz (RC_PREC_MIXED), and
    // per-phase CUDA-event timing behind getTimingData
    void setMixedPrecision(bool val = true) { p_.precision = val ? RC_PREC_MIXED : RC_PREC_FP64; }
    void setTimingFlag(bool val = true) { p_.phase_timing = val ? 1 : 0; }

    // ---- getters (:383-470) ----
    double getMinEigValueEst() const { return info_.min_eig_est; }
    double getMaxEigValueEst() const { return info_.max_eig_est; }
    double getGuardEigenvalue() const { return info_.guard_value; }
    long getSpectralBoundsIterCount() const { return (long)info_.lanczos_iterations; }
    std::vector<double> getEigVectorResiduals() const { return residuals_; }
    std::map<std::string, double> getFinalData() const {
        return {{"maxResidual", info_.max_residual},
                {"maxEigValueDifference", info_.max_eig_diff},
                {"maxRelEigValueGap", info_.max_rel_gap}};
    }
    std::map<std::string, long> getCountData() const {
        return {{"ortho", (long)info_.count_ortho},
                {"OpApply", (long)info_.count_opapply},
                {"eigenvalue", (long)info_.count_eigenvalue}};
    }
    // CUDA-event milliseconds per phase (setTimingFlag), where the reference reports wall-clock seconds
    std::map<std::string, double> getTimingData() const {
        return {{"ortho", info_.time_ortho_ms},
                {"OpApply", info_.time_filter_ms},
                {"eigenvalue", info_.time_eigenvalue_ms},
                {"totalTime", info_.time_total_ms}};
    }
    const rc_solve_info& getSolveInfo() const { return info_; }

    // ---- entry points ----
    // getMinEigenSystem(eigCount, minEigValueEst, maxEigValueBound, ...) (:709)
    long getMinEigenSystem(long eigCount, double minEigValueEst, double maxEigValueBound, double subspaceTol,
                           long subspaceIncrementSize, long bufferSize, Vtype& vStart, Otype& oP,
                           VRandomizeOpType& randOp, std::vector<double>& eigValues, std::vector<Vtype>& eigVectors) {
        return run(1, eigCount, minEigValueEst, maxEigValueBound, 0.0, subspaceTol, subspaceIncrementSize, bufferSize,
                   vStart, oP, randOp, eigValues, eigVectors);
    }
    // getMinEigenSystem(eigCount, subspaceTol, ...) (:728): spectral bounds by Lanczos first
    long getMinEigenSystem(long eigCount, double subspaceTol, long subspaceIncrementSize, long bufferSize,
                           Vtype& vStart, Otype& oP, VRandomizeOpType& randOp, std::vector<double>& eigValues,
                           std::vector<Vtype>& eigVectors) {
        return run(0, eigCount, 0.0, 0.0, 0.0, subspaceTol, subspaceIncrementSize, bufferSize, vStart, oP, randOp,
                   eigValues, eigVectors);
    }
    // getMinIntervalEigenSystem(lambdaMax, ...) (:761)
    long getMinIntervalEigenSystem(double lambdaMax, double subspaceTol, long subspaceIncrementSize, long bufferSize,
                                   long maxEigensystemDim, Vtype& vStart, Otype& oP, VRandomizeOpType& randOp,
                                   std::vector<double>& eigValues, std::vector<Vtype>& eigVectors) {
        return run(2, maxEigensystemDim, 0.0, 0.0, lambdaMax, subspaceTol, subspaceIncrementSize, bufferSize, vStart,
                   oP, randOp, eigValues, eigVectors);
    }
    // getMinIntervalEigenSystem(minEigValueEst, lambdaMax, maxEigValueBound, ...) (:812)
    long getMinIntervalEigenSystem(double minEigValueEst, double lambdaMax, double maxEigValueBound,
                                   double subspaceTol, long subspaceIncrementSize, long bufferSize,
                                   long maxEigensystemDim, Vtype& vStart, Otype& oP, VRandomizeOpType& randOp,
                                   std::vector<double>& eigValues, std::vector<Vtype>& eigVectors) {
        return run(3, maxEigensystemDim, minEigValueEst, maxEigValueBound, lambdaMax, subspaceTol,
                   subspaceIncrementSize, bufferSize, vStart, oP, randOp, eigValues, eigVectors);
    }

private:
    struct Binding {
        Otype* op;
        VRandomizeOpType* rand;
        const Vtype* proto;  // a vector of the problem's dimension, copied for scratch vectors
        long n;
        std::vector<Dtype> host;
        int failed = 0;
    };

    static Dtype* values(Vtype& v) { return static_cast<Dtype*>(VectorAccess<Vtype>::data(v)); }

    static Dtype scalar(const double* v) {
        if constexpr (std::is_same<Dtype, double>::value) return v[0];
        else return Dtype(v[0], v[1]);
    }

    // out = alpha A in + beta out on the device block (ld == n): the host operator, column by column
    static int apply_tramp(void* user, const void* in, void* out, int64_t n, int64_t s, int64_t ld,
                           const double* alpha, const double* beta, void* stream) {
        auto* b = static_cast<Binding*>(user);
        if (ld != n || n != b->n) return 1;
        const auto st = static_cast<cudaStream_t>(stream);
        const size_t bytes = (size_t)n * (size_t)s * sizeof(Dtype);
        b->host.resize(2 * (size_t)n * (size_t)s);
        Dtype* hin = b->host.data();
        Dtype* hout = hin + (size_t)n * s;
        const Dtype a = scalar(alpha), bt = scalar(beta);
        const bool useOut = bt != Dtype(0);
        if (cudaMemcpyAsync(hin, in, bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess) return 1;
        if (useOut && cudaMemcpyAsync(hout, out, bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess) return 1;
        if (cudaStreamSynchronize(st) != cudaSuccess) return 1;
        try {
            Vtype v(*b->proto);
            Dtype* vd = values(v);
            for (int64_t c = 0; c < s; ++c) {
                std::memcpy(vd, hin + c * n, (size_t)n * sizeof(Dtype));
                b->op->apply(v);
                Dtype* oc = hout + c * n;
                for (int64_t i = 0; i < n; ++i) oc[i] = useOut ? a * vd[i] + bt * oc[i] : a * vd[i];
            }
        } catch (...) {
            return 1;
        }
        if (cudaMemcpyAsync(out, hout, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) return 1;
        return cudaStreamSynchronize(st) == cudaSuccess ? 0 : 1;
    }

    // start and refresh blocks, one randomize(Vtype&) per column
    static void randomize_tramp(void* user, void* host_block, int64_t n, int64_t s) {
        auto* b = static_cast<Binding*>(user);
        try {
            Vtype v(*b->proto);
            for (int64_t c = 0; c < s; ++c) {
                b->rand->randomize(v);
                std::memcpy(static_cast<Dtype*>(host_block) + c * n, values(v), (size_t)n * sizeof(Dtype));
            }
        } catch (...) {
            b->failed = 1;
        }
    }

    void check(rc_status st, const char* what) const {
        if (st != RC_OK) throw std::runtime_error(std::string(what) + ": " + rc_ctx_last_error(ctx_));
    }

    rc_op* make_op(Otype& oP, long n, Binding* bind) {
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

    long run(int mode, long count, double minEst, double maxBound, double lambdaMax, double tol, long incr,
             long buffer, Vtype& vStart, Otype& oP, VRandomizeOpType& randOp, std::vector<double>& eigValues,
             std::vector<Vtype>& eigVectors) {
        const long n = (long)vStart.getDimension();
        if constexpr (std::is_same<Otype, CsrOperator<Dtype>>::value) {
            if ((long)oP.n != n) throw std::runtime_error("RayleighChebyshev: vStart and operator sizes differ");
        } else if constexpr (std::is_same<Otype, StencilOperator>::value) {
            if ((long)(oP.nx * oP.ny * oP.nz) != n)
                throw std::runtime_error("RayleighChebyshev: vStart and operator sizes differ");
        }
        Vtype lz(vStart);
        randOp.randomize(lz);  // the Lanczos start vector (LanczosMaxMinFinder.h:272)
        Binding bind{&oP, &randOp, &vStart, n, {}, 0};
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
        if (nonRandomStart_) {  // the vectors in eigVectors start the subspace
            const long cols = std::min<long>((long)eigVectors.size(), incr + buffer);
            if (cols > 0) {
                start.resize((size_t)n * cols);
                for (long c = 0; c < cols; ++c) {
                    if ((long)eigVectors[c].getDimension() != n) {
                        rc_op_destroy(op);
                        throw std::runtime_error("RayleighChebyshev: start vector of the wrong size");
                    }
                    std::memcpy(start.data() + (size_t)c * n, values(eigVectors[c]), (size_t)n * sizeof(Dtype));
                }
                p.non_random_start = 1;
                p.v0_cols = cols;
            }
        }
        const long cap = std::max<long>(count > 0 ? count : n, 1);
        std::vector<double> evals((size_t)cap), res((size_t)cap);
        std::vector<Dtype> evecs((size_t)n * cap);
        info_ = rc_solve_info();
        info_.struct_size = sizeof(rc_solve_info);
        const rc_status st = rc_solve(ctx_, op, &p, start.empty() ? nullptr : start.data(), evals.data(),
                                      evecs.data(), res.data(), &info_);
        rc_op_destroy(op);
        check(st, "rc_solve");
        if (bind.failed) throw std::runtime_error("RayleighChebyshev: the randomize op failed");
        const long found = (long)info_.found;
        eigValues.assign(evals.begin(), evals.begin() + found);
        residuals_.assign(res.begin(), res.begin() + found);
        eigVectors.assign((size_t)found, vStart);
        for (long c = 0; c < found; ++c)
            std::memcpy(values(eigVectors[c]), evecs.data() + (size_t)c * n, (size_t)n * sizeof(Dtype));
        return found;
    }

    rc_ctx* ctx_ = nullptr;
    rc_solve_params p_;
    rc_solve_info info_{};
    bool nonRandomStart_ = false;
    std::vector<double> residuals_;
};

}  // namespace rcb200
