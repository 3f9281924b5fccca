// ref_harness.cpp -- ORACLE / TEST INFRASTRUCTURE ONLY.
//
// Drives the reference's own CPU code, compiled from the reference headers (RayleighChebyshevLM,
// LanczosCpolyOperatorLM, LanczosMaxMinFinder, LanczosCpoly), on problems written by the Python
// test harness. The reference ships no vector, operator or driver classes, so the minimal
// Vtype/Otype/VRandomizeOpType below are this harness's own. Built by oracle/Makefile into
// oracle/_ref/ (never committed); used by tests and by bench.py's CPU baseline only.
//
//   ref_harness solve   <problem.bin> k=16 tol=1e-10 incr=16 buffer=8 stop=RESIDUAL_ONLY [threads=N]
//   ref_harness filter  <problem.bin> degree=m bound=B shift=S reps=1 out=<file> [threads=N]
//   ref_harness lanczos <problem.bin> tol=1e-6 which=max|both
//   ref_harness phases  <problem.bin> degree=m bound=B shift=S rescheck=k [do=filter,ortho,rr] [threads=N]
//       one inner iteration of RayleighChebyshevLM on the start block, phase by phase: the filter
//       (LanczosCpolyOperatorLM::apply, degree m), then orthogonalize (modified Gram-Schmidt),
//       formVtAV + computeVtVeigensystem (Jacobi) + createEigenVectorsAndResiduals, each timed;
//       `do` selects the phases that run (default all)
//   ref_harness cpoly   mmax=200 [shift=S bound=B star=L degmax=D]
//
// problem.bin (little endian): "RCPB", int32 version=1, int64 n, nnz, s_start, has_lz0,
//   int32 rowptr[n+1], int32 colind[nnz], double vals[nnz], double start[n*s_start] (column-major),
//   double lz0[n] if has_lz0.
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <random>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "RayleighChebyshevLM.h"

class HVec {
public:
    std::vector<double> d;
    HVec() {}
    HVec(const HVec& o) : d(o.d) {}
    void initialize() { d.clear(); }
    void initialize(const HVec& o) { d = o.d; }
    HVec& operator=(const HVec& o) {
        if (this != &o) d = o.d;
        return *this;
    }
    void operator+=(const HVec& o) {
        const long n = (long)d.size();
#pragma omp parallel for if (!omp_in_parallel())
        for (long i = 0; i < n; ++i) d[i] += o.d[i];
    }
    void operator-=(const HVec& o) {
        const long n = (long)d.size();
#pragma omp parallel for if (!omp_in_parallel())
        for (long i = 0; i < n; ++i) d[i] -= o.d[i];
    }
    void operator*=(double a) {
        const long n = (long)d.size();
#pragma omp parallel for if (!omp_in_parallel())
        for (long i = 0; i < n; ++i) d[i] *= a;
    }
    double dot(const HVec& o) const {
        const long n = (long)d.size();
        double s = 0.0;
#pragma omp parallel for reduction(+ : s) if (!omp_in_parallel())
        for (long i = 0; i < n; ++i) s += d[i] * o.d[i];
        return s;
    }
    double norm2() const { return std::sqrt(std::abs(dot(*this))); }
    long getDimension() const { return (long)d.size(); }
};

struct Problem {
    int64_t n = 0, nnz = 0, s_start = 0, has_lz0 = 0;
    std::vector<int32_t> rowptr, colind;
    std::vector<double> vals, start, lz0;
};

class HCsrOp {
public:
    const Problem* P = nullptr;
    std::vector<double> tmp;
    HCsrOp() {}
    HCsrOp(const HCsrOp& o) : P(o.P) {}
    void apply(HVec& v) {
        const long n = (long)P->n;
        tmp.resize(n);
#pragma omp parallel for schedule(static) if (!omp_in_parallel())
        for (long i = 0; i < n; ++i) {
            double s = 0.0;
            for (int32_t k = P->rowptr[i]; k < P->rowptr[i + 1]; ++k) s += P->vals[k] * v.d[P->colind[k]];
            tmp[i] = s;
        }
        v.d.swap(tmp);
    }
    void apply(std::vector<HVec>& V) {
        for (auto& v : V) apply(v);
    }
};

class HRand {
public:
    const Problem* P = nullptr;
    long calls = 0;
    std::mt19937_64 gen{3141592};
    std::uniform_real_distribution<double> dist{-1.0, 1.0};
    void randomize(HVec& v) {
        const long n = (long)P->n;
        v.d.resize(n);
        if (calls == 0 && P->has_lz0) {
            std::memcpy(v.d.data(), P->lz0.data(), n * sizeof(double));
        } else if (calls >= 1 && calls - 1 < P->s_start) {
            std::memcpy(v.d.data(), P->start.data() + (size_t)(calls - 1) * n, n * sizeof(double));
        } else {
            for (long i = 0; i < n; ++i) v.d[i] = dist(gen);
        }
        ++calls;
    }
};

// The protected inner-iteration routines of RayleighChebyshevLM (RayleighChebyshevLM.h:1236-1300),
// run on the caller's block with the member set-up getMinEigenSystem does (:917-998).
class RCPhaseProbe : public RayleighChebyshevLM<HVec, HCsrOp, HRand, double> {
public:
    void run(std::vector<HVec>& V, HCsrOp& op, long resCheck, bool do_ortho, bool do_rr, double& t_ortho,
             double& t_rr) {
        const long s = (long)V.size();
        OpPtr = &op;
        vArray = V;
        vArrayTmp = V;
        vTemp.initialize(V[0]);
#ifdef _OPENMP
        MtVarray.assign(omp_get_max_threads(), V[0]);
#endif
        VtAV.initialize(s, s);
        VtAVeigVector.initialize(s, s);
        VtAVeigValue.assign(s, 0.0);
        const auto t0 = std::chrono::steady_clock::now();
        if (do_ortho) orthogonalize(vArray);
        const auto t1 = std::chrono::steady_clock::now();
        if (do_rr) {
            formVtAV(vArray, VtAV);
            computeVtVeigensystem(VtAV, VtAVeigValue, VtAVeigVector);
            std::vector<double> res;
            createEigenVectorsAndResiduals(VtAVeigVector, vArray, resCheck, res);
        }
        const auto t2 = std::chrono::steady_clock::now();
        t_ortho = std::chrono::duration<double>(t1 - t0).count();
        t_rr = std::chrono::duration<double>(t2 - t1).count();
    }
};

static bool read_problem(const char* path, Problem& P) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    char magic[4];
    int32_t ver = 0;
    bool ok = std::fread(magic, 1, 4, f) == 4 && std::memcmp(magic, "RCPB", 4) == 0;
    ok = ok && std::fread(&ver, 4, 1, f) == 1 && ver == 1;
    int64_t hdr[4];
    ok = ok && std::fread(hdr, 8, 4, f) == 4;
    if (!ok) {
        std::fclose(f);
        return false;
    }
    P.n = hdr[0];
    P.nnz = hdr[1];
    P.s_start = hdr[2];
    P.has_lz0 = hdr[3];
    P.rowptr.resize(P.n + 1);
    P.colind.resize(P.nnz);
    P.vals.resize(P.nnz);
    P.start.resize((size_t)P.n * P.s_start);
    ok = std::fread(P.rowptr.data(), 4, P.n + 1, f) == (size_t)(P.n + 1);
    ok = ok && std::fread(P.colind.data(), 4, P.nnz, f) == (size_t)P.nnz;
    ok = ok && std::fread(P.vals.data(), 8, P.nnz, f) == (size_t)P.nnz;
    ok = ok && std::fread(P.start.data(), 8, P.start.size(), f) == P.start.size();
    if (P.has_lz0) {
        P.lz0.resize(P.n);
        ok = ok && std::fread(P.lz0.data(), 8, P.n, f) == (size_t)P.n;
    }
    std::fclose(f);
    return ok;
}

static std::map<std::string, std::string> parse_kv(int argc, char** argv, int first) {
    std::map<std::string, std::string> kv;
    for (int i = first; i < argc; ++i) {
        std::string a = argv[i];
        auto p = a.find('=');
        if (p != std::string::npos) kv[a.substr(0, p)] = a.substr(p + 1);
    }
    return kv;
}
static double getd(std::map<std::string, std::string>& kv, const char* k, double dflt) {
    return kv.count(k) ? std::atof(kv[k].c_str()) : dflt;
}
static long getl(std::map<std::string, std::string>& kv, const char* k, long dflt) {
    return kv.count(k) ? std::atol(kv[k].c_str()) : dflt;
}

static void print_vec(const char* name, const std::vector<double>& v, bool last = false) {
    std::printf("\"%s\": [", name);
    for (size_t i = 0; i < v.size(); ++i) std::printf("%s%.17g", i ? ", " : "", v[i]);
    std::printf("]%s\n", last ? "" : ",");
}

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: ref_harness solve|filter|lanczos|cpoly ...\n");
        return 2;
    }
    const std::string mode = argv[1];
    if (mode == "cpoly") {
        auto kv = parse_kv(argc, argv, 2);
        const long mmax = getl(kv, "mmax", 200);
        LanczosCpoly cp;
        std::vector<double> xs, ux;
        for (long m = 1; m <= mmax; ++m) {
            cp.initialize(m, 1, 1.0, 0.0);
            xs.push_back(cp.XStar);
            ux.push_back(cp.UpperXStar);
        }
        std::printf("{\n");
        print_vec("xstar", xs);
        print_vec("upper_xstar", ux);
        long deg = 0;
        double bound = 0.0;
        if (kv.count("star")) {
            LanczosCpoly c2;
            c2.getStarDegreeAndSpectralRadius(getd(kv, "shift", 0.0), getd(kv, "bound", 1.0), getd(kv, "star", 0.5),
                                              getl(kv, "degmax", 200), deg, bound);
        }
        std::printf("\"star_degree\": %ld, \"star_bound\": %.17g\n}\n", deg, bound);
        return 0;
    }
    if (argc < 3) return 2;
    auto kv = parse_kv(argc, argv, 3);
#ifdef _OPENMP
    if (kv.count("threads")) omp_set_num_threads((int)getl(kv, "threads", 1));
    const int threads = omp_get_max_threads();
#else
    const int threads = 1;
#endif
    Problem P;
    if (!read_problem(argv[2], P)) {
        std::fprintf(stderr, "cannot read problem file %s\n", argv[2]);
        return 3;
    }
    HCsrOp op;
    op.P = &P;
    HRand rnd;
    rnd.P = &P;
    HVec vStart;
    vStart.d.assign(P.n, 0.0);

    if (mode == "solve") {
        const long k = getl(kv, "k", 16);
        const double tol = getd(kv, "tol", 1e-10);
        const long incr = getl(kv, "incr", k);
        const long buffer = getl(kv, "buffer", 8);
        RayleighChebyshevLM<HVec, HCsrOp, HRand, double> rc;
        rc.setStopCondition(kv.count("stop") ? kv["stop"] : std::string("COMBINATION"));
        if (kv.count("max_inner")) rc.setMaxInnerLoopCount(getl(kv, "max_inner", 10000));
        std::vector<double> evals;
        std::vector<HVec> evecs;
        const auto t0 = std::chrono::steady_clock::now();
        const long found = rc.getMinEigenSystem(k, tol, incr, buffer, vStart, op, rnd, evals, evecs);
        const auto t1 = std::chrono::steady_clock::now();
        const double secs = std::chrono::duration<double>(t1 - t0).count();
        auto cd = rc.getCountData();
        auto fd = rc.getFinalData();
        std::printf("{\n\"found\": %ld,\n\"seconds\": %.9g,\n\"threads\": %d,\n", found, secs, threads);
        print_vec("eigenvalues", evals);
        print_vec("residuals", rc.getEigVectorResiduals());
        std::printf("\"count_ortho\": %ld, \"count_opapply\": %ld, \"count_eigenvalue\": %ld,\n", cd["ortho"],
                    cd["OpApply"], cd["eigenvalue"]);
        std::printf("\"max_residual\": %.17g, \"max_eig_diff\": %.17g,\n", fd["maxResidual"], fd["maxEigValueDifference"]);
        std::printf("\"min_eig_est\": %.17g, \"max_eig_est\": %.17g\n}\n", rc.getMinEigValueEst(), rc.getMaxEigValueEst());
        if (kv.count("vecs")) {
            FILE* f = std::fopen(kv["vecs"].c_str(), "wb");
            if (f) {
                for (auto& v : evecs) std::fwrite(v.d.data(), 8, v.d.size(), f);
                std::fclose(f);
            }
        }
        return 0;
    }
    if (mode == "filter") {
        const long degree = getl(kv, "degree", 10);
        const double bound = getd(kv, "bound", 1.0);
        const double shift = getd(kv, "shift", 0.0);
        const long reps = getl(kv, "reps", 1);
        std::vector<HVec> V(P.s_start);
        for (long c = 0; c < P.s_start; ++c) V[c].d.assign(P.start.begin() + c * P.n, P.start.begin() + (c + 1) * P.n);
        LanczosCpolyOperatorLM<HVec, HCsrOp> cOp;
        cOp.initialize(op);
        cOp.setLanczosCpolyParameters(degree, reps, bound, shift);
        const auto t0 = std::chrono::steady_clock::now();
        cOp.apply(V);
        const auto t1 = std::chrono::steady_clock::now();
        const double secs = std::chrono::duration<double>(t1 - t0).count();
        std::printf("{\"seconds\": %.9g, \"threads\": %d, \"degree\": %ld, \"upper_xstar\": %.17g}\n", secs, threads,
                    degree, cOp.lanczosCpoly.UpperXStar);
        if (kv.count("out")) {
            FILE* f = std::fopen(kv["out"].c_str(), "wb");
            if (!f) return 4;
            for (auto& v : V) std::fwrite(v.d.data(), 8, v.d.size(), f);
            std::fclose(f);
        }
        return 0;
    }
    if (mode == "phases") {
        const long degree = getl(kv, "degree", 10);
        const double bound = getd(kv, "bound", 1.0);
        const double shift = getd(kv, "shift", 0.0);
        const long resCheck = getl(kv, "rescheck", P.s_start);
        std::vector<HVec> V(P.s_start);
        for (long c = 0; c < P.s_start; ++c) V[c].d.assign(P.start.begin() + c * P.n, P.start.begin() + (c + 1) * P.n);
        const std::string what = kv.count("do") ? kv["do"] : std::string("filter,ortho,rr");
        const bool do_filter = what.find("filter") != std::string::npos;
        const bool do_ortho = what.find("ortho") != std::string::npos;
        const bool do_rr = what.find("rr") != std::string::npos;
        LanczosCpolyOperatorLM<HVec, HCsrOp> cOp;
        cOp.initialize(op);
        cOp.setLanczosCpolyParameters(degree, 1, bound, shift);
        const auto t0 = std::chrono::steady_clock::now();
        if (do_filter) cOp.apply(V);
        const auto t1 = std::chrono::steady_clock::now();
        double t_ortho = 0.0, t_rr = 0.0;
        if (do_ortho || do_rr) {
            RCPhaseProbe probe;
            probe.run(V, op, resCheck, do_ortho, do_rr, t_ortho, t_rr);
        }
        std::printf("{\"filter_seconds\": %.9g, \"degree\": %ld, \"ortho_seconds\": %.9g, \"rr_seconds\": %.9g, "
                    "\"threads\": %d}\n",
                    std::chrono::duration<double>(t1 - t0).count(), degree, t_ortho, t_rr, threads);
        return 0;
    }
    if (mode == "lanczos") {
        const double tol = getd(kv, "tol", 1e-6);
        LanczosMaxMinFinder<HVec, HCsrOp, HRand> lz;
        if (kv.count("which") && kv["which"] == "both") lz.setMinMaxEigStopCondition();
        else lz.setMaxEigStopCondition();
        HVec v(vStart), w(vStart), wt(vStart);
        double lmin = 0, lmax = 0;
        lz.getMinMaxEigenvalues(tol, v, w, wt, op, rnd, lmin, lmax);
        std::printf("{\"lmin\": %.17g, \"lmax\": %.17g, \"iters\": %ld}\n", lmin, lmax, lz.getIterationCount());
        return 0;
    }
    std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
    return 2;
}
