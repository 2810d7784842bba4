// CausalBP of the drop-in C++ API: property parsing, construction of the
// GPU engine through the C ABI (with the SEQFIX / TOPO update sequence of
// csrc/ext/causal_bp.cu:186-304 when asked for), and the three run entry points of
// csrc/ext/causal_bp.cu (run() :858-910, run(tol,maxIters,hist) :912-1004,
// run(tol,minIters,maxIters,hist) :1006-1143).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <iostream>
#include <string>
#include <vector>

#include <ext/causal_bp.h>
#include <utils/log.h>

#include "../../include/fastlbp_b200.h"
#include "model_internal.h"

namespace lbp {

namespace {

void check(int rc, const char *what) {
    if (rc != FLBP_OK) LOG_FATAL("%s failed: %s", what, flbp_last_error());
}

}  // namespace

void CausalBP::setProperties(const PropertySet &opts) {
    props.tol = opts.hasKey("tol") ? opts.getStringAs<Real>("tol") : 1e-9;
    props.logdomain = opts.hasKey("logdomain") ? opts.getStringAs<bool>("logdomain") : false;
    props.maxiter = opts.hasKey("maxiter") ? opts.getStringAs<size_t>("maxiter") : 10000;
    props.maxtime = opts.hasKey("maxtime") ? opts.getStringAs<Real>("maxtime") : 10;
    props.updates = Properties::UpdateType::SEQFIX;
    if (opts.hasKey("updates")) {
        const std::string u = opts.getStringAs<std::string>("updates");
        if (u == "PARALL") props.updates = Properties::UpdateType::PARALL;
        else if (u == "TOPO") props.updates = Properties::UpdateType::TOPO;
        else props.updates = Properties::UpdateType::SEQFIX;  // unknown names fall back to SEQFIX
    }
    props.verbose = opts.hasKey("verbose") ? opts.getStringAs<size_t>("verbose") : 0;
    props.damping = opts.hasKey("damping") ? opts.getStringAs<Real>("damping") : 0.0;
    props.precision = 32;
    if (opts.hasKey("precision")) {
        const std::string p = opts.getStringAs<std::string>("precision");
        if (p == "FP64" || p == "fp64") props.precision = 64;
        else if (p == "FP32" || p == "fp32") props.precision = 32;
        else std::cerr << "CausalBP: unknown precision '" << p << "', using FP32" << std::endl;
    }
    if (props.logdomain) {
        static bool warned = false;
        if (!warned) {
            std::cerr << "CausalBP: logdomain=true has no effect; messages are always kept as log-odds" << std::endl;
            warned = true;
        }
    }
}

void CausalBP::construct() {
    detail::GraphArrays a;
    std::string err;
    if (detail::build_arrays(*this, a, err)) LOG_FATAL("CausalBP: %s", err.c_str());
    flbp_engine_opts o;
    o.precision = props.precision;
    o.device = -1;
    o.damping = props.damping;
    o.stream = nullptr;
    check(flbp_engine_create(&a.desc, &o, &_engine), "flbp_engine_create");
    if (props.updates != Properties::UpdateType::PARALL) {
        // buildFixedUpdateSeq / buildTopoUpdateSeq (csrc/ext/causal_bp.cu:186-304): SEQFIX draws
        // its factor order from the thread's rnd_gen, once per construction, as the reference does
        std::vector<int32_t> order;
        int32_t kind = FLBP_UPDATES_TOPO;
        if (props.updates == Properties::UpdateType::SEQFIX) {
            std::vector<int> numbers(nrFactors());
            for (int i = 0; i < (int)numbers.size(); ++i) numbers[i] = i;
            std::shuffle(numbers.begin(), numbers.end(), rnd_gen);
            order.assign(numbers.begin(), numbers.end());
            kind = FLBP_UPDATES_SEQFIX;
        }
        std::vector<int64_t> seq((size_t)a.desc.n_slots);
        check(flbp_update_seq(&a.desc, kind, order.data(), seq.data()), "flbp_update_seq");
        check(flbp_set_update_seq(_engine, seq.data(), (int64_t)seq.size()), "flbp_set_update_seq");
    }
    _beliefsV.assign(nrVars(), 0.0);
}

CausalBP::CausalBP(const CausalFactorGraph &fg, const PropertySet &opts) : DAIAlg<CausalFactorGraph>(fg) {
    setProperties(opts);
    construct();
}

CausalBP::~CausalBP() { flbp_engine_destroy(_engine); }

void CausalBP::init() { check(flbp_init(_engine), "flbp_init"); }

void CausalBP::fetchBeliefs(bool lowpass) {
    _beliefsV.assign(nrVars(), 0.0);
    check(flbp_get_beliefs(_engine, _beliefsV.data(), (int64_t)nrVars()), "flbp_get_beliefs");
    if (lowpass) {
        _lowPassBeliefs.assign(nrVars(), 0.0);
        check(flbp_get_lowpass(_engine, _lowPassBeliefs.data(), (int64_t)nrVars()), "flbp_get_lowpass");
    } else {
        _lowPassBeliefs = _beliefsV;
    }
}

void CausalBP::run() {
    if (props.verbose >= 1) std::cerr << "Starting ..." << std::endl;
    const Real tic = toc();
    flbp_run_info info{};
    check(flbp_run_tol(_engine, props.tol, (int64_t)props.maxiter, props.maxtime, &info), "flbp_run_tol");
    _iters = (size_t)info.total_sweeps;
    fetchBeliefs(false);
    if (props.verbose >= 1) {
        const double maxDiff = info.sweeps ? info.maxdiff : INFINITY;
        if (maxDiff > props.tol) {
            if (props.verbose == 1) std::cerr << std::endl;
            std::cerr << "CausalBP::run:  WARNING: not converged after " << _iters << " passes (" << toc() - tic
                      << " seconds)...final maxdiff:" << maxDiff << std::endl;
        } else {
            if (props.verbose >= 3) std::cerr << "CausalBP::run:  ";
            std::cerr << "converged in " << _iters << " passes (" << toc() - tic << " seconds)." << std::endl;
        }
    }
}

Real CausalBP::run(Real tolerance, size_t maxIters, size_t histLength) {
    (void)tolerance;
    (void)histLength;
    flbp_run_info info{};
    check(flbp_run_fixed(_engine, (int64_t)maxIters, &info), "flbp_run_fixed");
    _iters = (size_t)info.total_sweeps;
    fetchBeliefs(true);
    return 1.0;
}

Real CausalBP::run(Real tolerance, size_t minIters, size_t maxIters, size_t histLength) {
    flbp_run_info info{};
    check(flbp_run_lowpass(_engine, tolerance, (int64_t)minIters, (int64_t)maxIters, (int64_t)histLength,
                           props.maxtime, &info),
          "flbp_run_lowpass");
    _iters = (size_t)info.total_sweeps;
    if (info.sweeps > 0 && info.maxdiff > _maxdiff) _maxdiff = info.maxdiff;
    fetchBeliefs(true);
    return info.frac;
}

Factor CausalBP::beliefV(size_t i) const {
    const Real b = _beliefsV[i];
    return Factor(var(i), Prob(std::vector<Real>{1 - b, b}));
}

Factor CausalBP::belief(const VarSet &vs) const {
    if (vs.size() == 0) return Factor();
    if (vs.size() == 1) return beliefV(findVar(*vs.begin()));
    LOG_FATAL("unreachable");
}

void CausalBP::transferMessagesToHost() {
    int64_t E = 0;
    for (size_t i = 0; i < nrVars(); i++) E += (int64_t)nbV(i).size();
    std::vector<double> m0((size_t)E), m1((size_t)E);
    check(flbp_get_fv_messages(_engine, m0.data(), m1.data(), E), "flbp_get_fv_messages");
    _edges.clear();
    _edges.reserve(nrVars());
    size_t k = 0;
    for (size_t i = 0; i < nrVars(); i++) {
        std::vector<EdgeProp> row;
        row.reserve(nbV(i).size());
        for (size_t n = 0; n < nbV(i).size(); n++, k++) row.push_back({Prob(std::vector<Real>{m0[k], m1[k]})});
        _edges.push_back(std::move(row));
    }
}

}  // namespace lbp
