/// @file causal_bp.h
/// @brief Loopy belief propagation over a CausalFactorGraph on a B200
/// (interface of FastLBP's include/ext/causal_bp.h:19-193).
///
/// Properties read from the PropertySet (exact value types, as in the
/// reference): "tol" (Real, 1e-9), "maxiter" (size_t, 10000), "maxtime"
/// (Real seconds, 10), "updates" (std::string: PARALL, SEQFIX or TOPO;
/// SEQFIX, the default, shuffles the factor order with rnd_gen at
/// construction as the reference does), "logdomain"
/// (bool), "verbose" (size_t). Added by this engine: "damping" (Real in
/// [0,1), 0) and "precision" (std::string "FP32" or "FP64", "FP32").
///
/// The sweeps run on the GPU through the C ABI of fastlbp_b200.h; the graph
/// topology is taken from the factors' variable sets, which equals the
/// rebuilt graph of examples/fl_wrapper.cu:45 for clamped graphs.
#pragma once

#include <memory>
#include <vector>

#include <ext/causal_fg.h>
#include <lbp/daialg.h>
#include <lbp/factor.h>
#include <lbp/properties.h>
#include <utils/utils.h>

struct flbp_engine;

namespace lbp {

class CausalBP : public DAIAlg<CausalFactorGraph> {
    struct Properties {
        enum class UpdateType { SEQFIX, PARALL, TOPO };
        size_t verbose;
        size_t maxiter;
        Real maxtime;
        Real tol;
        bool logdomain;
        UpdateType updates;
        Real damping;
        int precision;
    } props;

    Real _maxdiff = 0;
    size_t _iters = 0;

    struct EdgeProp {
        Prob message;
    };
    std::vector<std::vector<EdgeProp>> _edges;

    std::vector<Real> _beliefsV;
    std::vector<Real> _lowPassBeliefs;
    flbp_engine *_engine = nullptr;

    void setProperties(const PropertySet &opts);
    void construct();
    void fetchBeliefs(bool lowpass);

public:
    CausalBP(const CausalFactorGraph &fg, const PropertySet &opts);
    ~CausalBP();
    CausalBP(const CausalBP &) = delete;
    CausalBP &operator=(const CausalBP &) = delete;

    /// Single-variable belief; an empty set gives Factor(), larger sets are fatal.
    Factor belief(const VarSet &vs) const;
    /// Belief of variable i as Factor(var(i), (1-b, b)).
    Factor beliefV(size_t i) const;
    /// Messages to uniform; keeps the sweep counter, as the reference does.
    void init();
    /// Sweep until converged (max belief change <= tol), maxiter or maxtime.
    void run();
    /// Exactly maxIters sweeps; returns 1.
    Real run(Real tolerance, size_t maxIters, size_t histLength);
    /// Bingo's loop: converge, stop once enough variables converged after
    /// minIters, or give up after maxIters (then beliefs are the mean of the
    /// last histLength sweeps). Returns the fraction not yet converged.
    Real run(Real tolerance, size_t minIters, size_t maxIters, size_t histLength);
    /// Low-pass belief P(x_i = 1) of the last run.
    Real newBelief(size_t varIndex) const { return _lowPassBeliefs[varIndex]; }
    /// Copies the current factor-to-variable messages to the host (newMessage()).
    void transferMessagesToHost();
    const Prob &newMessage(size_t i, size_t _I) const { return _edges[i][_I].message; }

    /// Sweeps performed since construction.
    size_t Iterations() const { return _iters; }
    /// Largest final residual seen by the low-pass runs.
    Real maxDiff() const { return _maxdiff; }
    /// The underlying C-ABI engine handle.
    flbp_engine *engine() const { return _engine; }
};

}  // namespace lbp
