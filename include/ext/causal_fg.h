/// @file causal_fg.h
/// @brief Graph of causal factors (interface of FastLBP's include/ext/causal_fg.h:15-74).
///
/// Variables are the sorted unique labels of all factors; factors keep their
/// given order; nbF(I) lists vars(I) in label order and nbV(i) lists factors
/// in factor order, each entry carrying its position in the other list.
#pragma once

#include <map>

#include <ext/causal_factor.h>
#include <lbp/bipgraph.h>
#include <utils/log.h>

namespace lbp {

class CausalFactorGraph {
    BipartiteGraph _G;
    std::vector<Var> _vars;
    std::vector<CausalFactor> _factors;

    void setFactor(size_t I, const CausalFactor &newFactor) { _factors[I] = newFactor; }
    void setFactors(const std::map<size_t, CausalFactor> &facs) {
        for (const auto &kv : facs) setFactor(kv.first, kv.second);
    }
    void constructGraph(size_t nrEdges);

public:
    CausalFactorGraph() = default;
    CausalFactorGraph(const std::vector<CausalFactor> &P);
    CausalFactorGraph(std::vector<CausalFactor> &&P);
    ~CausalFactorGraph() = default;

    const Var &var(size_t i) const { return _vars[i]; }
    const CausalFactor &factor(size_t I) const { return _factors[I]; }
    const std::vector<Var> &vars() const { return _vars; }
    const std::vector<CausalFactor> &factors() const { return _factors; }
    const Neighbors &nbV(size_t i) const { return _G.nb1(i); }
    const Neighbor &nbV(size_t i, size_t _I) const { return _G.nb1(i)[_I]; }
    const Neighbors &nbF(size_t I) const { return _G.nb2(I); }
    size_t nrVars() const { return _vars.size(); }
    size_t nrFactors() const { return _factors.size(); }
    size_t nrEdges() const { return _G.nrEdges(); }
    /// Index of variable n; prints "var not found" and returns nrVars() when absent.
    size_t findVar(const Var &n) const;

    /// Reads a .causal_fg file; exits through LOG_FATAL when it cannot be opened.
    void ReadFromFile(const char *filename);

    /// Observe variable index i to value x: every factor containing it is
    /// replaced by gen_clamped(). The neighbour lists are not rebuilt;
    /// CausalFactorGraph(g.factors()) gives the rebuilt graph.
    void clamp(size_t i, size_t x);

    friend std::istream &operator>>(std::istream &is, CausalFactorGraph &fg);
};

}  // namespace lbp
