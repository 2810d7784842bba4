/// @file factorgraph.h
/// @brief Generic dense factor graph with the libDAI ".fg" reader (interface
/// of FastLBP's include/lbp/factorgraph.h:16-78). Kept so that drivers which
/// also accept non-causal graphs link; inference runs on CausalFactorGraph.
#pragma once

#include <iostream>
#include <vector>

#include <lbp/bipgraph.h>
#include <lbp/factor.h>

namespace lbp {

class FactorGraph {
    BipartiteGraph _G;
    std::vector<Var> _vars;
    std::vector<Factor> _factors;
    void constructGraph(size_t nrEdges);

public:
    FactorGraph() = default;
    ~FactorGraph() = default;
    FactorGraph(const std::vector<Factor> &P);

    const Var &var(size_t i) const { return _vars[i]; }
    const Factor &factor(size_t I) const { return _factors[I]; }
    const Neighbors &nbV(size_t i) const { return _G.nb1(i); }
    const Neighbors &nbF(size_t I) const { return _G.nb2(I); }
    size_t nrVars() const { return _vars.size(); }
    size_t nrFactors() const { return _factors.size(); }
    size_t findVar(const Var &n) const;
    void ReadFromFile(const char *filename);
    friend std::istream &operator>>(std::istream &is, FactorGraph &fg);
};

}  // namespace lbp
