/// @file daialg.h
/// @brief Inference-algorithm base classes (interface of FastLBP's
/// include/lbp/daialg.h:12-35). DAIAlg<GRM> holds its own copy of the graph.
#pragma once

#include <lbp/factorgraph.h>

namespace lbp {

class InfAlg {
public:
    InfAlg() = default;
    ~InfAlg() = default;
};

template <class GRM>
class DAIAlg : public InfAlg, public GRM {
public:
    DAIAlg() = default;
    DAIAlg(const GRM &grm) : InfAlg(), GRM(grm) {}
    ~DAIAlg() = default;
};

typedef DAIAlg<FactorGraph> DAIAlgFG;

}  // namespace lbp
