/// @file index.h
/// @brief Multi-index helpers for dense factors (interface of FastLBP's
/// include/lbp/index.h:13-68): IndexFor walks the joint states of a variable
/// set and reports the matching linear index into a sub-set; Permute converts
/// linear indices between a caller's variable order and the label order.
#pragma once

#include <vector>

#include <lbp/varset.h>

namespace lbp {

class IndexFor {
    long _index = 0;
    std::vector<long> _sum;
    std::vector<size_t> _state;
    std::vector<size_t> _ranges;

public:
    IndexFor() = default;
    IndexFor(const VarSet &indexVars, const VarSet &forVars);
    IndexFor &reset();
    operator size_t() const { return (size_t)_index; }
    IndexFor &operator++();
    void operator++(int) { ++(*this); }
    bool valid() const { return _index >= 0; }
};

class Permute {
    std::vector<size_t> _ranges;
    std::vector<size_t> _sigma;

public:
    Permute() = default;
    Permute(const std::vector<size_t> &rs, const std::vector<size_t> &sigma) : _ranges(rs), _sigma(sigma) {}
    /// Permutation from the order of `vars` to label order.
    Permute(const std::vector<Var> &vars, bool reverse = false);
    size_t convertLinearIndex(size_t li) const;
    const std::vector<size_t> &sigma() const { return _sigma; }
    size_t operator[](size_t i) const { return _sigma[i]; }
};

}  // namespace lbp
