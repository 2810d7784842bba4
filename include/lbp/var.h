/// @file var.h
/// @brief A discrete random variable: label plus number of states
/// (interface of FastLBP's include/lbp/var.h:14-53). Comparisons use the label only.
#pragma once

#include <stddef.h>

#include <iostream>

namespace lbp {

class Var {
    size_t _label;
    size_t _nstates;

public:
    Var(size_t label = 0, size_t nstates = 0) : _label(label), _nstates(nstates) {}
    ~Var() = default;
    size_t label() const { return _label; }
    size_t states() const { return _nstates; }
    bool operator<(const Var &n) const { return _label < n._label; }
    bool operator<=(const Var &n) const { return _label <= n._label; }
    bool operator!=(const Var &n) const { return _label != n._label; }
    bool operator==(const Var &n) const { return _label == n._label; }
    friend std::ostream &operator<<(std::ostream &os, const Var &n) { return os << "x" << n._label; }
};

}  // namespace lbp
