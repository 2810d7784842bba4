/// @file varset.h
/// @brief Set of variables ordered by label (interface of FastLBP's include/lbp/varset.h:15-43).
#pragma once

#include <iostream>

#include <lbp/smallset.h>
#include <lbp/var.h>

namespace lbp {

class VarSet : public SmallSet<Var> {
public:
    VarSet() = default;
    VarSet(const SmallSet<Var> &x) : SmallSet<Var>(x) {}
    VarSet(const Var &v) : SmallSet<Var>(v) {}
    ~VarSet() = default;

    template <typename VarIterator>
    VarSet(VarIterator begin, VarIterator end, size_t sizeHint = 0) : SmallSet<Var>(begin, end, sizeHint) {}

    /// Number of joint states of the variables.
    size_t nrStates() const {
        size_t s = 1;
        for (const auto &v : *this) s *= v.states();
        return s;
    }

    friend std::ostream &operator<<(std::ostream &os, const VarSet &vs) {
        os << "{";
        bool first = true;
        for (const auto &v : vs) {
            os << (first ? "" : ", ") << v;
            first = false;
        }
        return os << "}";
    }
};

}  // namespace lbp
