/// @file factor.h
/// @brief Dense probability factors over label-ordered variable sets
/// (interface of FastLBP's include/lbp/factor.h:17-88). CausalBP::belief()
/// returns its single-variable marginals as Factor.
#pragma once

#include <iostream>

#include <lbp/index.h>
#include <lbp/prob.h>
#include <lbp/varset.h>

namespace lbp {

template <typename T>
class TFactor {
    VarSet _vs;
    TProb<T> _p;

public:
    TFactor() = default;
    ~TFactor() = default;
    TFactor(const Var &v) : _vs(v), _p(v.states()) {}
    TFactor(const VarSet &vars) : _vs(vars), _p(vars.nrStates()) {}
    TFactor(const VarSet &vars, T p) : _vs(vars), _p(vars.nrStates(), p) {}
    TFactor(const VarSet &vars, const TProb<T> &p) : _vs(vars), _p(p) {
        if (_vs.nrStates() != _p.size()) std::cerr << "states dismatch" << std::endl;
    }

    void set(size_t i, T val) { _p.set(i, val); }
    const std::vector<T> &toVec() const { return _p.toVec(); }
    TProb<T> &p() { return _p; }
    T operator[](size_t i) const { return _p[i]; }
    const VarSet &vars() const { return _vs; }
    size_t nrStates() const { return _p.size(); }
    T normalize() { return _p.normalize(); }

    /// Marginal on `vars`, summing out the other variables.
    TFactor<T> marginal(const VarSet &vars, bool normed = true) const {
        VarSet res_vars = vars & _vs;
        TFactor<T> res(res_vars, (T)0);
        IndexFor i_res(res_vars, _vs);
        for (size_t i = 0; i < _p.size(); i++, ++i_res) res.set(i_res, res[i_res] + _p[i]);
        if (normed) res.normalize();
        return res;
    }
};

template <typename T>
std::ostream &operator<<(std::ostream &os, const TFactor<T> &f) {
    os << "(" << f.vars() << ", (";
    for (size_t i = 0; i < f.nrStates(); i++) os << (i == 0 ? "" : ", ") << f[i];
    return os << "))";
}

typedef TFactor<Real> Factor;

}  // namespace lbp
