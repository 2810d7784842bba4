/// @file causal_factor.h
/// @brief Noisy causal factor: a singleton prior, a noisy-AND rule or an OR
/// aggregation over binary variables (interface of FastLBP's
/// include/ext/causal_factor.h:14-76).
///
/// For AND ('*'): P(head=1 | all body 1) = p, P(head=1 | otherwise) = q.
/// For OR ('+'):  P(head=0 | all body 0) = p, P(head=0 | otherwise) = q.
/// Singleton ('I'): P(head=1) = p.
#pragma once

#include <iostream>

#include <lbp/prob.h>
#include <lbp/varset.h>

namespace lbp {

class CausalFactor {
public:
    enum CausalType {
        Singleton = 'I',
        DefiniteAnd = '*',
        DefiniteOr = '+',
    };

    /// Set once the head variable has been clamped; head_mask is then the
    /// one-hot indicator of the clamped state (element-wise product if the
    /// head is clamped again).
    bool head_clamped;
    Prob head_mask;

private:
    CausalType _type;
    Var _head;
    VarSet _body;
    Real _p;
    Real _q = 0;
    VarSet _vs;

public:
    /// Singleton factor on v with P(v=1) = p.
    CausalFactor(const Var &v, Real p = 1);
    /// AND (isAnd) or OR factor with the given head and body.
    CausalFactor(const Var &head, const VarSet &body, bool isAnd, Real p, Real q);

    Real prob() const { return _p; }
    Real prob_default() const { return _q; }
    /// 0 Singleton, 1 DefiniteAnd, 2 DefiniteOr.
    int type() const;
    const Var &head() const { return _head; }
    const VarSet &body() const { return _body; }
    /// Body plus head, in label order.
    const VarSet &vars() const { return _vs; }

    /// The factor after observing variable i = x (csrc/ext/causal_factor.cpp:63-100):
    /// a singleton head takes p = x; an AND/OR head becomes head-clamped; a body
    /// variable is removed, and x = 0 on AND or x = 1 on OR resolves the rule
    /// (p := q, empty body).
    CausalFactor gen_clamped(Var i, size_t x) const;

    friend std::ostream &operator<<(std::ostream &, const CausalFactor &);
};

}  // namespace lbp
