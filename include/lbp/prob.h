/// @file prob.h
/// @brief Vectors of probabilities (interface of FastLBP's include/lbp/prob.h:18-162).
#pragma once

#include <stddef.h>

#include <algorithm>
#include <functional>
#include <iostream>
#include <vector>

#include <utils/utils.h>

namespace lbp {

template <typename T>
struct fo_id {
    T operator()(const T &x) const { return x; }
};

/// Division where dividing by zero gives zero.
template <typename T>
struct fo_divides0 {
    T operator()(const T &x, const T &y) const { return y == (T)0 ? (T)0 : x / y; }
};

template <typename T>
class TProb {
    typedef std::vector<T> container_type;
    typedef TProb<T> this_type;
    container_type _p;

public:
    typedef typename container_type::const_iterator const_iterator;

    TProb() = default;
    ~TProb() = default;
    /// Uniform distribution over n states.
    explicit TProb(size_t n) : _p(n, n ? T(1) / (T)n : T(0)) {}
    explicit TProb(size_t n, T p) : _p(n, p) {}
    template <typename S>
    TProb(const std::vector<S> &v) : _p(v.begin(), v.end()) {}

    const_iterator begin() const { return _p.begin(); }
    const_iterator end() const { return _p.end(); }
    T get(size_t i) const { return _p.at(i); }
    void set(size_t i, T val) { _p.at(i) = val; }
    const std::vector<T> &toVec() const { return _p; }
    T operator[](size_t i) const { return _p[i]; }
    size_t size() const { return _p.size(); }

    template <typename unOp>
    T accumulateSum(T init, unOp op) const {
        T t = op(init);
        for (const auto &x : _p) t += op(x);
        return t;
    }
    T sum() const { return accumulateSum((T)0, fo_id<T>()); }

    T normalize() {
        T Z = sum();
        if (Z == (T)0) std::cerr << "Not normalizable!" << std::endl;
        else *this /= Z;
        return Z;
    }

    template <typename unaryOp>
    this_type &pwUnaryOp(unaryOp op) {
        std::transform(_p.begin(), _p.end(), _p.begin(), op);
        return *this;
    }

    this_type &operator/=(T x) {
        if (x != 1) {
            fo_divides0<T> d;
            for (auto &v : _p) v = d(v, x);
        }
        return *this;
    }

    template <typename binaryOp>
    this_type &pwBinaryOp(const this_type &q, binaryOp op) {
        if (size() != q.size())
            std::cerr << "The sizes of two vectors performing pointwise operation are not the same!" << std::endl;
        std::transform(_p.begin(), _p.end(), q._p.begin(), _p.begin(), op);
        return *this;
    }

    this_type &operator*=(const this_type &q) { return pwBinaryOp(q, std::multiplies<T>()); }
};

template <typename T>
std::ostream &operator<<(std::ostream &os, const TProb<T> &p) {
    os << "(";
    for (size_t i = 0; i < p.size(); i++) os << (i ? ", " : "") << p.get(i);
    return os << ")";
}

typedef TProb<Real> Prob;

}  // namespace lbp
