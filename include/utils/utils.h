/// @file utils.h
/// @brief Basic types and helpers of the drop-in API (interface of FastLBP's
/// include/utils/utils.h:21-136: Real, Size, stream printers, the .causal_fg
/// comment skipper, wall clock, __LOGSTR__ and the global RNG).
#pragma once

#include <sys/time.h>

#include <chrono>
#include <ctime>
#include <iostream>
#include <map>
#include <random>
#include <set>
#include <string>
#include <vector>

namespace lbp {

typedef double Real;
typedef size_t Size;

// Packed edge records of the reference's device layout, kept so code that
// names them still compiles; this engine does not use them.
struct Index2Real { Size ind, v; Real prob; };
struct Index3 { Size ind, v, src_ind; };
struct Index5Real2 { Size ind, v, src_ind, start_ind, end_ind; Real prob_default, prob; };
struct Index5Real4 { Size ind, v, src_ind, start_ind, end_ind; Real prob_default, prob, mask0, mask1; };
struct Index6Real2 { Size ind, v, src_ind, start_ind, end_ind, head; Real prob_default, prob; };
struct Index6Real4 { Size ind, v, src_ind, start_ind, end_ind, head; Real prob_default, prob, mask0, mask1; };
struct Index7Real4 { Size ind, v, src_ind, start_ind, end_ind, head, type; Real prob_default, prob, mask0, mask1; };

template <class T>
std::ostream &operator<<(std::ostream &os, const std::vector<T> &x) {
    os << "(";
    for (size_t i = 0; i < x.size(); i++) os << (i ? ", " : "") << x[i];
    return os << ")";
}

template <class T>
std::ostream &operator<<(std::ostream &os, const std::set<T> &x) {
    os << "{";
    bool first = true;
    for (const auto &v : x) {
        os << (first ? "" : ", ") << v;
        first = false;
    }
    return os << "}";
}

template <class T1, class T2>
std::ostream &operator<<(std::ostream &os, const std::map<T1, T2> &x) {
    os << "{";
    bool first = true;
    for (const auto &kv : x) {
        os << (first ? "" : ", ") << kv.first << "->" << kv.second;
        first = false;
    }
    return os << "}";
}

inline std::ostream &operator<<(std::ostream &os, const Index3 &x) { return os << x.ind; }

/// Skips every following line of `is` that starts with '#'. The line
/// argument is taken by value, as in the reference, so it is left unchanged.
inline void read_annotation(std::istream &is, std::string line) {
    while (is.peek() == '#') std::getline(is, line);
}

/// Wall-clock time in seconds.
inline Real toc() {
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return (Real)tv.tv_sec + (Real)tv.tv_usec / 1e6;
}

inline std::string nowstr() {
    std::time_t tt = std::chrono::system_clock::to_time_t(std::chrono::system_clock::now());
    std::string s = std::ctime(&tt);
    return s.substr(0, s.size() - 1);
}

#define __LOGSTR__ (lbp::nowstr() + " " + __FILE__ + ": " + (std::to_string)(__LINE__) + ". ")

typedef std::mt19937 rnd_gen_type;

/// Global random number generator (seeded by callers such as Bingo's driver).
extern thread_local rnd_gen_type rnd_gen;

}  // namespace lbp
