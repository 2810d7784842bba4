/// @file smallset.h
/// @brief Sorted set of unique elements stored in a vector (interface of
/// FastLBP's include/lbp/smallset.h:17-101).
#pragma once

#include <stddef.h>

#include <algorithm>
#include <iterator>
#include <vector>

#include <lbp/var.h>

namespace lbp {

template <typename T>
class SmallSet {
    std::vector<T> _elements;

public:
    typedef typename std::vector<T>::const_iterator const_iterator;
    typedef typename std::vector<T>::iterator iterator;

    SmallSet() = default;
    SmallSet(const T &t) : _elements(1, t) {}
    ~SmallSet() = default;

    template <typename TIterator>
    SmallSet(TIterator begin, TIterator end, size_t sizeHint) {
        _elements.reserve(sizeHint);
        _elements.insert(_elements.begin(), begin, end);
        std::sort(_elements.begin(), _elements.end());
        _elements.erase(std::unique(_elements.begin(), _elements.end()), _elements.end());
    }

    SmallSet &insert(const T &t) {
        auto it = std::lower_bound(_elements.begin(), _elements.end(), t);
        if (it == _elements.end() || *it != t) _elements.insert(it, t);
        return *this;
    }

    SmallSet &erase(const T &t) { return (*this /= t); }

    SmallSet operator&(const SmallSet &x) const {
        SmallSet res;
        std::set_intersection(_elements.begin(), _elements.end(), x._elements.begin(), x._elements.end(),
                              std::back_inserter(res._elements));
        return res;
    }

    /// True if x is a subset of *this.
    bool operator>>(const SmallSet &x) const {
        return std::includes(_elements.begin(), _elements.end(), x._elements.begin(), x._elements.end());
    }

    SmallSet &operator/=(const T &t) {
        auto pos = std::lower_bound(_elements.begin(), _elements.end(), t);
        if (pos != _elements.end() && *pos == t) _elements.erase(pos);
        return *this;
    }

    bool contains(const T &t) const { return std::binary_search(_elements.begin(), _elements.end(), t); }
    const_iterator begin() const { return _elements.begin(); }
    const_iterator end() const { return _elements.end(); }
    typename std::vector<T>::size_type size() const { return _elements.size(); }
};

}  // namespace lbp
