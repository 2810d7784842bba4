/// @file bipgraph.h
/// @brief Bipartite adjacency lists with dual indices (interface of FastLBP's
/// include/lbp/bipgraph.h:14-69). Nodes of type 1 are variables, type 2 factors.
#pragma once

#include <lbp/graph.h>

namespace lbp {

class BipartiteGraph {
    std::vector<Neighbors> _nb1;
    std::vector<Neighbors> _nb2;

public:
    BipartiteGraph() = default;
    ~BipartiteGraph() = default;

    const Neighbors &nb1(size_t i1) const { return _nb1[i1]; }
    const Neighbors &nb2(size_t i2) const { return _nb2[i2]; }

    /// Rebuild from a range of (type-1 node, type-2 node) edges, in order.
    template <typename EdgeInputIterator>
    void construct(size_t nrNodes1, size_t nrNodes2, EdgeInputIterator begin, EdgeInputIterator end,
                   bool check = true) {
        _nb1.assign(nrNodes1, Neighbors());
        _nb2.assign(nrNodes2, Neighbors());
        {  // room for every node's neighbours first (the edge order decides iter / dual as before)
            std::vector<size_t> d1(nrNodes1, 0), d2(nrNodes2, 0);
            for (EdgeInputIterator e = begin; e != end; ++e) {
                if (e->first < nrNodes1) d1[e->first]++;
                if (e->second < nrNodes2) d2[e->second]++;
            }
            for (size_t i = 0; i < nrNodes1; i++) _nb1[i].reserve(d1[i]);
            for (size_t i = 0; i < nrNodes2; i++) _nb2[i].reserve(d2[i]);
        }
        for (EdgeInputIterator e = begin; e != end; ++e) addEdge(e->first, e->second, check);
    }

    /// Append edge (n1, n2); with `check`, only when it is not present yet.
    BipartiteGraph &addEdge(size_t n1, size_t n2, bool check = true) {
        if (check)
            for (const auto &nb : _nb1[n1])
                if (nb.node == n2) return *this;
        const size_t it1 = _nb1[n1].size(), it2 = _nb2[n2].size();
        _nb1[n1].push_back(Neighbor(it1, n2, it2));
        _nb2[n2].push_back(Neighbor(it2, n1, it1));
        return *this;
    }

    size_t nrNodes1() const { return _nb1.size(); }
    size_t nrNodes2() const { return _nb2.size(); }

    size_t nrEdges() const {
        size_t s = 0;
        for (const auto &n : _nb1) s += n.size();
        return s;
    }
};

}  // namespace lbp
