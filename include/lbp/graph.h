/// @file graph.h
/// @brief Neighbour records of a bipartite graph (interface of FastLBP's include/lbp/graph.h:14-38).
#pragma once

#include <stddef.h>

#include <utility>
#include <vector>

namespace lbp {

/// One neighbour of a node: its position in the node's list (iter), the
/// neighbour's index (node) and this node's position in the neighbour's list (dual).
struct Neighbor {
    size_t iter;
    size_t node;
    size_t dual;
    Neighbor(size_t iter, size_t node, size_t dual) : iter(iter), node(node), dual(dual) {}
    operator size_t() const { return node; }
};

typedef std::vector<Neighbor> Neighbors;

typedef std::pair<size_t, size_t> Edge;

}  // namespace lbp
