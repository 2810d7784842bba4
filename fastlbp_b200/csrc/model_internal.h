// Internal helpers shared by the C++ API implementation and the graph-model C ABI.
#pragma once

#include <fstream>
#include <istream>
#include <string>
#include <vector>

#include <ext/causal_fg.h>

#include "../../include/fastlbp_b200.h"

namespace lbp {
namespace detail {

/// Thrown by the reader on a type line that is not 'I', '*' or '+'.
struct BadFactorType {};

/// .causal_fg reader; throws BadFactorType or the std:: conversion errors.
CausalFactorGraph parse_causal_fg(std::istream &is);
/// The same reader on text in memory, and on a whole open file (read at once).
CausalFactorGraph parse_causal_fg_text(const char *text, size_t n);
CausalFactorGraph read_causal_fg_file(std::ifstream &f);

/// A CausalFactorGraph as the engine's reference-order arrays.
struct GraphArrays {
    std::vector<int64_t> offsets, slot_var, head;
    std::vector<int32_t> type, clamped;
    std::vector<double> p, q, m0, m1;
    flbp_graph_desc desc{};
};

/// Factor-major arrays of CausalBP::construct() for the graph's factors,
/// with topology taken from each factor's vars(). Returns 0 or 1 (err set).
int build_arrays(const CausalFactorGraph &fg, GraphArrays &a, std::string &err);

}  // namespace detail
}  // namespace lbp
