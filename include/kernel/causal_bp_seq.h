/// @file causal_bp_seq.h
/// @brief Present so that code including FastLBP's kernel header
/// (e.g. examples/bingo_wrapper.cu:2) compiles unchanged. The reference's
/// per-kernel launch wrappers are internal to its CausalBP; this engine's
/// kernels are reached through CausalBP or the C ABI (fastlbp_b200.h).
#pragma once

#include <utils/utils.h>

namespace lbp {
namespace kernel {}
}  // namespace lbp
