// Host launchers of the direct-load sweep passes (direct.cu). Forms: 1 = at
// most 64 registers per thread (two 16-warp blocks per SM), 2 = at most 40
// (three blocks per SM; the widest groups spill).
#pragma once

#include <cuda_runtime.h>

#include "kernels.cuh"

namespace flbp {

template <typename T>
cudaError_t direct_factor_launch(int form, unsigned grid, const FactorArgs &a, const T *vf, T *fv, Ctl *ctl,
                                 cudaStream_t st);

// bmode: the variable pass's belief mode (0 none, 1 residual, 2 residual +
// count + history, 4 batched residual); always writes vf.
template <typename T>
cudaError_t direct_var_launch(int form, int bmode, bool damp, unsigned grid, const VarArgs &a, const T *fv, T *vf,
                              T *fvd, T d, Ctl *ctl, cudaStream_t st);

// Evidence sets on one graph (grid.y = set): the factor pass followed by
// the zeroing of the sets' cut entries ((set, entry) pairs), the variable
// pass with per-set residuals (BMODE 4, the set as the graph), and the
// initial +-inf v->f messages of the clamped variables ((set, slot, value)).
template <typename T>
cudaError_t sets_factor_launch(unsigned gx, unsigned n_sets, const FactorArgs &a, const T *vf, T *fv, Ctl *ctl,
                               const uint2 *cut, uint32_t n_cut, cudaStream_t st);
template <typename T>
cudaError_t sets_var_launch(bool damp, unsigned gx, unsigned n_sets, const VarArgs &a, const T *fv, T *vf, T *fvd,
                            T d, Ctl *ctl, cudaStream_t st);
template <typename T>
cudaError_t sets_init_slots(const uint4 *slots, uint32_t n, T *vf, uint64_t vf_stride, cudaStream_t st);

// Resident 16-warp blocks per SM of a form's factor (var = false) or
// variable pass.
template <typename T>
int direct_blocks_per_sm(int form, bool var, bool damp);

}  // namespace flbp
