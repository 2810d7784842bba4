// Launchers of the direct-load sweep passes (direct.cuh), compiled apart from
// the engine so that the two forms build in parallel.

#include <cuda_runtime.h>

#include "direct.cuh"
#include "direct_launch.h"

namespace flbp {

namespace {

template <typename T, int MINB>
void *factor_fn() {
    return (void *)factor_direct_kernel<T, MINB>;
}

template <typename T, int BMODE, bool DAMP, int MINB>
void *var_fn() {
    return (void *)var_direct_kernel<T, BMODE, true, DAMP, MINB>;
}

template <typename T, int MINB>
void *var_fn_any(int bmode, bool damp) {
    if (damp) {
        switch (bmode) {
            case 0: return var_fn<T, 0, true, MINB>();
            case 1: return var_fn<T, 1, true, MINB>();
            case 2: return var_fn<T, 2, true, MINB>();
            default: return var_fn<T, 4, true, MINB>();
        }
    }
    switch (bmode) {
        case 0: return var_fn<T, 0, false, MINB>();
        case 1: return var_fn<T, 1, false, MINB>();
        case 2: return var_fn<T, 2, false, MINB>();
        default: return var_fn<T, 4, false, MINB>();
    }
}

// form 1: at most 64 registers (2 blocks of 16 warps per SM); form 2: at most 40 (3 blocks)
template <typename T>
void *factor_kernel(int form) {
    return form == 2 ? factor_fn<T, 3>() : factor_fn<T, 2>();
}

template <typename T>
void *var_kernel(int form, int bmode, bool damp) {
    return form == 2 ? var_fn_any<T, 3>(bmode, damp) : var_fn_any<T, 2>(bmode, damp);
}

}  // namespace

template <typename T>
cudaError_t direct_factor_launch(int form, unsigned grid, const FactorArgs &a, const T *vf, T *fv, Ctl *ctl,
                                 cudaStream_t st) {
    FactorArgs args = a;
    const T *vfp = vf;
    T *fvp = fv;
    void *params[] = {&args, &vfp, &fvp, &ctl};
    return cudaLaunchKernel(factor_kernel<T>(form), dim3(grid), dim3(kDirectThreads), params, 0, st);
}

template <typename T>
cudaError_t direct_var_launch(int form, int bmode, bool damp, unsigned grid, const VarArgs &a, const T *fv, T *vf,
                              T *fvd, T d, Ctl *ctl, cudaStream_t st) {
    VarArgs args = a;
    const T *fvp = fv;
    T *vfp = vf, *fvdp = fvd;
    T dd = d;
    void *params[] = {&args, &fvp, &vfp, &fvdp, &dd, &ctl};
    return cudaLaunchKernel(var_kernel<T>(form, bmode, damp), dim3(grid), dim3(kDirectThreads), params, 0, st);
}

template <typename T>
int direct_blocks_per_sm(int form, bool var, bool damp) {
    int n = 0;
    const void *fn = var ? var_kernel<T>(form, 2, damp) : factor_kernel<T>(form);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kDirectThreads, 0) != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

template cudaError_t direct_factor_launch<float>(int, unsigned, const FactorArgs &, const float *, float *, Ctl *,
                                                 cudaStream_t);
template cudaError_t direct_factor_launch<double>(int, unsigned, const FactorArgs &, const double *, double *, Ctl *,
                                                  cudaStream_t);
template cudaError_t direct_var_launch<float>(int, int, bool, unsigned, const VarArgs &, const float *, float *,
                                              float *, float, Ctl *, cudaStream_t);
template cudaError_t direct_var_launch<double>(int, int, bool, unsigned, const VarArgs &, const double *, double *,
                                               double *, double, Ctl *, cudaStream_t);
template int direct_blocks_per_sm<float>(int, bool, bool);
template int direct_blocks_per_sm<double>(int, bool, bool);

}  // namespace flbp
