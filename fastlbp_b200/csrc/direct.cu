// Launchers of the direct-load sweep passes (direct.cuh), compiled apart from
// the engine so that the two forms build in parallel.

#include <cuda_runtime.h>

#include <algorithm>

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

// Evidence sets: cut entries get no message (their f->v values are zeroed
// after every factor pass), clamped variables' v->f messages start at +-inf.
template <typename T>
__global__ void sets_cut_kernel(const uint2 *__restrict__ cut, uint32_t n, T *fv, uint64_t fv_stride,
                                const int *done) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint2 c = cut[i];  // (set, entry)
        if (!done[c.x]) fv[c.x * fv_stride + c.y] = T(0);
    }
}

template <typename T>
__global__ void sets_slots_kernel(const uint4 *__restrict__ sl, uint32_t n, T *vf, uint64_t vf_stride) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint4 c = sl[i];  // (set, slot, value, -)
        vf[c.x * vf_stride + c.y] = c.z ? Num<T>::inf() : -Num<T>::inf();
    }
}

template <typename T>
cudaError_t sets_factor_launch(unsigned gx, unsigned n_sets, const FactorArgs &a, const T *vf, T *fv, Ctl *ctl,
                               const uint2 *cut, uint32_t n_cut, cudaStream_t st) {
    FactorArgs args = a;
    const T *vfp = vf;
    T *fvp = fv;
    void *params[] = {&args, &vfp, &fvp, &ctl};
    cudaError_t e = cudaLaunchKernel((const void *)factor_direct_kernel<T, 2, true>, dim3(gx, n_sets),
                                     dim3(kDirectThreads), params, 0, st);
    if (e == cudaSuccess && n_cut)
        sets_cut_kernel<T><<<std::min<uint32_t>((n_cut + 255) / 256, 4096), 256, 0, st>>>(cut, n_cut, fv,
                                                                                          a.set_fv_stride, a.set_done);
    return e == cudaSuccess ? cudaGetLastError() : e;
}

template <typename T>
cudaError_t sets_var_launch(bool damp, unsigned gx, unsigned n_sets, const VarArgs &a, const T *fv, T *vf, T *fvd,
                            T d, Ctl *ctl, cudaStream_t st) {
    VarArgs args = a;
    const T *fvp = fv;
    T *vfp = vf, *fvdp = fvd;
    T dd = d;
    void *params[] = {&args, &fvp, &vfp, &fvdp, &dd, &ctl};
    const void *fn = damp ? (const void *)var_direct_kernel<T, 4, true, true, 2, true>
                          : (const void *)var_direct_kernel<T, 4, true, false, 2, true>;
    return cudaLaunchKernel(fn, dim3(gx, n_sets), dim3(kDirectThreads), params, 0, st);
}

template <typename T>
cudaError_t sets_init_slots(const uint4 *slots, uint32_t n, T *vf, uint64_t vf_stride, cudaStream_t st) {
    if (!n) return cudaSuccess;
    sets_slots_kernel<T><<<std::min<uint32_t>((n + 255) / 256, 4096), 256, 0, st>>>(slots, n, vf, vf_stride);
    return cudaGetLastError();
}

template cudaError_t sets_factor_launch<float>(unsigned, unsigned, const FactorArgs &, const float *, float *, Ctl *,
                                               const uint2 *, uint32_t, cudaStream_t);
template cudaError_t sets_factor_launch<double>(unsigned, unsigned, const FactorArgs &, const double *, double *,
                                                Ctl *, const uint2 *, uint32_t, cudaStream_t);
template cudaError_t sets_var_launch<float>(bool, unsigned, unsigned, const VarArgs &, const float *, float *, float *,
                                            float, Ctl *, cudaStream_t);
template cudaError_t sets_var_launch<double>(bool, unsigned, unsigned, const VarArgs &, const double *, double *,
                                             double *, double, Ctl *, cudaStream_t);
template cudaError_t sets_init_slots<float>(const uint4 *, uint32_t, float *, uint64_t, cudaStream_t);
template cudaError_t sets_init_slots<double>(const uint4 *, uint32_t, double *, uint64_t, cudaStream_t);

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
