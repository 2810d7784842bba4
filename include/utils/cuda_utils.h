/// @file cuda_utils.h
/// @brief CUDA helpers of the drop-in API (interface of FastLBP's
/// include/utils/cuda_utils.h:16-33).
#pragma once

#include <cuda_runtime.h>

#include <iostream>

#include <utils/log.h>

namespace lbp {

#define CUDA_CHECK_ERROR(err)                                          \
    do {                                                               \
        cudaError_t err_ = (err);                                      \
        if (err_ != cudaSuccess) {                                     \
            LOG_FATAL("CUDA Error: %s", cudaGetErrorString(err_));     \
        }                                                              \
    } while (0)

const int kCudaThreadsNum = 128;
inline int CudaGetBlocks(const int N) { return (N + kCudaThreadsNum - 1) / kCudaThreadsNum; }

#define CUDA_KERNEL_LOOP(i, n) \
    for (size_t i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += blockDim.x * gridDim.x)

}  // namespace lbp
