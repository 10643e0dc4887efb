// Stand-in for the CUDA samples' helper_cuda.h, which the reference's
// GPU_kernel.cu includes for two error-check macros.  TEST INFRASTRUCTURE
// ONLY: used when building the reference's own kernels as a checker.
#pragma once
#include <cstdio>

#define checkCudaErrors(call)                                                         \
    do {                                                                              \
        cudaError_t err_ = (call);                                                    \
        if (err_ != cudaSuccess) fprintf(stderr, "CUDA: %s\n", cudaGetErrorString(err_)); \
    } while (0)

#define getLastCudaError(msg)                                                         \
    do {                                                                              \
        cudaError_t err_ = cudaGetLastError();                                        \
        if (err_ != cudaSuccess) fprintf(stderr, "%s: %s\n", (msg), cudaGetErrorString(err_)); \
    } while (0)
