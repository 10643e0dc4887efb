// Pre-included ahead of the reference's multigrid/MultiGrid_kernel.cu when it is
// built as a checker (TEST INFRASTRUCTURE ONLY).  That file reads its grids
// through legacy texture references (texture<T, 1, ...> globals bound with
// cudaBindTexture, fetched with tex1Dfetch), an API CUDA 12 removed.  Here a
// "texture" is a managed global holding a device pointer, and a fetch is a
// plain global load of element i.  The kernels read every bound grid only
// where no thread of the same launch writes it (red-black half sweeps,
// residual, restriction, prolongation), so a plain load returns what the
// texture fetch returned.  No definition of the reference file changes.
#pragma once
#include <cuda_runtime.h>

struct textureReference {
    int filterMode = 0;   // assigned by the file's setupTexture; no effect here
    const void *ptr = nullptr;
};

template <class T, int dim = 1, enum cudaTextureReadMode mode = cudaReadModeElementType>
struct refmg_texture : textureReference {};

// the file declares its four texture references as namespace-scope globals:
// managed, so that host code (setupTexture, the binding) and kernels both see them
#define texture __managed__ refmg_texture

template <class T, int dim, enum cudaTextureReadMode mode>
__device__ __forceinline__ T tex1Dfetch(const refmg_texture<T, dim, mode> &t, int i) {
    return static_cast<const T *>(t.ptr)[i];
}

// cudaBindTexture(offset, texref, devPtr, desc, size): the offset is 0 and the
// texture now reads devPtr.  The caller synchronises before it rebinds.
inline cudaError_t cudaBindTexture(size_t *offset, const textureReference *texref, const void *devPtr,
                                   const cudaChannelFormatDesc *, size_t = ~(size_t)0) {
    if (offset) *offset = 0;
    const_cast<textureReference *>(texref)->ptr = devPtr;
    return cudaSuccess;
}
