// C entry point over the reference's own spatial-hash kernels (particle_hash/
// particle_hash_kernel.cu, included where it lies, as its SpaceHashFunctional.cu
// does) and the stable key sort it uses (thrust::sort_by_key,
// SpaceHashFunctional.cu:97-102).  TEST INFRASTRUCTURE ONLY: the parity tests
// run it on the GPU as a checker of the oracle's and the product's hash.
//
// Steps of ParticleManager::setSpatialHashGrid / setHashParam / doSpatialHash
// (particle_hash/SpaceHashClass.h:46-58, SpaceHashClassImp.cpp): the float
// cell size and origin into the constant parameters, calcHashD, the sort,
// cellStart set to 0xFFFFFFFF, FindCellStartD.
#include <cuda_runtime.h>
#include <thrust/device_ptr.h>
#include <thrust/sort.h>

#include <cstdint>

#include "particle_hash_kernel.cu"

namespace {
struct Buf {
    void *p = nullptr;
    ~Buf() {
        if (p) cudaFree(p);
    }
};
}  // namespace

// pos4: N float4 positions; n: grid edge; h, origin: the float cell size and
// origin.  Outputs (host): keys and indices after the sort (N each), cellStart
// and cellEnd (n^3 each; cellEnd is written for occupied cells only, as in the
// reference: the caller pre-fills it); ms (may be NULL): device time of the
// three steps by CUDA events.  Returns 0 or a CUDA error code.
extern "C" int refgpu_hash(uint32_t n, float h, const float origin[3], uint32_t N, const float *pos4,
                           uint32_t *keys, uint32_t *index, uint32_t *cell_start, uint32_t *cell_end, float *ms) {
    const size_t C = (size_t)n * n * n;
    HashParams hp = {};
    hp.gridSize = make_uint3(n, n, n);
    hp.numCells = (uint)C;
    hp.worldOrigin = make_float3(origin[0], origin[1], origin[2]);
    hp.cellSize = make_float3(h, h, h);
    Buf d_pos, d_hash, d_idx, d_start, d_end;
    cudaError_t e = cudaMemcpyToSymbol(params, &hp, sizeof(HashParams));
    if (e == cudaSuccess) e = cudaMalloc(&d_pos.p, sizeof(float4) * (N ? N : 1));
    if (e == cudaSuccess) e = cudaMalloc(&d_hash.p, sizeof(uint) * (N ? N : 1));
    if (e == cudaSuccess) e = cudaMalloc(&d_idx.p, sizeof(uint) * (N ? N : 1));
    if (e == cudaSuccess) e = cudaMalloc(&d_start.p, sizeof(uint) * C);
    if (e == cudaSuccess) e = cudaMalloc(&d_end.p, sizeof(uint) * C);
    if (e == cudaSuccess) e = cudaMemcpy(d_pos.p, pos4, sizeof(float4) * N, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_end.p, cell_end, sizeof(uint) * C, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return (int)e;
    uint *hash = static_cast<uint *>(d_hash.p), *idx = static_cast<uint *>(d_idx.p);
    const uint threads = 256, blocks = (N + threads - 1) / threads;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    if (N) calcHashD<<<blocks, threads>>>(hash, idx, static_cast<float4 *>(d_pos.p), N);
    e = cudaGetLastError();
    if (e == cudaSuccess && N) {
        thrust::sort_by_key(thrust::device_ptr<uint>(hash), thrust::device_ptr<uint>(hash + N),
                            thrust::device_ptr<uint>(idx));
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemset(d_start.p, 0xff, sizeof(uint) * C);
    if (e == cudaSuccess && N)
        FindCellStartD<<<blocks, threads, (threads + 1) * sizeof(uint)>>>(static_cast<uint *>(d_start.p),
                                                                          static_cast<uint *>(d_end.p), hash, idx, N);
    cudaEventRecord(e1);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ms) *ms = t;
    if (e == cudaSuccess) e = cudaMemcpy(keys, hash, sizeof(uint) * N, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(index, idx, sizeof(uint) * N, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(cell_start, d_start.p, sizeof(uint) * C, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(cell_end, d_end.p, sizeof(uint) * C, cudaMemcpyDeviceToHost);
    return (int)e;
}
