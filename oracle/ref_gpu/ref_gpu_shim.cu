// C entry point over the reference's own GPU kernels, compiled from
// hybridFastSummation/GPU_kernel.cu where it lies (`make -C oracle refgpu`).
// TEST INFRASTRUCTURE ONLY: the parity tests run it on the GPU as a checker of
// the oracle and of the product; nothing in the product calls it.
//
// It runs the stages of BiotSavartSolver::computeFarFieldBuffer and
// evaluateVelocity (hybridFastSummation/BiotSavartSolverImp.cpp:440-487,
// 517-560, 622-639, 756-813) with the reference's host wrappers, in the
// reference's order, on the sorted vortices and cell tables the caller
// passes:
//   ParticleToMesh per component -> grid vorticity
//   getCurl(psi)                 -> grid velocity U
//   BiotSavartComputeFarField    -> far field
//   BiotSavartInterpolateFarField + BiotSavartPPCorrScaleMN at the points.
// The multigrid between P2M and the curl is not among them: its kernels use
// the texture-reference API that CUDA 12 removed, so psi comes in from the
// caller.  The evaluation points need no sorting: both evaluation kernels
// treat each point on its own.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

#include "ParticleMesh.h"

namespace {

struct DevBuf {
    void *p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

template <typename T>
cudaError_t upload(DevBuf &b, const T *src, size_t count) {
    cudaError_t e = cudaMalloc(&b.p, sizeof(T) * (count ? count : 1));
    if (e == cudaSuccess && src && count) e = cudaMemcpy(b.p, src, sizeof(T) * count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !src) e = cudaMemset(b.p, 0, sizeof(T) * (count ? count : 1));
    return e;
}

template <typename T>
T *ptr(DevBuf &b) {
    return static_cast<T *>(b.p);
}

struct Events {
    cudaEvent_t e[6];
    Events() {
        for (auto &x : e) cudaEventCreate(&x);
    }
    ~Events() {
        for (auto &x : e) cudaEventDestroy(x);
    }
    cudaEvent_t operator[](int i) const { return e[i]; }
};

}  // namespace

// n: grid edge (cubic); K: near-field radius; N vortices sorted by cell with
// strengths salpha (3 x N, component planes) and cell tables start / end
// (n^3, 0xFFFFFFFF for empty cells); psi (3 x n^3) the vector potential;
// origin / cell_h the domain as the solver holds it.  Outputs (host, FP64):
// vort, curl, far (3 x n^3 each), far_at (3 x M: the interpolated far field
// alone) and uvw (3 x M: far field + near-field correction); stage_ms (may be
// NULL): device time of P2M (3 components), curl, far field, interpolation and
// near field, by CUDA events around each.  Returns 0, or the CUDA error code
// of the first failing call.
extern "C" int refgpu_farfield_eval(uint32_t n, int K, uint32_t N, const float *spos4, const double *salpha,
                                    const uint32_t *start, const uint32_t *end, const double *psi,
                                    const double origin3[3], double cell_h, uint32_t M, const float *eval_a4,
                                    const float *eval_b4, int is_segment, double *vort, double *curl, double *far,
                                    double *far_at, double *uvw, float *stage_ms) {
    const size_t C = (size_t)n * n * n;
    const uint3 dim = make_uint3(n, n, n);
    const double4 origin = make_double4(origin3[0], origin3[1], origin3[2], 0.0);
    DevBuf d_pos, d_alpha, d_start, d_end, d_psi, d_vort, d_curl, d_far, d_ea, d_eb, d_u;
    cudaError_t e = upload(d_pos, spos4, 4 * (size_t)N);
    if (e == cudaSuccess) e = upload(d_alpha, salpha, 3 * (size_t)N);
    if (e == cudaSuccess) e = upload(d_start, start, C);
    if (e == cudaSuccess) e = upload(d_end, end, C);
    if (e == cudaSuccess) e = upload(d_psi, psi, 3 * C);
    if (e == cudaSuccess) e = upload<double>(d_vort, nullptr, 3 * C);
    if (e == cudaSuccess) e = upload<double>(d_curl, nullptr, 3 * C);
    if (e == cudaSuccess) e = upload<double>(d_far, nullptr, 3 * C);
    if (e == cudaSuccess) e = upload(d_ea, eval_a4, 4 * (size_t)M);
    if (e == cudaSuccess) e = upload(d_eb, is_segment == 1 ? eval_b4 : nullptr, 4 * (size_t)M);
    if (e == cudaSuccess) e = upload<double>(d_u, nullptr, 3 * (size_t)M);
    if (e != cudaSuccess) return (int)e;

    float4 *pos = ptr<float4>(d_pos);
    double *al = ptr<double>(d_alpha), *ps = ptr<double>(d_psi), *vg = ptr<double>(d_vort);
    double *cg = ptr<double>(d_curl), *fg = ptr<double>(d_far), *u = ptr<double>(d_u);
    uint32_t *st = ptr<uint32_t>(d_start), *en = ptr<uint32_t>(d_end);

    Events ev;
    // m_ParticleToMesh: one call per component
    cudaEventRecord(ev[0]);
    for (int c = 0; c < 3; c++)
        ParticleToMesh(st, en, pos, al + (size_t)c * N, cell_h, vg + c * C, dim, dim, N, origin);
    cudaEventRecord(ev[1]);
    // m_ComputeCurl
    getCurl(ps, ps + C, ps + 2 * C, cg, cg + C, cg + 2 * C, n, n, n, cell_h);
    cudaEventRecord(ev[2]);
    e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(vort, vg, sizeof(double) * 3 * C, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(curl, cg, sizeof(double) * 3 * C, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return (int)e;
    // computeFarFieldBuffer: far = U first, then the correction (which also
    // overwrites psi and U with the diagonal term's scratch)
    e = cudaMemcpy(fg, cg, sizeof(double) * 3 * C, cudaMemcpyDeviceToDevice);
    if (e != cudaSuccess) return (int)e;
    float t_p2m = 0.f, t_curl = 0.f, t_far = 0.f, t_interp = 0.f, t_pp = 0.f;
    cudaEventElapsedTime(&t_p2m, ev[0], ev[1]);
    cudaEventElapsedTime(&t_curl, ev[1], ev[2]);
    cudaEventRecord(ev[2]);
    BiotSavartComputeFarField(st, en, pos, vg, vg + C, vg + 2 * C, ps, ps + C, ps + 2 * C, cg, cg + C, cg + 2 * C,
                              fg, fg + C, fg + 2 * C, cell_h, dim, dim, K, N, origin);
    cudaEventRecord(ev[3]);
    e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(far, fg, sizeof(double) * 3 * C, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return (int)e;
    // evaluateVelocity
    float4 *ea = ptr<float4>(d_ea), *eb = ptr<float4>(d_eb);
    cudaEventElapsedTime(&t_far, ev[2], ev[3]);
    cudaEventRecord(ev[3]);
    BiotSavartInterpolateFarField(ea, fg, fg + C, fg + 2 * C, u, u + M, u + 2 * (size_t)M, cell_h, n, n, n, M, origin);
    cudaEventRecord(ev[4]);
    e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(far_at, u, sizeof(double) * 3 * M, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return (int)e;
    cudaEventElapsedTime(&t_interp, ev[3], ev[4]);
    cudaEventRecord(ev[4]);
    BiotSavartPPCorrScaleMN(st, en, ea, eb, (uint32_t)is_segment, pos, al, al + N, al + 2 * (size_t)N, u, u + M,
                            u + 2 * (size_t)M, cg, cg + C, cg + 2 * C, cell_h, dim, dim, K, M, N, origin);
    cudaEventRecord(ev[5]);
    e = cudaDeviceSynchronize();
    cudaEventElapsedTime(&t_pp, ev[4], ev[5]);
    if (stage_ms) {
        stage_ms[0] = t_p2m;
        stage_ms[1] = t_curl;
        stage_ms[2] = t_far;
        stage_ms[3] = t_interp;
        stage_ms[4] = t_pp;
    }
    if (e == cudaSuccess) e = cudaMemcpy(uvw, u, sizeof(double) * 3 * M, cudaMemcpyDeviceToHost);
    return (int)e;
}
