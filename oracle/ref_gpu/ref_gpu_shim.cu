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

// convertVortToSeg (HFS/VortexSimulationSystemImp.cpp:126-137): ComputePosb on
// the centres.  Outputs the two ends (enda = c - s/2, endb = c + s/2) and kappa.
extern "C" int refgpu_segments(uint32_t N, const float *cent4, const double *alpha, double h_seg, float *enda4,
                               float *endb4, double *kappa) {
    DevBuf d_c, d_a, d_b, d_al, d_k;
    cudaError_t e = upload(d_c, cent4, 4 * (size_t)N);
    if (e == cudaSuccess) e = upload(d_al, alpha, 3 * (size_t)N);
    if (e == cudaSuccess) e = upload<float>(d_a, nullptr, 4 * (size_t)N);
    if (e == cudaSuccess) e = upload<float>(d_b, nullptr, 4 * (size_t)N);
    if (e == cudaSuccess) e = upload<double>(d_k, nullptr, N);
    if (e != cudaSuccess) return (int)e;
    double *al = ptr<double>(d_al);
    ComputePosb(ptr<float4>(d_c), ptr<float4>(d_a), ptr<float4>(d_b), al, al + N, al + 2 * (size_t)N,
                ptr<double>(d_k), h_seg, N);
    e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(enda4, d_a.p, sizeof(float4) * N, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(endb4, d_b.p, sizeof(float4) * N, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(kappa, d_k.p, sizeof(double) * N, cudaMemcpyDeviceToHost);
    return (int)e;
}

// applyFlow + convertSegToVort + the first VectorAdd of computeStretching
// (HFS/VortexSimulationSystemImp.cpp:277-297, 315-330, 470-478): move both
// ends by their velocities ua / ub (3 x N; packed as the double4 of
// AddURotation), centres as the ends' midpoints (ComputePosa), then
// dv = kappa (endb - enda) - alpha (ComputeVortex) and dv = alpha + dv.
// enda4 / endb4 are moved in place.
extern "C" int refgpu_segment_update(uint32_t N, float *enda4, float *endb4, const double *alpha, const double *kappa,
                                     const double *ua, const double *ub, double dt, float *cent4, double *dv) {
    double4 *hua = new double4[N ? N : 1], *hub = new double4[N ? N : 1];
    for (uint32_t t = 0; t < N; t++) {
        hua[t] = make_double4(ua[t], ua[N + t], ua[2 * (size_t)N + t], 0.0);
        hub[t] = make_double4(ub[t], ub[N + t], ub[2 * (size_t)N + t], 0.0);
    }
    DevBuf d_a, d_b, d_c, d_al, d_k, d_ua, d_ub, d_dv;
    cudaError_t e = upload(d_a, enda4, 4 * (size_t)N);
    if (e == cudaSuccess) e = upload(d_b, endb4, 4 * (size_t)N);
    if (e == cudaSuccess) e = upload<float>(d_c, nullptr, 4 * (size_t)N);
    if (e == cudaSuccess) e = upload(d_al, alpha, 3 * (size_t)N);
    if (e == cudaSuccess) e = upload(d_k, kappa, N);
    if (e == cudaSuccess) e = upload(d_ua, hua, N);
    if (e == cudaSuccess) e = upload(d_ub, hub, N);
    if (e == cudaSuccess) e = upload<double>(d_dv, nullptr, 3 * (size_t)N);
    delete[] hua;
    delete[] hub;
    if (e != cudaSuccess) return (int)e;
    float4 *a = ptr<float4>(d_a), *b = ptr<float4>(d_b), *c = ptr<float4>(d_c);
    double *al = ptr<double>(d_al), *v = ptr<double>(d_dv);
    move_particle(a, dt, ptr<double4>(d_ua), N);
    move_particle(b, dt, ptr<double4>(d_ub), N);
    ComputePosa(a, b, c, N);
    ComputeVortex(a, b, al, al + N, al + 2 * (size_t)N, v, v + N, v + 2 * (size_t)N, ptr<double>(d_k), N);
    for (int q = 0; q < 3; q++) VectorAdd(al + q * (size_t)N, v + q * (size_t)N, v + q * (size_t)N, 1, 1, N);
    e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(enda4, a, sizeof(float4) * N, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(endb4, b, sizeof(float4) * N, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(cent4, c, sizeof(float4) * N, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(dv, v, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost);
    return (int)e;
}

// computeStretching's smoothing (HFS/VortexSimulationSystemImp.cpp:492-509):
// ParticleGaussianSmooth with the centres in caller order, the centres and the
// strengths sorted by cell, the cell tables, the solver's cell size and origin.
// out (3 x N) receives the smoothed strengths in caller order; ms (may be
// NULL) the kernel's device time.
extern "C" int refgpu_gaussian_smooth(uint32_t n, double cell_h, const double origin3[3], uint32_t N,
                                      const float *cent4, const float *scent4, const uint32_t *start,
                                      const uint32_t *end, const double *sdv, double nu, double dt, double *out,
                                      float *ms) {
    const size_t C = (size_t)n * n * n;
    DevBuf d_c, d_sc, d_s, d_e, d_in, d_out;
    cudaError_t e = upload(d_c, cent4, 4 * (size_t)N);
    if (e == cudaSuccess) e = upload(d_sc, scent4, 4 * (size_t)N);
    if (e == cudaSuccess) e = upload(d_s, start, C);
    if (e == cudaSuccess) e = upload(d_e, end, C);
    if (e == cudaSuccess) e = upload(d_in, sdv, 3 * (size_t)N);
    if (e == cudaSuccess) e = upload<double>(d_out, nullptr, 3 * (size_t)N);
    if (e != cudaSuccess) return (int)e;
    double *in = ptr<double>(d_in), *o = ptr<double>(d_out);
    Events ev;
    cudaEventRecord(ev[0]);
    ParticleGaussianSmooth(ptr<uint32_t>(d_s), ptr<uint32_t>(d_e), ptr<float4>(d_c), ptr<float4>(d_sc), nu, dt, o,
                           o + N, o + 2 * (size_t)N, in, in + N, in + 2 * (size_t)N, cell_h, make_uint3(n, n, n), N,
                           make_double4(origin3[0], origin3[1], origin3[2], 0.0));
    cudaEventRecord(ev[1]);
    e = cudaDeviceSynchronize();
    if (ms) cudaEventElapsedTime(ms, ev[0], ev[1]);
    if (e == cudaSuccess) e = cudaMemcpy(out, o, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost);
    return (int)e;
}

// addBaroclinicForce's device part (HFS/VortexSimulationSystemImp.cpp:412-446):
// AssignDensity on the heat particles sorted by density cell (sheat4, sheat,
// start, end), GradDensity, ParticleGetBaroclinic with dt_beta = 5 dt.  dim,
// h (double, L / dim), hf (the hash's float cell size) and origin3 describe
// the density grid.  alpha (3 x N) is updated in place; rho (dim^3) and grad
// (3 x dim^3, component planes) receive the grids, ms (may be NULL) the device
// time of the three kernels.  ParticleGetBaroclinic
// launches 256 blocks of N/256 + 1 threads (its block and grid sizes swapped),
// which covers every vortex while N/256 + 1 <= 1024.
extern "C" int refgpu_baroclinic(uint32_t dim, double h, float hf, const double origin3[3], uint32_t H,
                                 const float *sheat4, const float *sheat, const uint32_t *start, const uint32_t *end,
                                 uint32_t N, const float *cent4, double *alpha, double dt, float *rho, float *grad,
                                 float *ms) {
    if (N / 256 + 1 > 1024) return -1;
    const size_t C = (size_t)dim * dim * dim;
    DevBuf d_hp, d_h, d_s, d_e, d_rho, d_grad, d_c, d_al;
    cudaError_t e = upload(d_hp, sheat4, 4 * (size_t)H);
    if (e == cudaSuccess) e = upload(d_h, sheat, H);
    if (e == cudaSuccess) e = upload(d_s, start, C);
    if (e == cudaSuccess) e = upload(d_e, end, C);
    if (e == cudaSuccess) e = upload<float>(d_rho, nullptr, C);
    if (e == cudaSuccess) e = upload<float>(d_grad, nullptr, 3 * C);
    if (e == cudaSuccess) e = upload(d_c, cent4, 4 * (size_t)N);
    if (e == cudaSuccess) e = upload(d_al, alpha, 3 * (size_t)N);
    if (e != cudaSuccess) return (int)e;
    const double4 origin = make_double4(origin3[0], origin3[1], origin3[2], 0.0);
    const uint3 gd = make_uint3(dim, dim, dim);
    float *heat = ptr<float>(d_h);
    Events ev;
    cudaEventRecord(ev[0]);
    AssignDensity(ptr<uint32_t>(d_s), ptr<uint32_t>(d_e), ptr<float4>(d_hp), heat, heat, h, ptr<float>(d_rho), gd, gd,
                  H, origin);
    float3 *g3 = ptr<float3>(d_grad);
    GradDensity(ptr<float>(d_rho), g3, h, dim, dim, dim);
    double *al = ptr<double>(d_al);
    ParticleGetBaroclinic(ptr<float4>(d_c), al, al + N, al + 2 * (size_t)N, g3, dt * 5.0, N, dim, dim, dim,
                          1.0 / (double)hf, origin);
    cudaEventRecord(ev[1]);
    e = cudaDeviceSynchronize();
    if (ms) cudaEventElapsedTime(ms, ev[0], ev[1]);
    if (e == cudaSuccess) e = cudaMemcpy(rho, d_rho.p, sizeof(float) * C, cudaMemcpyDeviceToHost);
    float3 *hg = new float3[C ? C : 1];
    if (e == cudaSuccess) e = cudaMemcpy(hg, g3, sizeof(float3) * C, cudaMemcpyDeviceToHost);
    for (size_t c = 0; e == cudaSuccess && c < C; c++) {
        grad[c] = hg[c].x;
        grad[C + c] = hg[c].y;
        grad[2 * C + c] = hg[c].z;
    }
    delete[] hg;
    if (e == cudaSuccess) e = cudaMemcpy(alpha, al, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost);
    return (int)e;
}

// The scalar wrappers GPU_kernel.cu defines without a declaration in
// ParticleMesh.h (signatures as defined there).
void PotentialComputeScalarFarField(double *mass, double *gridval, double *phi, double cell_h, double G,
                                    double direction, uint3 gdim, uint3 hdim, int K);
void PotentialInterpolateFarFieldScalar(float4 *pos, double *far_force, double *p_force, double cell_h, uint dimx,
                                        uint dimy, uint dimz, uint num_particles, double4 origin);
void Potential_PPCorrMNScalar(uint *start, uint *end, float4 *pos_eval, float4 *pos_mass, double *mass,
                              double *p_phi, double invh, double h, double G, double direction, uint3 gdim,
                              uint3 hdim, uint2 gstride, uint2 hstride, int K, uint M, uint N, double4 origin);

// PotentialFieldSolver (HFS/PotentialFieldSolver.cpp:527-608 m_ParticleToMesh,
// 622-630 m_ComputeGradient, 645-672 computeFarFieldBuffer, 441-525
// evaluateGradient on unsorted points, 674-679 computeDphiDn, 695-739 the scalar
// path) with the reference's wrappers; the multigrid's phi comes in.  The
// masses come sorted by cell (spos4, smass, start, end) as m_ParticleToMesh
// leaves them, umass in caller order for computeDphiDn.  cell_h is the hash's
// float cell size, L the domain edge, origin3 the double origin.  Outputs:
// density, rhs (n^3), far (scalar: n^3; gradient: 3 x n^3 planes), out (M or
// 3 x M) and, for the gradient with normals, dphidn (M); ms (may be NULL,
// 3 entries): device time of density + RHS, of the far-field buffer, and of
// the evaluation at the points.
extern "C" int refgpu_potential(uint32_t n, int K, uint32_t N, const float *spos4, const double *smass,
                                const double *umass, const uint32_t *start, const uint32_t *end, const double *phi,
                                const double origin3[3], float cell_hf, double L, uint32_t M, const float *eval4,
                                int scalar, const double *normals, const double *areas, double *density, double *rhs,
                                double *far, double *out, double *dphidn, float *ms) {
    const size_t C = (size_t)n * n * n;
    const uint3 dim = make_uint3(n, n, n);
    const double cell_h = (double)cell_hf;
    const double4 origin = make_double4(origin3[0], origin3[1], origin3[2], 0.0);
    // monopole of m_ParticleToMesh, summed on the host in the sorted order
    double tw = 0.0, tm = 0.0, cx = 0.0, cy = 0.0, cz = 0.0;
    for (uint32_t i = 0; i < N; i++) {
        tw += fabs(smass[i]);
        tm += smass[i];
    }
    for (uint32_t i = 0; i < N; i++) {
        cx += spos4[4 * i] * fabs(smass[i]);
        cy += spos4[4 * i + 1] * fabs(smass[i]);
        cz += spos4[4 * i + 2] * fabs(smass[i]);
    }
    cx /= tw;
    cy /= tw;
    cz /= tw;
    DevBuf d_pos, d_m, d_um, d_s, d_e, d_rho, d_rhs, d_phi, d_g, d_far, d_ev, d_out, d_nrm, d_area, d_dp;
    cudaError_t e = upload(d_pos, spos4, 4 * (size_t)N);
    if (e == cudaSuccess) e = upload(d_m, smass, N);
    if (e == cudaSuccess) e = upload(d_um, umass, N);
    if (e == cudaSuccess) e = upload(d_s, start, C);
    if (e == cudaSuccess) e = upload(d_e, end, C);
    if (e == cudaSuccess) e = upload<double>(d_rho, nullptr, C);
    if (e == cudaSuccess) e = upload<double>(d_rhs, nullptr, C);
    if (e == cudaSuccess) e = upload(d_phi, phi, C);
    if (e == cudaSuccess) e = upload<double>(d_g, nullptr, 3 * C);
    if (e == cudaSuccess) e = upload<double>(d_far, nullptr, 3 * C);
    if (e == cudaSuccess) e = upload(d_ev, eval4, 4 * (size_t)M);
    if (e == cudaSuccess) e = upload<double>(d_out, nullptr, 3 * (size_t)M);
    if (e != cudaSuccess) return (int)e;
    uint32_t *st = ptr<uint32_t>(d_s), *en = ptr<uint32_t>(d_e);
    float4 *pos = ptr<float4>(d_pos), *pts = ptr<float4>(d_ev);
    double *rho = ptr<double>(d_rho), *rh = ptr<double>(d_rhs), *ph = ptr<double>(d_phi);
    Events ev;
    cudaEventRecord(ev[0]);
    ParticleToMesh(st, en, pos, ptr<double>(d_m), cell_h, rho, dim, dim, N, origin);
    e = cudaMemcpy(rh, rho, sizeof(double) * C, cudaMemcpyDeviceToDevice);
    if (e != cudaSuccess) return (int)e;
    ComputeRHS(rh, (double)(cell_hf * cell_hf), -1.0, (uint)C);
    applyDirichlet(rh, make_double4(cx, cy, cz, 0.0), tm, origin, cell_h, n, n, n);
    cudaEventRecord(ev[1]);
    e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(density, rho, sizeof(double) * C, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(rhs, rh, sizeof(double) * C, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return (int)e;
    const uint2 stride = make_uint2(n * n, n);
    if (scalar) {
        double *o = ptr<double>(d_out);
        cudaEventRecord(ev[2]);
        PotentialComputeScalarFarField(ptr<double>(d_um), rho, ph, cell_h, 1.0, 1.0, dim, dim, K);
        cudaEventRecord(ev[3]);
        PotentialInterpolateFarFieldScalar(pts, ph, o, cell_h, n, n, n, M, origin);
        Potential_PPCorrMNScalar(st, en, pts, pos, ptr<double>(d_m), o, 1.0 / cell_h, cell_h, 1.0, 1.0, dim, dim,
                                 stride, stride, K, M, N, origin);
        cudaEventRecord(ev[4]);
        e = cudaDeviceSynchronize();
        if (ms) {
            cudaEventElapsedTime(ms, ev[0], ev[1]);
            cudaEventElapsedTime(ms + 1, ev[2], ev[3]);
            cudaEventElapsedTime(ms + 2, ev[3], ev[4]);
        }
        if (e == cudaSuccess) e = cudaMemcpy(far, ph, sizeof(double) * C, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(out, o, sizeof(double) * M, cudaMemcpyDeviceToHost);
        return (int)e;
    }
    double3 *g3 = ptr<double3>(d_g), *f3 = ptr<double3>(d_far), *o3 = ptr<double3>(d_out);
    cudaEventRecord(ev[2]);
    ComputeGradient(ph, g3, cell_h, 1.0, n, n, n);
    PotentialComputeFarField(st, en, pos, ptr<double>(d_m), rho, ph, g3, f3, cell_h, 1.0, 1.0, dim, dim, K, M, origin);
    cudaEventRecord(ev[3]);
    PotentialInterpolateFarField(pts, f3, o3, cell_h, n, n, n, M, origin);
    Potential_PPCorrMN(st, en, pts, pos, ptr<double>(d_m), o3, 1.0 / cell_h, cell_h, 1.0, 1.0, dim, dim, stride,
                       stride, K, M, N, origin);
    const float3 bbmin = make_float3((float)origin3[0], (float)origin3[1], (float)origin3[2]);
    const float3 bbmax = make_float3((float)((double)bbmin.x + L), (float)((double)bbmin.y + L),
                                     (float)((double)bbmin.z + L));
    PotentialComputeGradForOutParticle(pts, tm, make_double3(cx, cy, cz), bbmin, bbmax, 1.0, 1.0, o3, M);
    cudaEventRecord(ev[4]);
    if (normals && areas) {
        e = upload(d_nrm, normals, 3 * (size_t)M);
        if (e == cudaSuccess) e = upload(d_area, areas, M);
        if (e == cudaSuccess) e = upload<double>(d_dp, nullptr, M);
        if (e != cudaSuccess) return (int)e;
        ComputeDphidn(ptr<double3>(d_nrm), o3, ptr<double>(d_um), ptr<double>(d_dp), ptr<double>(d_area), M);
    }
    e = cudaDeviceSynchronize();
    if (ms) {
        cudaEventElapsedTime(ms, ev[0], ev[1]);
        cudaEventElapsedTime(ms + 1, ev[2], ev[3]);
        cudaEventElapsedTime(ms + 2, ev[3], ev[4]);
    }
    double3 *hf = new double3[C ? C : 1];
    if (e == cudaSuccess) e = cudaMemcpy(hf, f3, sizeof(double3) * C, cudaMemcpyDeviceToHost);
    for (size_t c = 0; e == cudaSuccess && c < C; c++) {
        far[c] = hf[c].x;
        far[C + c] = hf[c].y;
        far[2 * C + c] = hf[c].z;
    }
    delete[] hf;
    double3 *ho = new double3[M ? M : 1];
    if (e == cudaSuccess) e = cudaMemcpy(ho, o3, sizeof(double3) * M, cudaMemcpyDeviceToHost);
    for (uint32_t t = 0; e == cudaSuccess && t < M; t++) {
        out[t] = ho[t].x;
        out[M + t] = ho[t].y;
        out[2 * (size_t)M + t] = ho[t].z;
    }
    delete[] ho;
    if (e == cudaSuccess && normals && areas) e = cudaMemcpy(dphidn, d_dp.p, sizeof(double) * M, cudaMemcpyDeviceToHost);
    return (int)e;
}
