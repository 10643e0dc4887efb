// Drives the C++ classes of include/pppm_compat.hpp with the reference's own
// call expressions:
//   * VortexSimulationSystem::computeURotation
//     (hybridFastSummation/VortexSimulationSystemImp.cpp:142-228):
//     setEvalParameter + evaluateVelocity, then getU(c)->getDevicePtr();
//   * computeStretching (:466-525): setVortParameter + sortVort, then
//     getSortPos()->getDevicePtr(), getSortVort(c)->getDevicePtr(),
//     getVortStartTable(), getCellh(), getOrigin();
//   * ParticleManager(uint) + initSpatialHash / setSpatialHashGrid(float3) /
//     doSpatialHash / getHashTable / getGridSize (particle_hash/SpaceHashClass.h);
//   * MultiGridSolver3DPeriod_double::m_FullMultiGrid and m_Vcycle
//     (multigrid/MultiGrid.h:188-209);
//   * PotentialFieldSolver (hybridFastSummation/PotentialFieldSolver.h).
//
// usage: compat_driver <in.bin> <out.bin> <n>
//   in.bin : uint32 N, float4[N] positions, double[3][N] strengths
//   out.bin: double[3][N] velocities, uint32[N] hash keys, uint32[N] indices,
//            double cell_h, double origin[3], double[n^3] multigrid x for a
//            test right-hand side, double[3][N] potential gradients,
//            double[n^3] x after one more V-cycle, float4[N] sorted positions,
//            double[3][N] sorted strengths, uint32[n^3] cell start table,
//            uint32[3] hash grid size
#include <cstdio>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "pppm_compat.hpp"

using namespace pppm_compat;

#define CK(x)                                                        \
    do {                                                             \
        if (!(x)) {                                                  \
            std::fprintf(stderr, "failed: %s (%s)\n", #x, lastError().c_str()); \
            return 2;                                                \
        }                                                            \
    } while (0)

int main(int argc, char **argv) {
    if (argc != 4) return 1;
    const unsigned n = (unsigned)std::atoi(argv[3]);
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 1;
    uint32_t N = 0;
    if (std::fread(&N, 4, 1, f) != 1) return 1;
    std::vector<float> pos(4 * (size_t)N);
    std::vector<double> al(3 * (size_t)N);
    if (std::fread(pos.data(), 4, pos.size(), f) != pos.size()) return 1;
    if (std::fread(al.data(), 8, al.size(), f) != al.size()) return 1;
    std::fclose(f);

    float4 *dpos = nullptr;
    double *dal = nullptr;
    CK(cudaMalloc(&dpos, 16 * (size_t)N) == cudaSuccess);
    CK(cudaMalloc(&dal, 24 * (size_t)N) == cudaSuccess);
    cudaMemcpy(dpos, pos.data(), 16 * (size_t)N, cudaMemcpyHostToDevice);
    cudaMemcpy(dal, al.data(), 24 * (size_t)N, cudaMemcpyHostToDevice);

    // the caller's arrays, as gf_GpuArray objects in the reference
    GpuArrayf4 *gf4_vort_cent = new GpuArrayf4(dpos, N);
    GpuArrayd vx(dal, N), vy(dal + N, N), vz(dal + 2 * (size_t)N, N);
    GpuArrayd *gd_vort[3] = {&vx, &vy, &vz};
    const uint u_num_vortices = N;

    BiotSavartSolver *g_vortexSolver = new BiotSavartSolver();
    CK(g_vortexSolver->initializeSolver(n, n, n, false, 1, N, N));
    CK(g_vortexSolver->setVortParameter(u_num_vortices, gf4_vort_cent, gd_vort));
    g_vortexSolver->computeFarFieldBuffer();
    CK(g_vortexSolver->lastOk());
    CK(g_vortexSolver->setEvalParameter(u_num_vortices, gf4_vort_cent));
    CK(g_vortexSolver->evaluateVelocity(gf4_vort_cent, 1));
    cudaDeviceSynchronize();

    std::vector<double> u(3 * (size_t)N);
    for (int c = 0; c < 3; c++)
        cudaMemcpy(u.data() + c * (size_t)N, g_vortexSolver->getU(c)->getDevicePtr(),
                   g_vortexSolver->getU(c)->getSize() * g_vortexSolver->getU(c)->typeSize(),
                   cudaMemcpyDeviceToHost);
    const double h = g_vortexSolver->getCellh();
    const double4 o = g_vortexSolver->getOrigin();

    // computeStretching's use of the sorted vortices and the cell tables
    g_vortexSolver->setVortParameter(u_num_vortices, gf4_vort_cent, gd_vort);
    g_vortexSolver->sortVort();
    const float4 *sorted_pos = g_vortexSolver->getSortPos()->getDevicePtr();
    std::vector<float> spos(4 * (size_t)N);
    std::vector<double> svort(3 * (size_t)N);
    cudaMemcpy(spos.data(), sorted_pos, 16 * (size_t)N, cudaMemcpyDeviceToHost);
    for (int c = 0; c < 3; c++)
        cudaMemcpy(svort.data() + c * (size_t)N, g_vortexSolver->getSortVort(c)->getDevicePtr(), 8 * (size_t)N,
                   cudaMemcpyDeviceToHost);
    const size_t C = (size_t)n * n * n;
    std::vector<uint32_t> cstart(C);
    cudaMemcpy(cstart.data(), g_vortexSolver->getVortStartTable(), 4 * C, cudaMemcpyDeviceToHost);

    // ParticleManager with the solver's grid (PH/SpaceHashClass.h:19, 46-54)
    ParticleManager pm(N);
    pm.initSpatialHash(N, n, n, n);
    pm.setSpatialHashGrid(n, (float)h, make_float3((float)o.x, (float)o.y, (float)o.z), N);
    pm.setHashParam();
    pm.doSpatialHash(gf4_vort_cent->getDevicePtr(), N);
    const uint3 gsize = pm.getGridSize();
    std::vector<uint32_t> keys(N), idx(N);
    cudaDeviceSynchronize();
    cudaMemcpy(keys.data(), pm.getHashTable(), 4 * (size_t)N, cudaMemcpyDeviceToHost);
    // reorder the indices 0..N-1 as data: the result is the sorted index table
    std::vector<float> iota(N);
    for (uint32_t t = 0; t < N; t++) iota[t] = (float)t;
    float *din = nullptr, *dout = nullptr;
    cudaMalloc(&din, 4 * (size_t)N);
    cudaMalloc(&dout, 4 * (size_t)N);
    cudaMemcpy(din, iota.data(), 4 * (size_t)N, cudaMemcpyHostToDevice);
    pm.reorderData(N, din, dout, 1, 1);
    std::vector<float> fidx(N);
    cudaMemcpy(fidx.data(), dout, 4 * (size_t)N, cudaMemcpyDeviceToHost);
    for (uint32_t t = 0; t < N; t++) idx[t] = (uint32_t)fidx[t];

    // MultiGridSolver3DPeriod_double: full multigrid, then one more V-cycle
    std::vector<double> b(C);
    for (size_t q = 0; q < C; q++) b[q] = std::sin(0.001 * (double)q) - 0.5;
    double *db = nullptr, *dx = nullptr;
    cudaMalloc(&db, 8 * C);
    cudaMalloc(&dx, 8 * C);
    cudaMemcpy(db, b.data(), 8 * C, cudaMemcpyHostToDevice);
    cudaMemset(dx, 0, 8 * C);
    MultiGridSolver3DPeriod_double mg;
    mg.m_InitialSystem((int)n, (int)n, (int)n);
    GpuArrayd X(dx, C), B(db, C);
    double res = 0;
    mg.m_FullMultiGrid(&X, &B, 1e-10, res);
    std::vector<double> x(C), xv(C);
    cudaDeviceSynchronize();
    cudaMemcpy(x.data(), dx, 8 * C, cudaMemcpyDeviceToHost);
    mg.m_Vcycle(&X, &B, 1e-10, res, 0);
    cudaDeviceSynchronize();
    cudaMemcpy(xv.data(), dx, 8 * C, cudaMemcpyDeviceToHost);

    // PotentialFieldSolver: masses = the x strengths at the vortex positions,
    // gradient evaluated at the same positions (HFS/PotentialFieldSolver.h)
    PotentialFieldSolver pf;
    CK(pf.initializeSolver(n, n, n, 1, N, N));
    CK(pf.setMassParameter(N, gf4_vort_cent, &vx));
    CK(pf.setEvalParameter(N, gf4_vort_cent));
    pf.computeFarFieldBuffer();
    CK(pf.lastOk());
    CK(pf.evaluateGradient(true));
    std::vector<double> grad(3 * (size_t)N);
    cudaDeviceSynchronize();
    cudaMemcpy(grad.data(), pf.getGradPhi()->getDevicePtr(), 24 * (size_t)N, cudaMemcpyDeviceToHost);
    pf.shutdown();

    FILE *g = std::fopen(argv[2], "wb");
    std::fwrite(u.data(), 8, u.size(), g);
    std::fwrite(keys.data(), 4, keys.size(), g);
    std::fwrite(idx.data(), 4, idx.size(), g);
    std::fwrite(&h, 8, 1, g);
    const double oo[3] = {o.x, o.y, o.z};
    std::fwrite(oo, 8, 3, g);
    std::fwrite(x.data(), 8, x.size(), g);
    std::fwrite(grad.data(), 8, grad.size(), g);
    std::fwrite(xv.data(), 8, xv.size(), g);
    std::fwrite(spos.data(), 4, spos.size(), g);
    std::fwrite(svort.data(), 8, svort.size(), g);
    std::fwrite(cstart.data(), 4, cstart.size(), g);
    const uint32_t gs[3] = {gsize.x, gsize.y, gsize.z};
    std::fwrite(gs, 4, 3, g);
    std::fclose(g);
    g_vortexSolver->shutdown();
    delete g_vortexSolver;
    delete gf4_vort_cent;
    std::printf("ok N=%u n=%u\n", N, n);
    return 0;
}
