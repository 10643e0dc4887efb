// Drives the C++ classes of include/pppm_compat.hpp the way the reference's
// VortexSimulationSystem::computeURotation drives BiotSavartSolver
// (hybridFastSummation/VortexSimulationSystemImp.cpp:142-228), plus the
// ParticleManager and MultiGridSolver3DPeriod_double counterparts.
//
// usage: compat_driver <in.bin> <out.bin> <n>
//   in.bin : uint32 N, float4[N] positions, double[3][N] strengths
//   out.bin: double[3][N] velocities, uint32[N] hash keys, uint32[N] indices,
//            double cell_h, double origin[3], double[n^3] multigrid x for b = u
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

    float4_ *dpos = nullptr;
    double *dal = nullptr;
    CK(cudaMalloc(&dpos, 16 * (size_t)N) == cudaSuccess);
    CK(cudaMalloc(&dal, 24 * (size_t)N) == cudaSuccess);
    cudaMemcpy(dpos, pos.data(), 16 * (size_t)N, cudaMemcpyHostToDevice);
    cudaMemcpy(dal, al.data(), 24 * (size_t)N, cudaMemcpyHostToDevice);

    GpuArrayf4 cent(dpos, N);
    GpuArrayd vx(dal, N), vy(dal + N, N), vz(dal + 2 * (size_t)N, N);
    GpuArrayd *omega[3] = {&vx, &vy, &vz};

    BiotSavartSolver solver;
    CK(solver.initializeSolver(n, n, n, false, 1, N, N));
    CK(solver.setVortParameter(N, &cent, omega));
    solver.computeFarFieldBuffer();
    CK(solver.lastOk());
    CK(solver.setEvalParameter(N, &cent));
    CK(solver.evaluateVelocity(&cent, 1));
    cudaDeviceSynchronize();

    std::vector<double> u(3 * (size_t)N);
    for (int c = 0; c < 3; c++)
        cudaMemcpy(u.data() + c * (size_t)N, solver.getU(c), 8 * (size_t)N, cudaMemcpyDeviceToHost);
    const double h = solver.getCellh();
    const double4_ o = solver.getOrigin();

    // ParticleManager with the solver's grid (PH/SpaceHashClass.h:46-54)
    ParticleManager pm;
    pm.initSpatialHash(N, n, n, n);
    const float of[3] = {(float)o.x, (float)o.y, (float)o.z};
    pm.setSpatialHashGrid(n, (float)h, of, N);
    pm.setHashParam();
    pm.doSpatialHash(dpos, N);
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

    // MultiGridSolver3DPeriod_double on b = u-component grid-sized slice
    const size_t C = (size_t)n * n * n;
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
    std::vector<double> x(C);
    cudaDeviceSynchronize();
    cudaMemcpy(x.data(), dx, 8 * C, cudaMemcpyDeviceToHost);

    // PotentialFieldSolver: masses = the x strengths at the vortex positions,
    // gradient evaluated at the same positions (HFS/PotentialFieldSolver.h)
    PotentialFieldSolver pf;
    CK(pf.initializeSolver(n, n, n, 1, N, N));
    CK(pf.setMassParameter(N, &cent, &vx));
    CK(pf.setEvalParameter(N, &cent));
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
    std::fclose(g);
    solver.shutdown();
    std::printf("ok N=%u n=%u\n", N, n);
    return 0;
}
