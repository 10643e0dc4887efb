// C entry point over the reference's own FP64 multigrid kernels
// (multigrid/MultiGrid_kernel.cu, included where it lies, with texref_compat.h
// pre-included for its texture references).  TEST INFRASTRUCTURE ONLY: the
// parity tests run it on the GPU as a checker of the oracle's and the
// product's multigrid.
//
// The reference's launch wrappers (multigrid/Multigrid.cu) and its solver class
// (multigrid/MultiGrid.cpp, MultiGrid.h) include OpenGL headers, so they are
// not compiled here.  Their steps are restated below: the launch shapes and
// arguments of the FP64 wrappers (Multigrid.cu:29-55, 202-330), the level rule
// (MultiGrid.h:114-127), the V-cycle and the full multigrid of
// MultiGridSolver3DPeriod_double (MultiGrid.cpp:128-250), and the per-component
// solve of BiotSavartSolver::m_SolvePoisson (HFS/BiotSavartSolverImp.cpp:603-620:
// psi = 0, then one full multigrid).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "helper_cuda.h"
#include "MultiGrid_kernel.cu"

namespace {

struct Dims {
    int x, y, z;
    size_t cells() const { return (size_t)x * y * z; }
};

// Device time of every launch and memset when timing is on: each is
// bracketed by CUDA events (the bindings synchronise the device anyway).
bool g_time = false;
double g_ms = 0.0;
template <class F>
void timed(F f) {
    if (!g_time) {
        f();
        return;
    }
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a);
    f();
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    g_ms += t;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
}

// the texture stand-in reads through a managed pointer: no launch may still be
// reading the old binding when it changes
void bind(const void *p, const textureReference *t) {
    cudaDeviceSynchronize();
    size_t off = 0;
    bindTextureDouble(&off, p, t, 0);
}

dim3 grid_for(const Dims &d) {
    return dim3(d.x / 32 + ((d.x % 32) ? 1 : 0), d.z * d.y / 16 + (((d.z * d.y) % 16) ? 1 : 0));
}

// mg_RBGS_periodic3D2 (Multigrid.cu:202-239): t x (red, black) sweeps in place
void rbgs(double *x, double *b, int t, const Dims &d) {
    for (int i = 0; i < t; i++) {
        bind(x, &x_level_tex_double);
        bind(b, &b_level_tex_double);
        const dim3 threads(32, 16);
        const dim3 blocks = grid_for(d);
        timed([&] {
            red_sweep_GS_periodic_kerneld_type2<<<blocks, threads>>>(
                x, d.x, d.y, d.z, 1.0 / (double)d.y, 1.0 / (double)(d.x * d.y), d.x * d.y, d.x, d.x - 1,
                (d.y - 1) * d.x, (d.z - 1) * d.x * d.y, 1.0 / 6.0, 0, 0, (uint)d.cells());
        });
        timed([&] {
            black_sweep_GS_periodic_kerneld_type2<<<blocks, threads>>>(
                x, d.x, d.y, d.z, 1.0 / (double)d.y, 1.0 / (double)(d.x * d.y), d.x * d.y, d.x, d.x - 1,
                (d.y - 1) * d.x, (d.z - 1) * d.x * d.y, 1.0 / 6.0, 0, 0, (uint)d.cells());
        });
    }
}

// mg_ComputeResidualPeriodic3D2 (Multigrid.cu:241-273)
void residual(double *x, double *b, double *r, const Dims &d) {
    bind(x, &x_level_tex_double);
    bind(b, &b_level_tex_double);
    timed([&] {
        compute_residual_periodic_kernel2<<<grid_for(d), dim3(32, 16)>>>(
            x, b, r, d.x, d.y, d.z, 1.0 / (double)d.y, 1.0 / (double)(d.x * d.y), d.x * d.y, d.x, d.x - 1,
            (d.y - 1) * d.x, (d.z - 1) * d.x * d.y, 1.0 / 6.0, 0, 0, (uint)d.cells());
    });
}

// mg_RestrictionPeriodic3D2 (Multigrid.cu:275-301): next from the fine r
void restrict_to(double *next, double *cur, const Dims &nd) {
    bind(cur, &b_level_tex_double);
    timed([&] {
        restriction_periodic_kernel2<<<grid_for(nd), dim3(32, 16)>>>(
            next, nd.x, nd.y, nd.z, 1.0 / (double)nd.y, 1.0 / (double)(nd.x * nd.y), nd.x * nd.y * 4, nd.x * 2,
            nd.x - 1, (nd.y - 1) * nd.x, (nd.z - 1) * nd.x * nd.y, 1.0 / 6.0, 0, (uint)nd.cells());
    });
}

// mg_ProlongationPeriodic3D2 (Multigrid.cu:303-330): next += coarse
void prolong_into(double *next, double *coarse, const Dims &nd) {
    bind(coarse, &x_level_tex_double);
    timed([&] {
        prolongation_periodic_kernel2<<<grid_for(nd), dim3(32, 16)>>>(
            next, nd.x, nd.y, nd.z, 1.0 / (double)nd.y, 1.0 / (double)(nd.x * nd.y), nd.x * nd.y / 4, nd.x / 2,
            nd.x - 1, (nd.y - 1) * nd.x, (nd.z - 1) * nd.x * nd.y, 1.0 / 6.0, 0, (uint)nd.cells());
    });
}

// mg_exact_periodic3D2 (Multigrid.cu:46-55)
void exact(double *x, double *b, double *res, const Dims &d) {
    cudaDeviceSynchronize();
    timed([&] {
        exact_solve_period3D_jacobi_kerneld<<<1, std::min<int>(512, (int)d.cells())>>>(b, x, res, d.x, d.y, d.z,
                                                                                       (uint)d.cells());
    });
}

struct Solver {
    std::vector<Dims> sys;
    std::vector<double *> xk, bk, rk;
    int L = 0;

    void zero(double *p, const Dims &d) {
        timed([&] { cudaMemset(p, 0, sizeof(double) * d.cells()); });
    }

    // MultiGridSolver3DPeriod_double::m_Vcycle (MultiGrid.cpp:128-201)
    void vcycle(double *x, double *b, int level) {
        xk[level] = x;
        bk[level] = b;
        for (int i = level + 1; i < L; i++) {
            zero(xk[i], sys[i]);
            zero(bk[i], sys[i]);
            zero(rk[i], sys[i]);
        }
        zero(rk[level], sys[level]);
        for (int i = level; i < L - 1; ++i) {
            rbgs(xk[i], bk[i], 4, sys[i]);
            residual(xk[i], bk[i], rk[i], sys[i]);
            restrict_to(bk[i + 1], rk[i], sys[i + 1]);
        }
        exact(xk[L - 1], bk[L - 1], xk[L - 1], sys[L - 1]);
        for (int i = L - 2; i >= level; --i) {
            prolong_into(xk[i], xk[i + 1], sys[i]);
            rbgs(xk[i], bk[i], 4, sys[i]);
        }
        for (int i = level + 1; i < L; i++) {
            zero(xk[i], sys[i]);
            zero(bk[i], sys[i]);
            zero(rk[i], sys[i]);
        }
    }

    // MultiGridSolver3DPeriod_double::m_FullMultiGrid (MultiGrid.cpp:202-250)
    void fmg(double *x, double *b) {
        xk[0] = x;
        bk[0] = b;
        for (int i = 1; i < L; i++) {
            zero(xk[i], sys[i]);
            zero(bk[i], sys[i]);
            zero(rk[i], sys[i]);
        }
        zero(rk[0], sys[0]);
        for (int i = 0; i < L - 1; ++i) {
            residual(xk[i], bk[i], rk[i], sys[i]);
            restrict_to(bk[i + 1], rk[i], sys[i + 1]);
        }
        exact(xk[L - 1], bk[L - 1], xk[L - 1], sys[L - 1]);
        for (int i = L - 2; i >= 0; --i) {
            prolong_into(xk[i], xk[i + 1], sys[i]);
            vcycle(xk[i], bk[i], i);
        }
        vcycle(xk[0], b, 0);
    }
};

}  // namespace

// Solves sum_nbr(x) - 6x = b (zero ghost values) for comps right-hand sides
// on an n^3 grid, each from x = 0 by `repeats` full multigrids in a row, each
// from the x the previous one left: BiotSavartSolver::m_SolvePoisson runs one
// per component, PotentialFieldSolver::m_SolvePoisson three
// (HFS/PotentialFieldSolver.cpp:610-619).  b_host, x_host: [comps][n^3] FP64.
// ms (may be NULL): the summed device time of the solves' launches and
// memsets.  Returns 0 or a CUDA error code.
extern "C" int refgpu_mg_fmg(uint32_t n, uint32_t comps, uint32_t repeats, const double *b_host, double *x_host,
                             float *ms) {
    g_time = ms != nullptr;
    g_ms = 0.0;
    Solver S;
    // MultiGrid<T>::m_ComputeLevels (MultiGrid.h:114-127)
    Dims d{(int)n, (int)n, (int)n};
    S.sys.push_back(d);
    while ((long long)d.x * d.y * d.z > 512) {
        d.x = std::max(d.x / 2, 1);
        d.y = std::max(d.y / 2, 1);
        d.z = std::max(d.z / 2, 1);
        S.sys.push_back(d);
    }
    S.L = (int)S.sys.size();
    S.xk.assign(S.L, nullptr);
    S.bk.assign(S.L, nullptr);
    S.rk.assign(S.L, nullptr);
    std::vector<double *> owned;
    auto alloc = [&](size_t cells) {
        double *p = nullptr;
        if (cudaMalloc(&p, sizeof(double) * std::max<size_t>(cells, 1)) != cudaSuccess) return (double *)nullptr;
        owned.push_back(p);
        return p;
    };
    bool ok = true;
    for (int i = 1; i < S.L; i++) {
        S.xk[i] = alloc(S.sys[i].cells());
        S.bk[i] = alloc(S.sys[i].cells());
        S.rk[i] = alloc(S.sys[i].cells());
        ok = ok && S.xk[i] && S.bk[i] && S.rk[i];
    }
    S.rk[0] = alloc(S.sys[0].cells());
    double *x0 = alloc(S.sys[0].cells()), *b0 = alloc(S.sys[0].cells());
    ok = ok && S.rk[0] && x0 && b0;
    int rc = 0;
    if (ok) {
        // MultiGrid<T>::m_InitialSystem: the coarsest level's neighbour tables
        initIdxBuffer(S.sys[S.L - 1].x, S.sys[S.L - 1].y, S.sys[S.L - 1].z);
        const size_t C = S.sys[0].cells();
        for (uint32_t c = 0; c < comps && rc == 0; c++) {
            cudaMemcpy(b0, b_host + c * C, sizeof(double) * C, cudaMemcpyHostToDevice);
            timed([&] { cudaMemset(x0, 0, sizeof(double) * C); });   // m_SolvePoisson: psi = 0
            for (uint32_t r = 0; r < repeats; r++) S.fmg(x0, b0);
            cudaError_t e = cudaDeviceSynchronize();
            if (e == cudaSuccess) e = cudaMemcpy(x_host + c * C, x0, sizeof(double) * C, cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) rc = (int)e;
        }
    } else {
        rc = (int)cudaErrorMemoryAllocation;
    }
    for (double *p : owned) cudaFree(p);
    if (ms) *ms = (float)g_ms;
    g_time = false;
    return rc;
}
