// Geometric multigrid for sum_nbr(x) - 6x = b with zero ghost values, the
// operator of MG/MultiGrid_kernel.cu:722-934 (the "periodic" kernels zero
// every neighbour outside the box).
//
// Schedule (MG/MultiGrid.cpp:128-250): full multigrid — restrict b to every
// level, solve the coarsest, then per level prolong + V(4,4) — followed by one
// more V(4,4) at the finest level.  Levels halve while the level has more than
// 512 cells (MG/MultiGrid.h:114-127).  Red-black SOR, omega = 1.43f, odd
// cells (i+j+k odd) first (MG/Multigrid.cu:202-239); residual
// b - (sum_nbr - 6x); restriction 0.5 * sum of the 8 children; prolongation
// by injection; 100 Jacobi sweeps on the coarsest level
// (MG/MultiGrid_kernel.cu:422-498; the reference updates in place from 512
// racing threads, Jacobi is its race-free reading).
//
// Precision: the full-multigrid part runs in FP32.  The final V-cycle runs as
// an FP64 defect correction — r = b - A psi in FP64, an FP32 V-cycle on
// A e = r from e = 0, psi += e in FP64 — which equals the reference's
// V(psi, b) in exact arithmetic because the V-cycle is a consistent linear
// iteration.  The coarsest solve is FP64.  Every kernel handles the three
// potential components of a scene in one launch (grid y = component).
#include <cmath>

#include "pppm_internal.cuh"

namespace pppm {

namespace {

constexpr float kOmegaF = 1.43f;
constexpr float kOneMinusOmegaF = 1.0f - 1.43f;  // formed in float, MG/MultiGrid_kernel.cu:766
constexpr int kMGThreads = 256;

__device__ __forceinline__ float nb_sum(const float *__restrict__ x, int i, int j, int k, int d, size_t c) {
    const size_t dd = (size_t)d * d;
    const float lv = (i > 0) ? x[c - 1] : 0.f;
    const float rv = (i < d - 1) ? x[c + 1] : 0.f;
    const float uv = (j < d - 1) ? x[c + d] : 0.f;
    const float dv = (j > 0) ? x[c - d] : 0.f;
    const float fv = (k > 0) ? x[c - dd] : 0.f;
    const float bv = (k < d - 1) ? x[c + dd] : 0.f;
    return ((lv + rv) + (uv + dv)) + (fv + bv);
}

__device__ __forceinline__ double nb_sum64(const double *__restrict__ x, int i, int j, int k, int d, size_t c) {
    const size_t dd = (size_t)d * d;
    const double lv = (i > 0) ? x[c - 1] : 0.0;
    const double rv = (i < d - 1) ? x[c + 1] : 0.0;
    const double uv = (j < d - 1) ? x[c + d] : 0.0;
    const double dv = (j > 0) ? x[c - d] : 0.0;
    const double fv = (k > 0) ? x[c - dd] : 0.0;
    const double bv = (k < d - 1) ? x[c + dd] : 0.0;
    return ((lv + rv) + (uv + dv)) + (fv + bv);
}

// log2(d) for a power-of-two edge, else -1: index arithmetic then uses shifts
// instead of integer division (every level of the 32..512 grids).
inline int edge_log2(int d) {
    if (d <= 0 || (d & (d - 1))) return -1;
    int l = 0;
    while ((1 << l) < d) l++;
    return l;
}

// t -> (i, j, k) on an a x d x d index box (x fastest); la = log2(a) or -1,
// ld = log2(d) or -1.
__device__ __forceinline__ void split3(uint32_t t, int a, int d, int la, int ld, int &i, int &j, int &k) {
    if (la >= 0 && ld >= 0) {
        i = (int)(t & (uint32_t)(a - 1));
        j = (int)((t >> la) & (uint32_t)(d - 1));
        k = (int)(t >> (la + ld));
    } else {
        i = (int)(t % (uint32_t)a);
        j = (int)((t / (uint32_t)a) % (uint32_t)d);
        k = (int)(t / ((uint32_t)a * (uint32_t)d));
    }
}

// One half sweep over the cells with (i+j+k) % 2 == color.
__global__ void __launch_bounds__(kMGThreads)
rbsor_kernel(float *__restrict__ x, const float *__restrict__ b, int d, int color, int ld) {
    const int half = d >> 1;
    const uint32_t per = (uint32_t)half * d * d;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= per) return;
    const size_t comp = blockIdx.y;
    const size_t cells = (size_t)d * d * d;
    float *xc = x + comp * cells;
    const float *bc = b + comp * cells;
    int ih, j, k;
    split3(t, half, d, ld > 0 ? ld - 1 : -1, ld, ih, j, k);
    const int i = 2 * ih + ((j + k + color) & 1);
    const size_t c = ((size_t)k * d + j) * d + i;
    const float r = nb_sum(xc, i, j, k, d, c) - bc[c];
    xc[c] = kOneMinusOmegaF * xc[c] + (kOmegaF * r) * (1.0f / 6.0f);
}

// Residual at the fine level restricted to the coarse level in one pass:
// bc = 0.5 * sum over the 8 children of (bf - (sum_nbr(xf) - 6 xf)).
__global__ void __launch_bounds__(kMGThreads)
resid_restrict_kernel(const float *__restrict__ xf, const float *__restrict__ bf, float *__restrict__ bc,
                      int dc, int x_zero, int ldc) {
    const uint32_t per = (uint32_t)dc * dc * dc;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= per) return;
    const size_t comp = blockIdx.y;
    const int df = 2 * dc;
    const size_t fcells = (size_t)df * df * df;
    const float *x = xf + comp * fcells;
    const float *b = bf + comp * fcells;
    int ic, jc, kc;
    split3(t, dc, dc, ldc, ldc, ic, jc, kc);
    float sum = 0.f;
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const int i = 2 * ic + (q & 1), j = 2 * jc + ((q >> 1) & 1), k = 2 * kc + (q >> 2);
        const size_t c = ((size_t)k * df + j) * df + i;
        float r = b[c];
        if (!x_zero) r -= nb_sum(x, i, j, k, df, c) - 6.f * x[c];
        sum += r;
    }
    bc[comp * per + t] = sum * 0.5f;
}

__global__ void __launch_bounds__(kMGThreads)
prolong_kernel(float *__restrict__ xf, const float *__restrict__ xc, int df, int ldf) {
    const uint32_t per = (uint32_t)df * df * df;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= per) return;
    const size_t comp = blockIdx.y;
    const int dc = df >> 1;
    int i, j, k;
    split3(t, df, df, ldf, ldf, i, j, k);
    xf[comp * per + t] += xc[comp * (size_t)dc * dc * dc + ((size_t)(k >> 1) * dc + (j >> 1)) * dc + (i >> 1)];
}

// Coarsest level: 100 Jacobi sweeps x <- (sum_nbr(x) - b) / 6 in FP64
// shared memory, one block per component, d^3 <= 512.
__global__ void __launch_bounds__(512) coarse_kernel(float *__restrict__ x, const float *__restrict__ b, int d) {
    __shared__ double xa[512], xb[512], bb[512];
    const int cells = d * d * d;
    const size_t comp = blockIdx.x;
    const int t = threadIdx.x;
    if (t < cells) {
        xa[t] = (double)x[comp * cells + t];
        bb[t] = (double)b[comp * cells + t];
    }
    __syncthreads();
    const int i = t % d, j = (t / d) % d, k = t / (d * d);
    double *cur = xa, *nxt = xb;
    for (int it = 0; it < 100; it++) {
        if (t < cells) {
            double r = nb_sum64(cur, i, j, k, d, (size_t)t);
            r -= bb[t];
            nxt[t] = r / 6;
        }
        __syncthreads();
        double *tmp = cur; cur = nxt; nxt = tmp;
    }
    if (t < cells) x[comp * cells + t] = (float)cur[t];
}

// The coarsest solve always starts from x = 0 in the reference schedule at
// two or more levels, so its 100 Jacobi sweeps are one fixed linear map
// x = P b.  Column j of P is the sweep applied to the unit vector e_j (one
// block per column); P is stored row-major [row][col].
__global__ void __launch_bounds__(512) coarse_op_column_kernel(double *__restrict__ op, int d) {
    __shared__ double xa[512], xb[512];
    const int cells = d * d * d;
    const int col = blockIdx.x;
    const int t = threadIdx.x;
    if (t < cells) xa[t] = 0.0;
    __syncthreads();
    const int i = t % d, j = (t / d) % d, k = t / (d * d);
    double *cur = xa, *nxt = xb;
    for (int it = 0; it < 100; it++) {
        if (t < cells) {
            double r = nb_sum64(cur, i, j, k, d, (size_t)t);
            r -= (t == col) ? 1.0 : 0.0;
            nxt[t] = r / 6;
        }
        __syncthreads();
        double *tmp = cur; cur = nxt; nxt = tmp;
    }
    if (t < cells) op[(size_t)t * cells + col] = cur[t];
}

// x = P b per component: one warp per (row, component), lanes stride the row.
__global__ void __launch_bounds__(256)
coarse_apply_kernel(const double *__restrict__ op, float *__restrict__ x, const float *__restrict__ b, int cells,
                    int comps) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= cells * comps) return;
    const int row = warp % cells, comp = warp / cells;
    const double *prow = op + (size_t)row * cells;
    const float *bc = b + (size_t)comp * cells;
    double acc = 0.0;
    for (int c = lane; c < cells; c += 32) acc = fma(prow[c], (double)bc[c], acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) x[(size_t)comp * cells + row] = (float)acc;
}

// r = b - (sum_nbr(psi) - 6 psi) in FP64, stored as the FP32 right-hand side
// of the correction equation.  b is read from b64 (FP64) or formed as
// -(vort * h2f) from the FP32 P2M grid.  Optional squared norms of r and b.
__global__ void __launch_bounds__(kMGThreads)
dc_residual_kernel(const double *__restrict__ psi, const double *__restrict__ b64, const float *__restrict__ vort,
                   const DevParams *__restrict__ P, float *__restrict__ rout, int d, int ld,
                   double *__restrict__ norms) {
    const uint32_t per = (uint32_t)d * d * d;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t comp = blockIdx.y;
    double r2 = 0.0, b2 = 0.0;
    if (t < per) {
        const double *x = psi + comp * per;
        int i, j, k;
        split3(t, d, d, ld, ld, i, j, k);
        double bv;
        if (b64)
            bv = b64[comp * per + t];
        else
            bv = (double)(-(vort[comp * per + t] * P->h2f));
        const double r = bv - (nb_sum64(x, i, j, k, d, t) - 6.0 * x[t]);
        rout[comp * per + t] = (float)r;
        r2 = r * r;
        b2 = bv * bv;
    }
    if (norms) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            r2 += __shfl_xor_sync(0xffffffffu, r2, o);
            b2 += __shfl_xor_sync(0xffffffffu, b2, o);
        }
        __shared__ double sr[kMGThreads / 32], sb[kMGThreads / 32];
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (lane == 0) { sr[warp] = r2; sb[warp] = b2; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double a = 0.0, c = 0.0;
            for (int w = 0; w < kMGThreads / 32; w++) { a += sr[w]; c += sb[w]; }
            atomicAdd(&norms[0], a);
            atomicAdd(&norms[1], c);
        }
    }
}

__global__ void dc_update_kernel(double *__restrict__ psi, const float *__restrict__ x, size_t count, int init) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    psi[t] = (init ? 0.0 : psi[t]) + (double)x[t];
}

inline dim3 grid_for(uint32_t per, int comps) { return dim3((per + kMGThreads - 1) / kMGThreads, comps); }

// Coarsest solve from x = 0: the precomputed operator when available, else
// the sweeps themselves.
void coarse_solve(const MGPlan &m) {
    const Level &c = m.lv[m.levels - 1];
    ::pppm::note_launch();
    if (m.coarse_op && m.levels >= 2) {
        const unsigned warps = c.cells * (unsigned)m.comps;
        coarse_apply_kernel<<<(warps * 32 + 255) / 256, 256, 0, m.st>>>(m.coarse_op, c.x, c.b, (int)c.cells, m.comps);
    } else {
        coarse_kernel<<<m.comps, 512, 0, m.st>>>(c.x, c.b, (int)c.d);
    }
}

}  // namespace

cudaError_t build_coarse_operator(int d, double *op, cudaStream_t st) {
    ::pppm::note_launch();
    coarse_op_column_kernel<<<d * d * d, 512, 0, st>>>(op, d);
    return cudaGetLastError();
}

int mg_level_count(uint32_t n) {
    // MG/MultiGrid.h:114-127
    long long x = n;
    int L = 0;
    while (x * x * x > 512) {
        L++;
        x = x / 2;
        if (x == 0) x = 1;
    }
    return L + 1;
}

// Every level above the coarsest must have an even edge, or restriction and
// prolongation would index outside the coarse grid.
bool mg_shape_ok(uint32_t n) {
    const int L = mg_level_count(n);
    uint32_t d = n;
    for (int l = 0; l < L - 1; l++) {
        if (d & 1u) return false;
        d >>= 1;
    }
    return true;
}

// One FP32 V(4,4) cycle from level `level` down (MG/MultiGrid.cpp:128-201).
static cudaError_t vcycle32(const MGPlan &m, int level) {
    const int L = m.levels;
    for (int j = level + 1; j < L; j++)
        PPPM_CUDA_TRY(cudaMemsetAsync(m.lv[j].x, 0, sizeof(float) * m.comps * (size_t)m.lv[j].cells, m.st));
    for (int j = level; j < L - 1; j++) {
        const int d = (int)m.lv[j].d;
        const dim3 g = grid_for((uint32_t)(d / 2) * d * d, m.comps);
        for (int it = 0; it < 4; it++) {
            ::pppm::note_launch();
            rbsor_kernel<<<g, kMGThreads, 0, m.st>>>(m.lv[j].x, m.lv[j].b, d, 1, edge_log2(d));
            ::pppm::note_launch();
            rbsor_kernel<<<g, kMGThreads, 0, m.st>>>(m.lv[j].x, m.lv[j].b, d, 0, edge_log2(d));
        }
        ::pppm::note_launch();
        resid_restrict_kernel<<<grid_for(m.lv[j + 1].cells, m.comps), kMGThreads, 0, m.st>>>(
            m.lv[j].x, m.lv[j].b, m.lv[j + 1].b, (int)m.lv[j + 1].d, 0, edge_log2((int)m.lv[j + 1].d));
    }
    coarse_solve(m);
    for (int j = L - 2; j >= level; j--) {
        const int d = (int)m.lv[j].d;
        ::pppm::note_launch();
        prolong_kernel<<<grid_for(m.lv[j].cells, m.comps), kMGThreads, 0, m.st>>>(m.lv[j].x, m.lv[j + 1].x, d,
                                                                                  edge_log2(d));
        const dim3 g = grid_for((uint32_t)(d / 2) * d * d, m.comps);
        for (int it = 0; it < 4; it++) {
            ::pppm::note_launch();
            rbsor_kernel<<<g, kMGThreads, 0, m.st>>>(m.lv[j].x, m.lv[j].b, d, 1, edge_log2(d));
            ::pppm::note_launch();
            rbsor_kernel<<<g, kMGThreads, 0, m.st>>>(m.lv[j].x, m.lv[j].b, d, 0, edge_log2(d));
        }
    }
    return cudaGetLastError();
}

// Full multigrid in FP32 with lv[0].b holding the right-hand side
// (MG/MultiGrid.cpp:202-246; x = 0 on entry, so the residual chain is a
// plain restriction of b).
static cudaError_t fmg32(const MGPlan &m) {
    const int L = m.levels;
    for (int j = 0; j < L; j++)
        PPPM_CUDA_TRY(cudaMemsetAsync(m.lv[j].x, 0, sizeof(float) * m.comps * (size_t)m.lv[j].cells, m.st));
    for (int j = 0; j < L - 1; j++) {
        ::pppm::note_launch();
        resid_restrict_kernel<<<grid_for(m.lv[j + 1].cells, m.comps), kMGThreads, 0, m.st>>>(
            m.lv[j].x, m.lv[j].b, m.lv[j + 1].b, (int)m.lv[j + 1].d, 1, edge_log2((int)m.lv[j + 1].d));
    }
    coarse_solve(m);
    PPPM_CUDA_TRY(cudaGetLastError());
    for (int j = L - 2; j >= 0; j--) {
        ::pppm::note_launch();
        prolong_kernel<<<grid_for(m.lv[j].cells, m.comps), kMGThreads, 0, m.st>>>(
            m.lv[j].x, m.lv[j + 1].x, (int)m.lv[j].d, edge_log2((int)m.lv[j].d));
        PPPM_CUDA_TRY(vcycle32(m, j));
    }
    return cudaGetLastError();
}

// FP64 residual of the current psi, stored as the FP32 right-hand side of the
// correction equation (optionally with squared norms of r and b).
static cudaError_t dc_residual(const MGPlan &m, bool want_norms) {
    const uint32_t C0 = m.lv[0].cells;
    if (want_norms) PPPM_CUDA_TRY(cudaMemsetAsync(m.norms, 0, 2 * sizeof(double), m.st));
    ::pppm::note_launch();
    dc_residual_kernel<<<grid_for(C0, m.comps), kMGThreads, 0, m.st>>>(m.psi, m.b64, m.vort, m.P, m.lv[0].b,
                                                                       (int)m.lv[0].d, edge_log2((int)m.lv[0].d),
                                                                       want_norms ? m.norms : nullptr);
    return cudaGetLastError();
}

// e = V32(0, r); psi += e.
static cudaError_t dc_correct(const MGPlan &m) {
    const uint32_t C0 = m.lv[0].cells;
    PPPM_CUDA_TRY(cudaMemsetAsync(m.lv[0].x, 0, sizeof(float) * m.comps * (size_t)C0, m.st));
    PPPM_CUDA_TRY(vcycle32(m, 0));
    const size_t cnt = (size_t)m.comps * C0;
    ::pppm::note_launch();
    dc_update_kernel<<<(unsigned)((cnt + 255) / 256), 256, 0, m.st>>>(m.psi, m.lv[0].x, cnt, 0);
    return cudaGetLastError();
}

// One V(4,4) cycle applied to an FP64 iterate x64 as a defect correction:
// lv[0].b already holds r = b - A x64 (FP32), then e = V32(0, r) and
// x64 += e — the reference's m_Vcycle(x, b) in exact arithmetic, the V-cycle
// being a consistent linear iteration (MG/MultiGrid.cpp:128-201).
cudaError_t mg_vcycle_update(const MGPlan &m, double *x64) {
    const uint32_t C0 = m.lv[0].cells;
    PPPM_CUDA_TRY(cudaMemsetAsync(m.lv[0].x, 0, sizeof(float) * m.comps * (size_t)C0, m.st));
    PPPM_CUDA_TRY(vcycle32(m, 0));
    const size_t cnt = (size_t)m.comps * C0;
    ::pppm::note_launch();
    dc_update_kernel<<<(unsigned)((cnt + 255) / 256), 256, 0, m.st>>>(x64, m.lv[0].x, cnt, 0);
    return cudaGetLastError();
}

static cudaError_t read_relres(const MGPlan &m, double *relres) {
    double h[2];
    PPPM_CUDA_TRY(cudaMemcpyAsync(h, m.norms, sizeof(h), cudaMemcpyDeviceToHost, m.st));
    PPPM_CUDA_TRY(cudaStreamSynchronize(m.st));
    *relres = h[1] > 0 ? std::sqrt(h[0] / h[1]) : 0.0;
    return cudaSuccess;
}

// Whole solve: FMG in FP32, psi = x0, then the reference's final V-cycle as
// an FP64 defect correction (this completes m_FullMultiGrid; cycles = 1).
// CONVERGED then adds correction cycles while ||r||/||b|| > tol and
// cycles < max_cycles, and reports the relative residual of the final psi.
cudaError_t mg_solve(const MGPlan &m, int mode, double tol, int max_cycles, int *cycles_out, double *relres_out) {
    PPPM_CUDA_TRY(fmg32(m));
    const size_t cnt = (size_t)m.comps * m.lv[0].cells;
    ::pppm::note_launch();
    dc_update_kernel<<<(unsigned)((cnt + 255) / 256), 256, 0, m.st>>>(m.psi, m.lv[0].x, cnt, 1);
    PPPM_CUDA_TRY(cudaGetLastError());
    PPPM_CUDA_TRY(dc_residual(m, false));
    PPPM_CUDA_TRY(dc_correct(m));
    int cycles = 1;
    double rel = -1.0;
    if (mode == PPPM_MG_CONVERGED) {
        for (;;) {
            PPPM_CUDA_TRY(dc_residual(m, true));
            PPPM_CUDA_TRY(read_relres(m, &rel));
            if (!(rel > tol) || cycles >= max_cycles) break;
            PPPM_CUDA_TRY(dc_correct(m));
            cycles++;
        }
    }
    if (cycles_out) *cycles_out = cycles;
    if (relres_out) *relres_out = rel;
    return cudaSuccess;
}

// Captures the reference-schedule solve (no host synchronisation inside) as a
// CUDA graph on a private stream; the graph is replayed on the scene stream.
cudaError_t mg_capture_graph(const MGPlan &m_in, cudaGraphExec_t *exec, unsigned *kernel_nodes) {
    MGPlan m = m_in;
    cudaStream_t cap = nullptr;
    PPPM_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    m.st = cap;
    cudaGraph_t g = nullptr;
    const unsigned long long before = launch_count();
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaError_t body = mg_solve(m, PPPM_MG_REFERENCE, 0.0, 1, nullptr, nullptr);
        e = cudaStreamEndCapture(cap, &g);
        if (e == cudaSuccess) e = body;
    }
    *kernel_nodes = (unsigned)(launch_count() - before);
    if (e == cudaSuccess) e = cudaGraphInstantiate(exec, g, 0);
    if (g) cudaGraphDestroy(g);
    cudaStreamDestroy(cap);
    return e;
}

static MGPlan scene_plan(pppm_scene *s) {
    MGPlan m;
    m.levels = s->levels;
    for (int l = 0; l < s->levels; l++) m.lv[l] = s->lv[l];
    m.comps = 3;
    m.st = s->stream;
    m.psi = s->psi;
    m.b64 = nullptr;
    m.vort = s->vort;
    m.P = s->dparams;
    m.norms = s->norms;
    m.coarse_op = s->coarse_op;
    return m;
}

// Captures the scene's reference-schedule graph (called at scene creation,
// under the device lock).
cudaError_t prepare_multigrid_graph(pppm_scene *s) {
    if (s->prm.mg_mode != PPPM_MG_REFERENCE || s->mg_graph) return cudaSuccess;
    std::lock_guard<std::recursive_mutex> lk(device_lock());
    return mg_capture_graph(scene_plan(s), &s->mg_graph, &s->mg_graph_kernels);
}

cudaError_t run_multigrid(pppm_scene *s) {
    MGPlan m;
    m.levels = s->levels;
    for (int l = 0; l < s->levels; l++) m.lv[l] = s->lv[l];
    m.comps = 3;
    m.st = s->stream;
    m.psi = s->psi;
    m.b64 = nullptr;
    m.vort = s->vort;
    m.P = s->dparams;
    m.norms = s->norms;
    m.coarse_op = s->coarse_op;
    int cyc = 0;
    double rel = -1.0;
    if (s->prm.mg_mode == PPPM_MG_REFERENCE) {
        if (!s->mg_graph) PPPM_CUDA_TRY(prepare_multigrid_graph(s));
        PPPM_CUDA_TRY(cudaGraphLaunch(s->mg_graph, s->stream));
        for (unsigned q = 0; q < s->mg_graph_kernels; q++) note_launch();
        s->mg_cycles_last = 1;
        s->mg_relres_last = -1.0;
        return cudaSuccess;
    }
    PPPM_CUDA_TRY(mg_solve(m, s->prm.mg_mode, s->prm.mg_tol, s->prm.mg_max_cycles, &cyc, &rel));
    s->mg_cycles_last = cyc;
    s->mg_relres_last = rel;
    return cudaSuccess;
}

}  // namespace pppm
