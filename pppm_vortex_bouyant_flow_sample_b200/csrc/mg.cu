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
//
// Where the level's edge allows, the half sweeps and the prolongation take a
// group of 4 consecutive cells of a row per thread and the restriction a pair
// of coarse cells, with 128-bit loads; their values equal the one-cell
// kernels' bit for bit.  The temporally blocked smoother of mg_tb.cu is
// opt-in (PPPM_MG_TB), as it measured slower inside a whole solve.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <mutex>

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

// The SOR update of one cell from its neighbour sum and right-hand side
// (MG/MultiGrid_kernel.cu:766, omega = 1.43f), one expression for every
// smoother kernel so that they round alike.
__device__ __forceinline__ float sor_update(float x, float nb, float b) {
    const float r = nb - b;
    return kOneMinusOmegaF * x + (kOmegaF * r) * (1.0f / 6.0f);
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
    xc[c] = sor_update(xc[c], nb_sum(xc, i, j, k, d, c), bc[c]);
}

__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }

// The same half sweep with a thread per group of 4 consecutive cells of a
// row (edge a multiple of 4): it updates the group's 2 cells of the colour
// from 128-bit loads of its row, the rows and planes either side and b, plus
// one scalar either side, with nb_sum's terms in nb_sum's order (the values
// equal rbsor_kernel's bit for bit).  Half the threads of rbsor_kernel, and
// every loaded sector fully used.
__global__ void __launch_bounds__(kMGThreads)
rbsor4_kernel(float *__restrict__ x, const float *__restrict__ b, int d, int color, int ld) {
    const int q = d >> 2;  // groups per row
    const uint32_t per = (uint32_t)q * d * d;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= per) return;
    const size_t comp = blockIdx.y;
    const size_t cells = (size_t)d * d * d, dd = (size_t)d * d;
    float *xc = x + comp * cells;
    const float *bc = b + comp * cells;
    int g, j, k;
    split3(t, q, d, ld >= 2 ? ld - 2 : -1, ld, g, j, k);
    const int i0 = 4 * g;
    const size_t c = ((size_t)k * d + j) * d + i0;
    const bool odd = ((j + k + color) & 1) != 0;  // the colour's cells: i0 + odd, i0 + odd + 2
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 v = ld4(xc + c);
    const float xl = i0 > 0 ? xc[c - 1] : 0.f;
    const float xr = i0 + 4 < d ? xc[c + 4] : 0.f;
    const float4 up = (j < d - 1) ? ld4(xc + c + d) : z4;
    const float4 dn = (j > 0) ? ld4(xc + c - d) : z4;
    const float4 fr = (k > 0) ? ld4(xc + c - dd) : z4;
    const float4 bk = (k < d - 1) ? ld4(xc + c + dd) : z4;
    const float4 bb = ld4(bc + c);
    const float nb_lo = (((odd ? v.x : xl) + (odd ? v.z : v.y)) + ((odd ? up.y : up.x) + (odd ? dn.y : dn.x))) +
                        ((odd ? fr.y : fr.x) + (odd ? bk.y : bk.x));
    const float nb_hi = (((odd ? v.z : v.y) + (odd ? xr : v.w)) + ((odd ? up.w : up.z) + (odd ? dn.w : dn.z))) +
                        ((odd ? fr.w : fr.z) + (odd ? bk.w : bk.z));
    const int o = odd ? 1 : 0;
    xc[c + o] = sor_update(odd ? v.y : v.x, nb_lo, odd ? bb.y : bb.x);
    xc[c + o + 2] = sor_update(odd ? v.w : v.z, nb_hi, odd ? bb.w : bb.z);
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

// The same with a thread per pair of coarse cells along x (coarse edge even):
// their 16 fine children, 4 consecutive cells in each of the 4 fine rows
// (j, k) in {2jc, 2jc+1} x {2kc, 2kc+1}, read with 128-bit loads of the rows,
// their neighbour rows and b.  The rows are taken in the children's order
// (x fastest, then y, then z), so each coarse sum adds the same terms in the
// same order as resid_restrict_kernel.
__global__ void __launch_bounds__(kMGThreads)
resid_restrict2_kernel(const float *__restrict__ xf, const float *__restrict__ bf, float *__restrict__ bc,
                       int dc, int x_zero, int ldc) {
    const int h = dc >> 1;  // coarse pairs per row
    const uint32_t per2 = (uint32_t)h * dc * dc;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= per2) return;
    const size_t comp = blockIdx.y;
    const int df = 2 * dc;
    const size_t fcells = (size_t)df * df * df, dd = (size_t)df * df;
    const float *x = xf + comp * fcells;
    const float *b = bf + comp * fcells;
    int ip, jc, kc;
    split3(t, h, dc, ldc >= 1 ? ldc - 1 : -1, ldc, ip, jc, kc);
    const int i0 = 4 * ip;
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    float s0 = 0.f, s1 = 0.f;
#pragma unroll
    for (int rrow = 0; rrow < 4; rrow++) {
        const int j = 2 * jc + (rrow & 1), k = 2 * kc + (rrow >> 1);
        const size_t c = ((size_t)k * df + j) * df + i0;
        const float4 bb = ld4(b + c);
        float r[4] = {bb.x, bb.y, bb.z, bb.w};
        if (!x_zero) {
            const float4 v = ld4(x + c);
            const float xl = i0 > 0 ? x[c - 1] : 0.f;
            const float xr = i0 + 4 < df ? x[c + 4] : 0.f;
            const float4 up = (j < df - 1) ? ld4(x + c + df) : z4;
            const float4 dn = (j > 0) ? ld4(x + c - df) : z4;
            const float4 fr = (k > 0) ? ld4(x + c - dd) : z4;
            const float4 bk = (k < df - 1) ? ld4(x + c + dd) : z4;
            const float xs[6] = {xl, v.x, v.y, v.z, v.w, xr};
            const float us[4] = {up.x, up.y, up.z, up.w}, ds[4] = {dn.x, dn.y, dn.z, dn.w};
            const float fs[4] = {fr.x, fr.y, fr.z, fr.w}, bs[4] = {bk.x, bk.y, bk.z, bk.w};
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const float nb = ((xs[e] + xs[e + 2]) + (us[e] + ds[e])) + (fs[e] + bs[e]);
                r[e] -= nb - 6.f * xs[e + 1];
            }
        }
        s0 += r[0];
        s0 += r[1];
        s1 += r[2];
        s1 += r[3];
    }
    *reinterpret_cast<float2 *>(bc + comp * (size_t)dc * dc * dc + ((size_t)kc * dc + jc) * dc + 2 * ip) =
        make_float2(s0 * 0.5f, s1 * 0.5f);
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

// The same prolongation by injection with a thread per group of 4 fine cells
// of a row (fine edge a multiple of 4): one 128-bit read-modify-write of the
// fine cells and the 2 coarse cells under them (each cell gets the same single
// addition as in prolong_kernel).
__global__ void __launch_bounds__(kMGThreads)
prolong4_kernel(float *__restrict__ xf, const float *__restrict__ xc, int df, int ldf) {
    const int q = df >> 2;
    const uint32_t per = (uint32_t)q * df * df;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= per) return;
    const size_t comp = blockIdx.y;
    const int dc = df >> 1;
    int g, j, k;
    split3(t, q, df, ldf >= 2 ? ldf - 2 : -1, ldf, g, j, k);
    float4 *f = reinterpret_cast<float4 *>(xf + comp * (size_t)df * df * df + ((size_t)k * df + j) * df + 4 * g);
    const float *cr = xc + comp * (size_t)dc * dc * dc + ((size_t)(k >> 1) * dc + (j >> 1)) * dc + 2 * g;
    const float c0 = cr[0], c1 = cr[1];
    float4 v = *f;
    v.x += c0;
    v.y += c0;
    v.z += c1;
    v.w += c1;
    *f = v;
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

// Where a level's x lives between kernels of the blocked smoother.
enum XAt { kXZero = 0, kXMain = 1, kXAlt = 2 };

static bool tb_level(const MGPlan &m, int j) { return m.tb_var[j] >= 0 && m.lv[j].x2; }

static float *x_ptr(const MGPlan &m, int j, XAt at) { return at == kXAlt ? m.lv[j].x2 : m.lv[j].x; }

// Four red-black iterations (8 half sweeps, odd cells first) at level j,
// starting from `in` (zero, or x in one of the two copies) plus, when xc is
// set, the injected coarse correction xc[parent] (the prolongation that
// precedes the reference's post-smoothing).  Blocked levels run 8 / T passes
// of the blocked smoother, ping-ponging between the two copies; the others run
// the half sweeps in place on the main copy.  Returns where the result is:
// a pre-smoothing from zero ends in the main copy for an even pass count and
// in the second copy for an odd one, a post-smoothing from there always ends
// in the main copy.
// bc = the restricted residual of the level above (a pair of coarse cells per
// thread where the coarse edge is even).
static void launch_restrict(const MGPlan &m, const float *xf, const float *bf, float *bc, int dc, int x_zero) {
    if ((dc % 2) == 0)
        resid_restrict2_kernel<<<grid_for((uint32_t)(dc / 2) * dc * dc, m.comps), kMGThreads, 0, m.st>>>(
            xf, bf, bc, dc, x_zero, edge_log2(dc));
    else
        resid_restrict_kernel<<<grid_for((uint32_t)dc * dc * dc, m.comps), kMGThreads, 0, m.st>>>(
            xf, bf, bc, dc, x_zero, edge_log2(dc));
}

// x += the coarser level's xc injected (a group of 4 cells per thread where
// the edge allows).
static void launch_prolong(const MGPlan &m, float *x, const float *xc, int d) {
    if ((d % 4) == 0)
        prolong4_kernel<<<grid_for((uint32_t)(d / 4) * d * d, m.comps), kMGThreads, 0, m.st>>>(x, xc, d,
                                                                                                edge_log2(d));
    else
        prolong_kernel<<<grid_for((uint32_t)d * d * d, m.comps), kMGThreads, 0, m.st>>>(x, xc, d, edge_log2(d));
}

static cudaError_t smooth(const MGPlan &m, int j, XAt in, const float *xc, XAt *out) {
    const Level &L = m.lv[j];
    const int d = (int)L.d;
    if (tb_level(m, j)) {
        int T = 0, TX = 0, TY = 0;
        tb_variant_shape(m.tb_var[j], &T, &TX, &TY);
        const int passes = 8 / T;
        if (xc && !m.tb_fuse_prolong) {
            // the prolongation as its own kernel into the pass's input
            const XAt at = (in == kXZero) ? kXMain : in;
            float *dst = x_ptr(m, j, at);
            if (in == kXZero) PPPM_CUDA_TRY(cudaMemsetAsync(dst, 0, sizeof(float) * m.comps * (size_t)L.cells, m.st));
            ::pppm::note_launch();
            launch_prolong(m, dst, xc, d);
            in = at;
            xc = nullptr;
        }
        XAt cur = in;
        for (int p = 0; p < passes; p++) {
            const XAt dst = (cur == kXAlt) ? kXMain : kXAlt;
            const CUtensorMap &mx = (cur == kXAlt) ? m.tb_maps[j].x2 : m.tb_maps[j].x;
            PPPM_CUDA_TRY(tb_smooth(m.tb_var[j], mx, m.tb_maps[j].b, L.b, cur != kXZero, p == 0 ? xc : nullptr,
                                    x_ptr(m, j, dst), d, m.comps, m.tb_zchunk[j], m.err, m.st));
            cur = dst;
        }
        *out = cur;
        return cudaSuccess;
    }
    if (in == kXZero) PPPM_CUDA_TRY(cudaMemsetAsync(L.x, 0, sizeof(float) * m.comps * (size_t)L.cells, m.st));
    if (xc) {
        ::pppm::note_launch();
        launch_prolong(m, L.x, xc, d);
    }
    if ((d % 4) == 0) {
        const dim3 g = grid_for((uint32_t)(d / 4) * d * d, m.comps);
        for (int it = 0; it < 4; it++) {
            ::pppm::note_launch();
            rbsor4_kernel<<<g, kMGThreads, 0, m.st>>>(L.x, L.b, d, 1, edge_log2(d));
            ::pppm::note_launch();
            rbsor4_kernel<<<g, kMGThreads, 0, m.st>>>(L.x, L.b, d, 0, edge_log2(d));
        }
    } else {
        const dim3 g = grid_for((uint32_t)(d / 2) * d * d, m.comps);
        for (int it = 0; it < 4; it++) {
            ::pppm::note_launch();
            rbsor_kernel<<<g, kMGThreads, 0, m.st>>>(L.x, L.b, d, 1, edge_log2(d));
            ::pppm::note_launch();
            rbsor_kernel<<<g, kMGThreads, 0, m.st>>>(L.x, L.b, d, 0, edge_log2(d));
        }
    }
    *out = kXMain;
    return cudaGetLastError();
}

// One FP32 V(4,4) cycle from level `level` down (MG/MultiGrid.cpp:128-201).
// The cycle's x at `level` starts at zero plus, when xc is set, the injected
// correction from level + 1 (the full multigrid's prolongation); the coarser
// levels start at zero as the reference zeroes them.  The result is left in
// lv[level].x.
static cudaError_t vcycle32(const MGPlan &m, int level, const float *xc = nullptr) {
    const int L = m.levels;
    XAt at[kMaxLevels];
    for (int j = level; j < L - 1; j++) {
        PPPM_CUDA_TRY(smooth(m, j, kXZero, j == level ? xc : nullptr, &at[j]));
        ::pppm::note_launch();
        launch_restrict(m, x_ptr(m, j, at[j]), m.lv[j].b, m.lv[j + 1].b, (int)m.lv[j + 1].d, 0);
    }
    // the coarsest solve starts from zero (a cycle on the coarsest level alone
    // included: it is only ever asked for from a zero start)
    if (level == L - 1 || !m.coarse_op)
        PPPM_CUDA_TRY(cudaMemsetAsync(m.lv[L - 1].x, 0, sizeof(float) * m.comps * (size_t)m.lv[L - 1].cells, m.st));
    coarse_solve(m);
    for (int j = L - 2; j >= level; j--) {
        XAt res;
        PPPM_CUDA_TRY(smooth(m, j, at[j], m.lv[j + 1].x, &res));
    }
    return cudaGetLastError();
}

// Full multigrid in FP32 with lv[0].b holding the right-hand side
// (MG/MultiGrid.cpp:202-246; x = 0 on entry, so the residual chain is a
// plain restriction of b).
static cudaError_t fmg32(const MGPlan &m) {
    const int L = m.levels;
    for (int j = 0; j < L - 1; j++) {
        ::pppm::note_launch();
        launch_restrict(m, m.lv[j].x, m.lv[j].b, m.lv[j + 1].b, (int)m.lv[j + 1].d, 1);
    }
    PPPM_CUDA_TRY(cudaMemsetAsync(m.lv[L - 1].x, 0, sizeof(float) * m.comps * (size_t)m.lv[L - 1].cells, m.st));
    coarse_solve(m);
    PPPM_CUDA_TRY(cudaGetLastError());
    for (int j = L - 2; j >= 0; j--) PPPM_CUDA_TRY(vcycle32(m, j, m.lv[j + 1].x));
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

size_t mg_tb_extra_floats(const MGPlan &m) {
    size_t f = 0;
    for (int j = 0; j < m.levels; j++)
        if (m.lv[j].d >= m.tb_min_edge && (m.lv[j].d % 4) == 0) f += (size_t)m.comps * m.lv[j].cells;
    return f;
}

// z-chunk length of a level for a variant: fill the resident CTA slots in
// whole waves, each chunk paying 2T extra planes of pipeline start and end.
static int pick_zchunk(int d, int comps, int variant, int sms, int per_sm) {
    int T = 0, TX = 0, TY = 0;
    tb_variant_shape(variant, &T, &TX, &TY);
    const long slots = (long)sms * std::max(per_sm, 1);
    const long tiles = (long)((d + TX - 1) / TX) * ((d + TY - 1) / TY) * comps;
    const long cmax = std::max(1L, (long)(d / (2 * T)));
    long best_c = 1;
    double best = -1.0;
    for (long c = 1; c <= cmax; c++) {
        const long zc = (d + c - 1) / c, n_cta = tiles * ((d + zc - 1) / zc);
        const long waves = (n_cta + slots - 1) / slots;
        const double eff = (double)n_cta / (double)(waves * slots) * (double)zc / (double)(zc + 2 * T);
        if (eff > best + 1e-9) {
            best = eff;
            best_c = c;
        }
    }
    return (int)((d + best_c - 1) / best_c);
}

namespace {
// Autotuner results: fastest smoother (variant, or -1 for the plain half
// sweeps) per (device, level edge, components), measured once per process.
struct TuneKey {
    int dev, d, comps;
    bool operator==(const TuneKey &o) const { return dev == o.dev && d == o.d && comps == o.comps; }
};
struct TuneEntry {
    TuneKey key;
    int variant;
    float ms[16];  // measured time of 8 half sweeps per candidate (index variant + 1)
};
std::mutex g_tune_mutex;
TuneEntry g_tune[64];
int g_tune_count = 0;
}  // namespace

// Times 8 half sweeps (four red-black iterations) of level j with the plain
// kernels and with every blocked variant, on the level's own buffers (zeroed
// first), and returns the fastest.  Every candidate computes the same values
// bit for bit, so the choice only changes the time.
static cudaError_t tune_level(MGPlan &m, int j, int sms, int dev, int *best_out, float *ms_out) {
    Level &L = m.lv[j];
    const int d = (int)L.d;
    const int nvar = tb_variant_count();
    cudaStream_t st = nullptr;
    PPPM_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    const size_t bytes = sizeof(float) * m.comps * (size_t)L.cells;
    if (e == cudaSuccess) e = cudaMemsetAsync(L.x, 0, bytes, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(L.x2, 0, bytes, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(L.b, 0, bytes, st);
    int best = -1;
    float best_ms = 1e30f;
    for (int v = -1; v < nvar && e == cudaSuccess; v++) {
        MGPlan t = m;
        t.st = st;
        for (int q = 0; q < kMaxLevels; q++) t.tb_var[q] = -1;
        if (v >= 0) {
            int per_sm = 1;
            e = tb_prepare(v, &per_sm);
            if (e == cudaSuccess) e = tb_make_map(&t.tb_maps[j].x, L.x, d, m.comps, v);
            if (e == cudaSuccess) e = tb_make_map(&t.tb_maps[j].x2, L.x2, d, m.comps, v);
            if (e == cudaSuccess) e = tb_make_map(&t.tb_maps[j].b, L.b, d, m.comps, v);
            if (e != cudaSuccess) break;
            t.tb_var[j] = v;
            t.tb_zchunk[j] = pick_zchunk(d, m.comps, v, sms, per_sm);
        }
        float tmin = 1e30f;
        for (int rep = 0; rep < 4 && e == cudaSuccess; rep++) {
            XAt out;
            e = cudaEventRecord(e0, st);
            if (e == cudaSuccess) e = smooth(t, j, kXMain, nullptr, &out);
            if (e == cudaSuccess) e = cudaEventRecord(e1, st);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float ms = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0) tmin = std::min(tmin, ms);  // the first run warms up
        }
        if (e != cudaSuccess) break;
        if (v + 1 < 16) ms_out[v + 1] = tmin;
        if (tmin < best_ms) {
            best_ms = tmin;
            best = v;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    *best_out = best;
    (void)dev;
    return e;
}

// Points each qualifying level's x2 into `pool` (mg_tb_extra_floats floats),
// picks its smoother — `forced` (a variant, or -1 for the plain half sweeps)
// when >= -1, else the autotuner's choice — and builds its tensor maps and
// z-chunk.
cudaError_t mg_tb_setup(MGPlan &m, float *pool, int forced) {
    for (int j = 0; j < kMaxLevels; j++) m.tb_var[j] = -1;
    if (!pool) return cudaSuccess;
    {
        // Once the blocked smoother (up to ~200 KB of shared memory per CTA)
        // has run, the SMs stay partitioned for shared memory unless a kernel
        // asks otherwise; the plain stencil kernels read their neighbours
        // through L1 and measured 11% slower at 128^3 in that state.  They
        // ask for the largest L1.
        static std::once_flag once;
        static cudaError_t carve = cudaSuccess;
        std::call_once(once, [] {
            const void *k[] = {(const void *)rbsor_kernel, (const void *)rbsor4_kernel,
                               (const void *)prolong4_kernel, (const void *)resid_restrict_kernel,
                               (const void *)resid_restrict2_kernel,
                               (const void *)prolong_kernel, (const void *)dc_residual_kernel,
                               (const void *)dc_update_kernel};
            for (const void *f : k)
                if (carve == cudaSuccess)
                    carve = cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout,
                                                 cudaSharedmemCarveoutMaxL1);
        });
        PPPM_CUDA_TRY(carve);
    }
    int dev = 0, sms = 148;
    PPPM_CUDA_TRY(cudaGetDevice(&dev));
    PPPM_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const char *f = getenv("PPPM_MG_TB_FUSE");
    m.tb_fuse_prolong = (f && *f == '1');
    for (int j = 0; j < m.levels; j++) {
        Level &L = m.lv[j];
        if (!(L.d >= m.tb_min_edge && (L.d % 4) == 0)) continue;
        L.x2 = pool;
        pool += (size_t)m.comps * L.cells;
    }
    for (int j = 0; j < m.levels; j++) {
        Level &L = m.lv[j];
        if (!L.x2) continue;
        int v = forced;
        if (forced < -1) {
            const TuneKey key{dev, (int)L.d, m.comps};
            bool found = false;
            {
                std::lock_guard<std::mutex> lk(g_tune_mutex);
                for (int q = 0; q < g_tune_count; q++)
                    if (g_tune[q].key == key) { v = g_tune[q].variant; found = true; }
            }
            if (!found) {
                TuneEntry te{};
                te.key = key;
                for (float &x : te.ms) x = -1.f;
                PPPM_CUDA_TRY(tune_level(m, j, sms, dev, &te.variant, te.ms));
                v = te.variant;
                std::lock_guard<std::mutex> lk(g_tune_mutex);
                if (g_tune_count < 64) g_tune[g_tune_count++] = te;
            }
        }
        if (v < 0 || v >= tb_variant_count()) continue;
        int per_sm = 1;
        PPPM_CUDA_TRY(tb_prepare(v, &per_sm));
        PPPM_CUDA_TRY(tb_make_map(&m.tb_maps[j].x, L.x, (int)L.d, m.comps, v));
        PPPM_CUDA_TRY(tb_make_map(&m.tb_maps[j].x2, L.x2, (int)L.d, m.comps, v));
        PPPM_CUDA_TRY(tb_make_map(&m.tb_maps[j].b, L.b, (int)L.d, m.comps, v));
        m.tb_zchunk[j] = pick_zchunk((int)L.d, m.comps, v, sms, per_sm);
        m.tb_var[j] = v;
    }
    return cudaSuccess;
}

// Text summary of the autotuner's measurements (one line per level edge).
size_t mg_tune_report(char *buf, size_t cap) {
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    size_t w = 0;
    auto put = [&](const char *fmt, auto... args) {
        if (w < cap) {
            const int k = snprintf(buf + w, cap - w, fmt, args...);
            if (k > 0) w += (size_t)k;
        }
    };
    for (int q = 0; q < g_tune_count; q++) {
        const TuneEntry &t = g_tune[q];
        put("edge %d comps %d: chosen %d; ms per 8 half sweeps: plain %.4f", t.key.d, t.key.comps, t.variant,
            (double)t.ms[0]);
        for (int v = 0; v + 1 < 16 && v < tb_variant_count(); v++) {
            int T = 0, TX = 0, TY = 0, G4 = 0;
            tb_variant_shape(v, &T, &TX, &TY, &G4);
            put(", v%d(T%d %dx%d%s) %.4f", v, T, TX, TY, G4 ? " g4" : "", (double)t.ms[v + 1]);
        }
        put("\n");
    }
    return w < cap ? w : cap;
}

// The plain half sweeps (rbsor4_kernel) measured faster inside a whole solve
// than every blocked variant at 96^3 to 256^3 (256^3: 5.67 ms against 5.85 ms
// with the autotuner's pick), and once a blocked pass has run, its large
// shared-memory split slows the plain stencil kernels that follow.  So the
// plain sweeps are the default; PPPM_MG_TB=auto runs the autotuner, an index
// forces a variant.
int mg_tb_default_variant() {
    const char *e = getenv("PPPM_MG_TB");
    if (e && *e) {
        if (strcmp(e, "auto") == 0) return -2;
        const int v = atoi(e);
        return (v >= 0 && v < tb_variant_count()) ? v : -1;
    }
    return -1;
}

static MGPlan scene_plan(pppm_scene *s) {
    MGPlan m = s->mg_tb;  // blocked-smoother variant, maps, z-chunks, error flag
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
    MGPlan m = scene_plan(s);
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
