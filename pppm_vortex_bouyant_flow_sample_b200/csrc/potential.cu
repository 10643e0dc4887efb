// Scalar PPPM: the reference's PotentialFieldSolver
// (HFS/PotentialFieldSolver.cpp:45-739, kernels HFS/GPU_kernel.cu:524-1748 and
// 2977-3115), the boundary-element companion of the vortex path: masses
// (sources of a single-layer potential) on a grid, a Poisson solve with the
// monopole as Dirichlet data, and evaluation of the potential or its
// gradient at arbitrary points with a near-field particle correction.
//
//   setDomain            2 x the mass bounding box (:343-373)
//   m_ParticleToMesh     reference hash, NGP deposit rho = sum m / h^3,
//                        rhs = -h^2 rho, monopole (total mass, |m|-weighted
//                        centre), applyDirichlet: each boundary cell's rhs
//                        loses M / (4 pi |ghost - centre|) per outside face
//   m_SolvePoisson       phi = 0, then three full-multigrid calls, each from
//                        the current phi (pppm_mg_full_multigrid)
//   gradient buffer      periodic central differences of phi, minus the
//                        mesh's own near-field image over the (2K+1)^3 cells
//                        (Green's-gradient table) and the diagonal term
//                        (PotentialComputeFarField :988-1197)
//   scalar buffer        phi minus sum G_ij rho h^2 over the (2K+1)^3 cells
//                        (G_ii = 0.25, G_ij = 1 / (4 pi d)) (:1200-1298)
//   evaluation           hat-weighted interpolation over 5^3 cells plus the
//                        particle correction inside the (K+0.5)h box
//                        (gradient: 1/r^3 kernel, core a = 0.05; potential:
//                        1/r kernel, core a = 0.125, the cell range shifted
//                        towards the point's half of its cell); gradients at
//                        points outside the grid box are zero
//
// Grids and sums are FP64 as in the reference; one thread per cell or per
// evaluation point, points visited in hash order.
#include <algorithm>
#include <cmath>

#include "pppm_internal.cuh"

extern "C" __attribute__((visibility("hidden"))) void pppm_set_error(const char *fmt, ...);

struct pppm_potential {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t n = 0, C = 0;
    int K = 1;
    uint32_t capN = 0, capM = 0;
    uint32_t N = 0;
    // masses
    float4 *mpos = nullptr;
    double *mass = nullptr;
    uint32_t *key[2] = {nullptr, nullptr}, *idx[2] = {nullptr, nullptr};
    uint32_t *hist = nullptr;
    size_t hist_cap = 0;
    uint32_t *sidx = nullptr;
    uint32_t *start = nullptr, *end = nullptr;
    float4 *srec = nullptr;   // sorted {rel.x, rel.y, rel.z, 0}
    double *smass = nullptr;  // sorted masses
    // grids (FP64)
    double *density = nullptr, *rhs = nullptr, *phi = nullptr, *far = nullptr;  // far: [3][C] or [C]
    double *mono = nullptr;   // [4] centre, total mass
    double *mono_part = nullptr;
    float *bbox = nullptr, *host_bbox = nullptr;
    pppm_mg *mg = nullptr;
    // evaluation order
    uint32_t *ekey[2] = {nullptr, nullptr}, *eidx[2] = {nullptr, nullptr};
    // domain of the last build
    double origin[3] = {0, 0, 0}, L = 0, cell_h = 0;
    float h_f = 0, of[3] = {0, 0, 0};
    int built = 0;  // 0 none, 1 gradient buffer, 2 scalar buffer
};

namespace pppm {
namespace {

constexpr int kRedBlocks = 296;
constexpr double kG = 1.0;  // G * direction of the reference's calls (single-layer potential)

__global__ void pot_bbox_kernel(const float4 *__restrict__ pos, uint32_t N, float *__restrict__ out) {
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < N; t += gridDim.x * blockDim.x) {
        const float4 p = pos[t];
        mn[0] = fminf(mn[0], p.x); mn[1] = fminf(mn[1], p.y); mn[2] = fminf(mn[2], p.z);
        mx[0] = fmaxf(mx[0], p.x); mx[1] = fmaxf(mx[1], p.y); mx[2] = fmaxf(mx[2], p.z);
    }
    __shared__ float sh[6][8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        for (int o = 16; o > 0; o >>= 1) {
            mn[c] = fminf(mn[c], __shfl_xor_sync(0xffffffffu, mn[c], o));
            mx[c] = fmaxf(mx[c], __shfl_xor_sync(0xffffffffu, mx[c], o));
        }
        if (lane == 0) { sh[c][w] = mn[c]; sh[3 + c][w] = mx[c]; }
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int c = threadIdx.x;
        float v = sh[c][0];
        for (int q = 1; q < (int)(blockDim.x >> 5); q++) v = c < 3 ? fminf(v, sh[c][q]) : fmaxf(v, sh[c][q]);
        out[c * gridDim.x + blockIdx.x] = v;
    }
}

__global__ void pot_records_kernel(const float4 *__restrict__ pos, const double *__restrict__ mass,
                                   const uint32_t *__restrict__ sidx, uint32_t N, double ox, double oy, double oz,
                                   float4 *__restrict__ srec, double *__restrict__ smass) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    const uint32_t i = sidx[s];
    const float4 p = pos[i];
    srec[s] = make_float4((float)((double)p.x - ox), (float)((double)p.y - oy), (float)((double)p.z - oz), 0.f);
    smass[s] = mass[i];
}

// ParticleToMesh_kernel (HFS/GPU_kernel.cu:218-294): a particle adds m to the
// cell whose centre lies within half a cell on every axis (NGP, in FP64 on
// the float relative coordinate).  That cell is the particle's hash cell or a
// neighbour, so the 3^3 hash cells around the grid cell hold every candidate.
// Then rhs = -(h_f^2) rho (ComputeRHS, h_f^2 rounded to float).
__global__ void pot_p2m_kernel(const uint32_t *__restrict__ start, const uint32_t *__restrict__ end,
                               const float4 *__restrict__ srec, const double *__restrict__ smass, int d,
                               double invh, double h2, double *__restrict__ rho, double *__restrict__ rhs) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (uint32_t)d * d * d) return;
    const int i = (int)(c % d), j = (int)((c / d) % d), k = (int)(c / ((uint32_t)d * d));
    const double gx = (double)(float)((double)i + 0.5), gy = (double)(float)((double)j + 0.5),
                 gz = (double)(float)((double)k + 0.5);
    double sum = 0.0;
    for (int kk = max(k - 1, 0); kk <= min(k + 1, d - 1); kk++)
        for (int jj = max(j - 1, 0); jj <= min(j + 1, d - 1); jj++)
            for (int ii = max(i - 1, 0); ii <= min(i + 1, d - 1); ii++) {
                const uint32_t r = ((uint32_t)kk * d + jj) * d + ii;
                const uint32_t s0 = start[r];
                if (s0 == kEmpty) continue;
                const uint32_t s1 = end[r];
                for (uint32_t p = s0; p < s1; p++) {
                    const float4 q = srec[p];
                    const double r1 = (double)q.x * invh - gx, r2 = (double)q.y * invh - gy,
                                 r3 = (double)q.z * invh - gz;
                    if (r1 < 0.5 && r1 >= -0.5 && r2 < 0.5 && r2 >= -0.5 && r3 < 0.5 && r3 >= -0.5) sum += 1.0 * smass[p];
                }
            }
    const double v = invh * invh * invh * sum;
    rho[c] = v;
    rhs[c] = v * h2 * -1.0;
}

// Monopole of the masses (m_ParticleToMesh :578-596): sum |m|, sum m and the
// |m|-weighted sum of positions, in FP64; per block, then one block in order.
__global__ void pot_mono_partial_kernel(const float4 *__restrict__ pos, const double *__restrict__ mass, uint32_t N,
                                        double *__restrict__ part) {
    double a[5] = {0, 0, 0, 0, 0};
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < N; t += gridDim.x * blockDim.x) {
        const double m = mass[t], am = fabs(m);
        const float4 p = pos[t];
        a[0] += am;
        a[1] += m;
        a[2] += (double)p.x * am;
        a[3] += (double)p.y * am;
        a[4] += (double)p.z * am;
    }
    __shared__ double sh[5][8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 5; q++) {
        for (int o = 16; o > 0; o >>= 1) a[q] += __shfl_xor_sync(0xffffffffu, a[q], o);
        if (lane == 0) sh[q][w] = a[q];
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        double v = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) v += sh[threadIdx.x][q];
        part[threadIdx.x * gridDim.x + blockIdx.x] = v;
    }
}

__global__ void pot_mono_final_kernel(const double *__restrict__ part, int nb, double *__restrict__ mono) {
    if (threadIdx.x != 0) return;
    double a[5] = {0, 0, 0, 0, 0};
    for (int q = 0; q < 5; q++)
        for (int b = 0; b < nb; b++) a[q] += part[q * nb + b];
    mono[0] = a[2] / a[0];
    mono[1] = a[3] / a[0];
    mono[2] = a[4] / a[0];
    mono[3] = a[1];
}

// compute_r (HFS/GPU_kernel.cu:204-211): 4 pi |r1 - r2|, 1e12 when coincident.
__device__ __forceinline__ double compute_r(double ax, double ay, double az, double bx, double by, double bz) {
    const double r_sqr = (ax - bx) * (ax - bx) + (ay - by) * (ay - by) + (az - bz) * (az - bz);
    return r_sqr > 1e-12 ? kFourPi * sqrt(r_sqr) : 1e+12;
}

// apply_Dirichlet_kernel (HFS/GPU_kernel.cu:2977-3115), faces in the
// reference's order (-x, +x, -y, +y, -z, +z).
__global__ void pot_dirichlet_kernel(double *__restrict__ rhs, const double *__restrict__ mono, int d, double h,
                                     double ox, double oy, double oz) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (uint32_t)d * d * d) return;
    const int i = (int)(c % d), j = (int)((c / d) % d), k = (int)(c / ((uint32_t)d * d));
    if (i != 0 && i != d - 1 && j != 0 && j != d - 1 && k != 0 && k != d - 1) return;
    const double cx = mono[0], cy = mono[1], cz = mono[2], M = mono[3];
    double r = rhs[c];
    auto ghost = [&](double gi, double gj, double gk) {
        r -= M / compute_r(gi * h + ox, gj * h + oy, gk * h + oz, cx, cy, cz);
    };
    if (i == 0) ghost((double)i - 1.0 + 0.5, (double)j + 0.5, (double)k + 0.5);
    if (i == d - 1) ghost((double)i + 1.0 + 0.5, (double)j + 0.5, (double)k + 0.5);
    if (j == 0) ghost((double)i + 0.5, (double)j - 1.0 + 0.5, (double)k + 0.5);
    if (j == d - 1) ghost((double)i + 0.5, (double)j + 1.0 + 0.5, (double)k + 0.5);
    if (k == 0) ghost((double)i + 0.5, (double)j + 0.5, (double)k - 1.0 + 0.5);
    if (k == d - 1) ghost((double)i + 0.5, (double)j + 0.5, (double)k + 1.0 + 0.5);
    rhs[c] = r;
}

__device__ __forceinline__ void periodic_grad(const double *__restrict__ f, int d, uint32_t c, int i, int j, int k,
                                              double invh, double g[3]) {
    const uint32_t dd = (uint32_t)d * d;
    const double l = f[c - i + (i + d - 1) % d], r = f[c - i + (i + 1) % d];
    const double dn = f[c - j * d + ((j + d - 1) % d) * d], t = f[c - j * d + ((j + 1) % d) * d];
    const double fr = f[c - k * dd + ((k + d - 1) % d) * dd], b = f[c - k * dd + ((k + 1) % d) * dd];
    g[0] = 1.0 * (r - l) * 0.5 * invh;
    g[1] = 1.0 * (t - dn) * 0.5 * invh;
    g[2] = 1.0 * (b - fr) * 0.5 * invh;
}

// Gradient buffer: far = grad(phi) - sum_{c' != 0} D[c'] m(c + c')
// - grad(0.250580605913965 rho h^2), every gradient periodic central
// differences; D is the central-difference gradient of 1/(4 pi r) between
// cell centres, built per block in shared memory.
__global__ void pot_far_gradient_kernel(const double *__restrict__ phi, const double *__restrict__ rho, int d, int K,
                                        double h, double *__restrict__ far) {
    extern __shared__ double table[];  // [3][(2K+1)^3]
    const int W = 2 * K + 1, T = W * W * W;
    for (int e = threadIdx.x; e < T; e += blockDim.x) {
        const int ii = e % W - K, jj = (e / W) % W - K, kk = e / (W * W) - K;
        double tx = 0, ty = 0, tz = 0;
        if (!(ii == 0 && jj == 0 && kk == 0)) {
            const double Xpx = ((double)ii + 0.5) * h, Xpy = ((double)jj + 0.5) * h, Xpz = ((double)kk + 0.5) * h;
            const double Xx = 0.5 * h, Xy = 0.5 * h, Xz = 0.5 * h;
            auto inv_r = [](double ax, double ay, double az, double bx, double by, double bz) {
                const double r_sqr = (ax - bx) * (ax - bx) + (ay - by) * (ay - by) + (az - bz) * (az - bz);
                return 1.0 / ((r_sqr > 1e-12) ? kFourPi * sqrt(r_sqr) : 1e+24);
            };
            tx = 0.5 * (inv_r(Xx + h, Xy, Xz, Xpx, Xpy, Xpz) - inv_r(Xx - h, Xy, Xz, Xpx, Xpy, Xpz)) / h;
            ty = 0.5 * (inv_r(Xx, Xy + h, Xz, Xpx, Xpy, Xpz) - inv_r(Xx, Xy - h, Xz, Xpx, Xpy, Xpz)) / h;
            tz = 0.5 * (inv_r(Xx, Xy, Xz + h, Xpx, Xpy, Xpz) - inv_r(Xx, Xy, Xz - h, Xpx, Xpy, Xpz)) / h;
        }
        table[e] = tx;
        table[T + e] = ty;
        table[2 * T + e] = tz;
    }
    __syncthreads();
    const uint32_t C = (uint32_t)d * d * d;
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    const int i = (int)(c % d), j = (int)((c / d) % d), k = (int)(c / ((uint32_t)d * d));
    const double invh = 1.0 / h;
    double g[3];
    periodic_grad(phi, d, c, i, j, k, invh, g);
    double fm[3] = {0, 0, 0};
    const double v = h * h * h;
    for (int kk = k - K; kk <= k + K; kk++)
        for (int jj = j - K; jj <= j + K; jj++)
            for (int ii = i - K; ii <= i + K; ii++) {
                if (!(kk >= 0 && kk < d && jj >= 0 && jj < d && ii >= 0 && ii < d)) continue;
                const double m = kG * rho[((uint32_t)kk * d + jj) * d + ii] * v;
                const int e = ((kk - k + K) * W + (jj - j + K)) * W + (ii - i + K);
                fm[0] += table[e] * m;
                fm[1] += table[T + e] * m;
                fm[2] += table[2 * T + e] * m;
            }
    // diagonal term: its periodic gradient from the six neighbours' densities
    const double dg = 0.250580605913965 * h * h * kG;
    const uint32_t dd = (uint32_t)d * d;
    const double rl = rho[c - i + (i + d - 1) % d], rr = rho[c - i + (i + 1) % d];
    const double rd = rho[c - j * d + ((j + d - 1) % d) * d], rt = rho[c - j * d + ((j + 1) % d) * d];
    const double rf = rho[c - k * dd + ((k + d - 1) % d) * dd], rb = rho[c - k * dd + ((k + 1) % d) * dd];
    const double gd[3] = {1.0 * (dg * rr - dg * rl) * 0.5 * invh, 1.0 * (dg * rt - dg * rd) * 0.5 * invh,
                          1.0 * (dg * rb - dg * rf) * 0.5 * invh};
    far[c] = (g[0] - fm[0]) - gd[0];
    far[C + c] = (g[1] - fm[1]) - gd[1];
    far[2 * (size_t)C + c] = (g[2] - fm[2]) - gd[2];
}

__global__ void pot_gradient_only_kernel(const double *__restrict__ phi, int d, double h, double *__restrict__ far) {
    const uint32_t C = (uint32_t)d * d * d;
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    const int i = (int)(c % d), j = (int)((c / d) % d), k = (int)(c / ((uint32_t)d * d));
    double g[3];
    periodic_grad(phi, d, c, i, j, k, 1.0 / h, g);
    far[c] = g[0];
    far[C + c] = g[1];
    far[2 * (size_t)C + c] = g[2];
}

// Scalar buffer: phi - sum over the (2K+1)^3 cells of G_ij rho h^2.
__global__ void pot_far_scalar_kernel(const double *__restrict__ phi, const double *__restrict__ rho, int d, int K,
                                      double h, double *__restrict__ far) {
    const uint32_t C = (uint32_t)d * d * d;
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    const int i = (int)(c % d), j = (int)((c / d) % d), k = (int)(c / ((uint32_t)d * d));
    double s = 0.0;
    for (int kk = k - K; kk <= k + K; kk++)
        for (int jj = j - K; jj <= j + K; jj++)
            for (int ii = i - K; ii <= i + K; ii++) {
                if (!(kk >= 0 && kk < d && jj >= 0 && jj < d && ii >= 0 && ii < d)) continue;
                const double m = kG * rho[((uint32_t)kk * d + jj) * d + ii] * (h * h);
                double w;
                if (i == ii && j == jj && k == kk) {
                    w = 0.25;
                } else {
                    const double x = (double)ii - (double)i, y = (double)jj - (double)j, z = (double)kk - (double)k;
                    w = 1.0 / (kFourPi * sqrt(x * x + y * y + z * z));
                }
                s += w * m;
            }
    far[c] = phi[c] - s;
}

__global__ void pot_eval_keys_kernel(const float4 *__restrict__ pos, uint32_t M, double ox, double oy, double oz,
                                     double invh, int d, uint32_t *__restrict__ key, uint32_t *__restrict__ idx) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M) return;
    const float4 p = pos[t];
    const double qx = floor((double)(float)((double)p.x - ox) * invh);
    const double qy = floor((double)(float)((double)p.y - oy) * invh);
    const double qz = floor((double)(float)((double)p.z - oz) * invh);
    const double dn = (double)d;
    uint32_t k = (uint32_t)d * d * d;  // outside the grid: last
    if (qx >= 0 && qx < dn && qy >= 0 && qy < dn && qz >= 0 && qz < dn)
        k = ((uint32_t)qz * d + (uint32_t)qy) * d + (uint32_t)qx;
    key[t] = k;
    idx[t] = t;
}

__device__ __forceinline__ double hat(double r) {
    const double rr = fabs(r);
    return rr < 1.0 ? 1.0 - rr : 0.0;
}

__device__ __forceinline__ int clamp_cell(double q, int n) {
    if (!(q >= -3.0)) return -3;
    if (q > (double)(n + 2)) return n + 2;
    return (int)q;
}

// Evaluation at the sorted points: interpolation of the buffer (hat weights
// over the 5^3 cells around the point's cell, none when that cell is outside
// the grid) plus the particle correction.  GRAD: the gradient buffer [3][C]
// and the 1/r^3 kernel; else the scalar buffer [C] and the 1/r kernel.
template <bool GRAD>
__global__ void pot_eval_kernel(const uint32_t *__restrict__ eidx, uint32_t M, const float4 *__restrict__ eval4,
                                const double *__restrict__ far, const uint32_t *__restrict__ start,
                                const uint32_t *__restrict__ end, const float4 *__restrict__ srec,
                                const double *__restrict__ smass, int d, int K, double ox, double oy, double oz,
                                double invh, float bbmin_x, float bbmin_y, float bbmin_z, float bbmax_x,
                                float bbmax_y, float bbmax_z, double *__restrict__ ox_, double *__restrict__ oy_,
                                double *__restrict__ oz_, uint32_t ostride) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= M) return;
    const uint32_t q = eidx[s];
    const float4 e = eval4[q];
    const float px = (float)((double)e.x - ox), py = (float)((double)e.y - oy), pz = (float)((double)e.z - oz);
    const double qx = (double)px * invh, qy = (double)py * invh, qz = (double)pz * invh;
    const int i = clamp_cell(floor(qx), d), j = clamp_cell(floor(qy), d), k = clamp_cell(floor(qz), d);
    const size_t C = (size_t)d * d * d;
    double g[3] = {0, 0, 0};
    if (i >= 0 && i < d && j >= 0 && j < d && k >= 0 && k < d) {
        double hx[5], hy[5], hz[5];
#pragma unroll
        for (int a = 0; a < 5; a++) {
            hx[a] = hat((double)(float)((double)(i - 2 + a) + 0.5) - qx);
            hy[a] = hat((double)(float)((double)(j - 2 + a) + 0.5) - qy);
            hz[a] = hat((double)(float)((double)(k - 2 + a) + 0.5) - qz);
        }
#pragma unroll
        for (int cz = 0; cz < 5; cz++) {
            const int kk = k - 2 + cz;
            if (kk < 0 || kk >= d || hz[cz] == 0.0) continue;
#pragma unroll
            for (int cy = 0; cy < 5; cy++) {
                const int jj = j - 2 + cy;
                if (jj < 0 || jj >= d || hy[cy] == 0.0) continue;
#pragma unroll
                for (int cx = 0; cx < 5; cx++) {
                    const int ii = i - 2 + cx;
                    if (ii < 0 || ii >= d || hx[cx] == 0.0) continue;
                    const double w = hx[cx] * hy[cy] * hz[cz];
                    const size_t gi = ((size_t)kk * d + jj) * d + ii;
                    if (GRAD) {
                        g[0] += far[gi] * w;
                        g[1] += far[C + gi] * w;
                        g[2] += far[2 * C + gi] * w;
                    } else {
                        g[0] += far[gi] * w;
                    }
                }
            }
        }
    }
    if (K >= 0) {
        const double cr = ((double)K + 0.5) / invh;
        int lo[3], hi[3];
        const int cc[3] = {i, j, k};
        const double qq[3] = {qx, qy, qz};
#pragma unroll
        for (int a = 0; a < 3; a++) {
            if (GRAD) {
                lo[a] = cc[a] - K - 1;
                hi[a] = cc[a] + K + 1;
            } else if (qq[a] > (double)cc[a] + 0.5) {
                lo[a] = cc[a] - K;
                hi[a] = cc[a] + K + 1;
            } else {
                lo[a] = cc[a] - K - 1;
                hi[a] = cc[a] + K;
            }
            lo[a] = max(lo[a], 0);
            hi[a] = min(hi[a], d - 1);
        }
        const double a_core = GRAD ? 0.05 : 0.125;
        double f[3] = {0, 0, 0};
        for (int kk = lo[2]; kk <= hi[2]; kk++)
            for (int jj = lo[1]; jj <= hi[1]; jj++)
                for (int ii = lo[0]; ii <= hi[0]; ii++) {
                    const uint32_t r = ((uint32_t)kk * d + jj) * d + ii;
                    const uint32_t s0 = start[r];
                    if (s0 == kEmpty) continue;
                    const uint32_t s1 = end[r];
                    for (uint32_t p = s0; p < s1; p++) {
                        const float4 b = srec[p];
                        const float fx = b.x - px, fy = b.y - py, fz = b.z - pz;
                        if (!(fabs((double)fx) < cr && fabs((double)fy) < cr && fabs((double)fz) < cr)) continue;
                        const double dx = fx, dy = fy, dz = fz;
                        const double r1 = sqrt(dx * dx + dy * dy + dz * dz);
                        if (GRAD) {
                            double r3;
                            if (r1 > a_core) r3 = kFourPi * r1 * r1 * r1;
                            else r3 = (r1 < 1e-12) ? 1e+14 : kFourPi * a_core * a_core * a_core;
                            f[0] += kG * dx / r3 * smass[p];
                            f[1] += kG * dy / r3 * smass[p];
                            f[2] += kG * dz / r3 * smass[p];
                        } else {
                            double r2;
                            if (r1 > a_core) r2 = kFourPi * r1;
                            else r2 = (r1 < 1e-12) ? 1e+14 : kFourPi * a_core;
                            f[0] += kG / r2 * smass[p];
                        }
                    }
                }
        g[0] += f[0];
        g[1] += f[1];
        g[2] += f[2];
    }
    if (GRAD) {
        // Potentialparticle_outside_kernel (HFS/GPU_kernel.cu:1678-1716)
        const double x = e.x, y = e.y, z = e.z;
        if (x < bbmin_x || x > bbmax_x || y < bbmin_y || y > bbmax_y || z < bbmin_z || z > bbmax_z)
            g[0] = g[1] = g[2] = 0.0;
        ox_[(size_t)q * ostride] = g[0];
        oy_[(size_t)q * ostride] = g[1];
        oz_[(size_t)q * ostride] = g[2];
    } else {
        ox_[q] = g[0];
    }
}

// Potentialcompute_dphi_dn_kernel (HFS/GPU_kernel.cu:1719-1740).
__global__ void pot_dphidn_kernel(const double *__restrict__ nx, const double *__restrict__ ny,
                                  const double *__restrict__ nz, const double *__restrict__ gx,
                                  const double *__restrict__ gy, const double *__restrict__ gz,
                                  const double *__restrict__ mass, const double *__restrict__ area, uint32_t M,
                                  double *__restrict__ out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M) return;
    out[t] = -0.5 * mass[t] / area[t] + (nx[t] * gx[t] + ny[t] * gy[t] + nz[t] * gz[t]);
}

template <typename T>
cudaError_t grow(T **p, size_t count) {
    cudaFree(*p);
    *p = nullptr;
    return ::pppm::device_malloc((void **)p, sizeof(T) * (count ? count : 1));
}

// Capacities are raised only once every buffer they cover exists: a failed
// growth leaves capacity 0 (and no masses), so the next call allocates again
// instead of using a freed buffer.
cudaError_t ensure_hist(pppm_potential *P) {
    const size_t need = radix_hist_entries(std::max(P->capN, P->capM));
    if (need <= P->hist_cap) return cudaSuccess;
    P->hist_cap = 0;
    PPPM_CUDA_TRY(grow(&P->hist, need));
    P->hist_cap = need;
    return cudaSuccess;
}

cudaError_t grow_masses(pppm_potential *P, uint32_t N) {
    PPPM_CUDA_TRY(grow(&P->mpos, N));
    PPPM_CUDA_TRY(grow(&P->mass, N));
    for (int q = 0; q < 2; q++) {
        PPPM_CUDA_TRY(grow(&P->key[q], N));
        PPPM_CUDA_TRY(grow(&P->idx[q], N));
    }
    PPPM_CUDA_TRY(grow(&P->srec, N));
    PPPM_CUDA_TRY(grow(&P->smass, N));
    return cudaSuccess;
}

cudaError_t ensure_masses(pppm_potential *P, uint32_t N) {
    std::lock_guard<std::recursive_mutex> lk(device_lock());
    if (N > P->capN) {
        P->capN = 0;
        P->N = 0;        // the masses went with the old buffers
        P->built = 0;
        PPPM_CUDA_TRY(grow_masses(P, N));
        P->capN = N;
    }
    return ensure_hist(P);
}

cudaError_t ensure_eval(pppm_potential *P, uint32_t M) {
    std::lock_guard<std::recursive_mutex> lk(device_lock());
    if (M > P->capM) {
        P->capM = 0;
        for (int q = 0; q < 2; q++) {
            PPPM_CUDA_TRY(grow(&P->ekey[q], M));
            PPPM_CUDA_TRY(grow(&P->eidx[q], M));
        }
        P->capM = M;
    }
    return ensure_hist(P);
}

}  // namespace
}  // namespace pppm

static pppm_status pot_fail(const char *where, cudaError_t e) {
    pppm_set_error("%s: %s", where, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? PPPM_ERR_OOM : PPPM_ERR_CUDA;
}

extern "C" pppm_status pppm_potential_create(uint32_t n, int K, uint32_t cap_mass, uint32_t cap_eval, void *stream,
                                             pppm_potential **out) {
    using namespace pppm;
    if (!out || n < 4 || n > 512 || !mg_shape_ok(n) || K < -1 || K > kMaxK) {
        pppm_set_error("pppm_potential_create: invalid argument (n=%u, K=%d)", n, K);
        return PPPM_ERR_INVALID;
    }
    std::lock_guard<std::recursive_mutex> lk(device_lock());
    pppm_potential *P = new pppm_potential;
    P->stream = (cudaStream_t)stream;
    cudaGetDevice(&P->device);
    P->n = n;
    P->C = n * n * n;
    P->K = K;
    cudaError_t e = cudaSuccess;
    const size_t C = P->C;
    if (e == cudaSuccess) e = grow(&P->start, C);
    if (e == cudaSuccess) e = grow(&P->end, C);
    if (e == cudaSuccess) e = grow(&P->density, C);
    if (e == cudaSuccess) e = grow(&P->rhs, C);
    if (e == cudaSuccess) e = grow(&P->phi, C);
    if (e == cudaSuccess) e = grow(&P->far, 3 * C);
    if (e == cudaSuccess) e = grow(&P->mono, 4);
    if (e == cudaSuccess) e = grow(&P->mono_part, 5 * kRedBlocks);
    if (e == cudaSuccess) e = grow(&P->bbox, 6 * kRedBlocks);
    if (e == cudaSuccess) e = ::pppm::host_malloc((void **)&P->host_bbox, sizeof(float) * 6 * kRedBlocks);
    if (e == cudaSuccess) e = ensure_masses(P, std::max(cap_mass, 1u));
    if (e == cudaSuccess) e = ensure_eval(P, std::max(cap_eval, 1u));
    pppm_status st = PPPM_OK;
    if (e != cudaSuccess) st = pot_fail("pppm_potential_create", e);
    if (st == PPPM_OK) st = pppm_mg_create(n, stream, &P->mg);
    if (st != PPPM_OK) {
        pppm_potential_destroy(P);
        return st;
    }
    *out = P;
    return PPPM_OK;
}

extern "C" pppm_status pppm_potential_destroy(pppm_potential *P) {
    if (!P) return PPPM_OK;
    if (P->stream) cudaStreamSynchronize(P->stream);
    std::lock_guard<std::recursive_mutex> lk(pppm::device_lock());
    cudaFree(P->mpos); cudaFree(P->mass);
    for (int q = 0; q < 2; q++) {
        cudaFree(P->key[q]); cudaFree(P->idx[q]); cudaFree(P->ekey[q]); cudaFree(P->eidx[q]);
    }
    cudaFree(P->hist); cudaFree(P->start); cudaFree(P->end); cudaFree(P->srec); cudaFree(P->smass);
    cudaFree(P->density); cudaFree(P->rhs); cudaFree(P->phi); cudaFree(P->far); cudaFree(P->mono);
    cudaFree(P->mono_part); cudaFree(P->bbox);
    if (P->host_bbox) cudaFreeHost(P->host_bbox);
    if (P->mg) pppm_mg_destroy(P->mg);
    delete P;
    return PPPM_OK;
}

extern "C" pppm_status pppm_potential_set_masses(pppm_potential *P, uint32_t N, const float *pos4,
                                                 const double *mass) {
    if (!P || N == 0 || !pos4 || !mass) {
        pppm_set_error("pppm_potential_set_masses: NULL pointer or N == 0");
        return PPPM_ERR_INVALID;
    }
    cudaError_t e = pppm::ensure_masses(P, N);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(P->mpos, pos4, sizeof(float4) * N, cudaMemcpyDeviceToDevice, P->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(P->mass, mass, sizeof(double) * N, cudaMemcpyDeviceToDevice, P->stream);
    if (e != cudaSuccess) return pot_fail("pppm_potential_set_masses", e);
    P->N = N;
    P->built = 0;
    return PPPM_OK;
}

// computeFarFieldBuffer (scalar = 0) / computeFarFieldPotentialBuffer (scalar = 1).
extern "C" pppm_status pppm_potential_build(pppm_potential *P, int scalar) {
    using namespace pppm;
    if (!P || P->N == 0) {
        pppm_set_error("pppm_potential_build: call pppm_potential_set_masses first");
        return P ? PPPM_ERR_STATE : PPPM_ERR_INVALID;
    }
    cudaStream_t st = P->stream;
    const uint32_t N = P->N, n = P->n, C = P->C;
    note_launch();
    pot_bbox_kernel<<<kRedBlocks, 256, 0, st>>>(P->mpos, N, P->bbox);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(P->host_bbox, P->bbox, sizeof(float) * 6 * kRedBlocks, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return pot_fail("pppm_potential_build (bbox)", e);
    double mn[3], mx[3];
    for (int c = 0; c < 3; c++) {
        float lo = P->host_bbox[c * kRedBlocks], hi = P->host_bbox[(3 + c) * kRedBlocks];
        for (int q = 1; q < kRedBlocks; q++) {
            lo = std::min(lo, P->host_bbox[c * kRedBlocks + q]);
            hi = std::max(hi, P->host_bbox[(3 + c) * kRedBlocks + q]);
        }
        mn[c] = lo;
        mx[c] = hi;
    }
    const double L = 2.0 * std::max(std::max(mx[0] - mn[0], mx[1] - mn[1]), mx[2] - mn[2]);
    if (!(L > 0.0) || !std::isfinite(L)) {
        pppm_set_error("pppm_potential_build: masses span no volume");
        return PPPM_ERR_DOMAIN;
    }
    for (int c = 0; c < 3; c++) P->origin[c] = (mn[c] + 0.5 * (mx[c] - mn[c])) - 0.5 * L;
    P->L = L;
    P->h_f = (float)(L / (double)n);
    P->cell_h = (double)P->h_f;
    for (int c = 0; c < 3; c++) P->of[c] = (float)P->origin[c];
    uint32_t *skey = nullptr;
    e = launch_explicit_hash(st, P->mpos, N, P->h_f, P->of, n, P->key, P->idx, P->hist, &skey, &P->sidx, P->start,
                             P->end);
    const double invh = 1.0 / P->cell_h;
    if (e == cudaSuccess) {
        note_launch();
        pot_records_kernel<<<(N + 255) / 256, 256, 0, st>>>(P->mpos, P->mass, P->sidx, N, P->origin[0], P->origin[1],
                                                             P->origin[2], P->srec, P->smass);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        note_launch();
        pot_p2m_kernel<<<(C + 255) / 256, 256, 0, st>>>(P->start, P->end, P->srec, P->smass, (int)n, invh,
                                                        (double)(P->h_f * P->h_f), P->density, P->rhs);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        note_launch();
        pot_mono_partial_kernel<<<kRedBlocks, 256, 0, st>>>(P->mpos, P->mass, N, P->mono_part);
        note_launch();
        pot_mono_final_kernel<<<1, 32, 0, st>>>(P->mono_part, kRedBlocks, P->mono);
        note_launch();
        pot_dirichlet_kernel<<<(C + 255) / 256, 256, 0, st>>>(P->rhs, P->mono, (int)n, P->cell_h, P->origin[0],
                                                              P->origin[1], P->origin[2]);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(P->phi, 0, sizeof(double) * C, st);
    if (e != cudaSuccess) return pot_fail("pppm_potential_build", e);
    for (int it = 0; it < 3; it++) {
        const pppm_status s2 = pppm_mg_full_multigrid(P->mg, P->phi, P->rhs, PPPM_MG_REFERENCE, 1e-7, 1, nullptr);
        if (s2 != PPPM_OK) return s2;
    }
    const int K = P->K;
    if (!scalar) {
        note_launch();
        if (K >= 0) {
            const int W = 2 * K + 1;
            const size_t smem = sizeof(double) * 3 * (size_t)W * W * W;
            pot_far_gradient_kernel<<<(C + 127) / 128, 128, smem, st>>>(P->phi, P->density, (int)n, K, P->cell_h,
                                                                        P->far);
        } else {
            pot_gradient_only_kernel<<<(C + 255) / 256, 256, 0, st>>>(P->phi, (int)n, P->cell_h, P->far);
        }
    } else {
        note_launch();
        if (K >= 0)
            pot_far_scalar_kernel<<<(C + 255) / 256, 256, 0, st>>>(P->phi, P->density, (int)n, K, P->cell_h, P->far);
        else
            e = cudaMemcpyAsync(P->far, P->phi, sizeof(double) * C, cudaMemcpyDeviceToDevice, st);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return pot_fail("pppm_potential_build (far field)", e);
    P->built = scalar ? 2 : 1;
    return PPPM_OK;
}

static pppm_status pot_eval(pppm_potential *P, uint32_t M, const float *eval4, double *a, double *b, double *c,
                            bool grad, uint32_t ostride = 1) {
    using namespace pppm;
    if (!P || (M > 0 && (!eval4 || !a || (grad && (!b || !c))))) {
        pppm_set_error("pppm_potential_eval: invalid argument");
        return PPPM_ERR_INVALID;
    }
    if (P->built != (grad ? 1 : 2)) {
        pppm_set_error("pppm_potential_eval: build the %s buffer first", grad ? "gradient" : "scalar");
        return PPPM_ERR_STATE;
    }
    if (M == 0) return PPPM_OK;
    cudaStream_t st = P->stream;
    cudaError_t e = ensure_eval(P, M);
    const float4 *ev = reinterpret_cast<const float4 *>(eval4);
    const uint32_t n = P->n;
    const double invh = 1.0 / P->cell_h;
    uint32_t *skey = nullptr, *sidx = nullptr;
    if (e == cudaSuccess) {
        note_launch();
        pot_eval_keys_kernel<<<(M + 255) / 256, 256, 0, st>>>(ev, M, P->origin[0], P->origin[1], P->origin[2], invh,
                                                              (int)n, P->ekey[0], P->eidx[0]);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = radix_sort_pairs(st, M, key_bits(n) + 1, P->ekey, P->eidx, P->hist, &skey, &sidx);
    if (e == cudaSuccess) {
        const float bbmax[3] = {(float)(P->of[0] + P->L), (float)(P->of[1] + P->L), (float)(P->of[2] + P->L)};
        note_launch();
        if (grad)
            pot_eval_kernel<true><<<(M + 127) / 128, 128, 0, st>>>(
                sidx, M, ev, P->far, P->start, P->end, P->srec, P->smass, (int)n, P->K, P->origin[0], P->origin[1],
                P->origin[2], invh, P->of[0], P->of[1], P->of[2], bbmax[0], bbmax[1], bbmax[2], a, b, c, ostride);
        else
            pot_eval_kernel<false><<<(M + 127) / 128, 128, 0, st>>>(
                sidx, M, ev, P->far, P->start, P->end, P->srec, P->smass, (int)n, P->K, P->origin[0], P->origin[1],
                P->origin[2], invh, P->of[0], P->of[1], P->of[2], bbmax[0], bbmax[1], bbmax[2], a, nullptr, nullptr,
                1);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return pot_fail("pppm_potential_eval", e);
    return PPPM_OK;
}

extern "C" pppm_status pppm_potential_eval_gradient(pppm_potential *P, uint32_t M, const float *eval4, double *gx,
                                                    double *gy, double *gz) {
    return pot_eval(P, M, eval4, gx, gy, gz, true);
}

extern "C" pppm_status pppm_potential_eval_gradient3(pppm_potential *P, uint32_t M, const float *eval4,
                                                     double *grad3) {
    return pot_eval(P, M, eval4, grad3, grad3 ? grad3 + 1 : nullptr, grad3 ? grad3 + 2 : nullptr, true, 3);
}

extern "C" pppm_status pppm_potential_eval_scalar(pppm_potential *P, uint32_t M, const float *eval4, double *phi) {
    return pot_eval(P, M, eval4, phi, nullptr, nullptr, false);
}

extern "C" pppm_status pppm_potential_dphidn(pppm_potential *P, uint32_t M, const double *nx, const double *ny,
                                             const double *nz, const double *gx, const double *gy, const double *gz,
                                             const double *mass, const double *area, double *out) {
    if (!P || (M > 0 && (!nx || !ny || !nz || !gx || !gy || !gz || !mass || !area || !out))) {
        pppm_set_error("pppm_potential_dphidn: invalid argument");
        return PPPM_ERR_INVALID;
    }
    if (M == 0) return PPPM_OK;
    pppm::note_launch();
    pppm::pot_dphidn_kernel<<<(M + 255) / 256, 256, 0, P->stream>>>(nx, ny, nz, gx, gy, gz, mass, area, M, out);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PPPM_OK : pot_fail("pppm_potential_dphidn", e);
}

extern "C" pppm_status pppm_potential_grids(pppm_potential *P, double origin_length[4], const double **density,
                                            const double **rhs, const double **phi, const double **far,
                                            double monopole_host[4]) {
    if (!P || P->built == 0) {
        pppm_set_error("pppm_potential_grids: nothing built");
        return PPPM_ERR_STATE;
    }
    if (origin_length) {
        for (int c = 0; c < 3; c++) origin_length[c] = P->origin[c];
        origin_length[3] = P->L;
    }
    if (density) *density = P->density;
    if (rhs) *rhs = P->rhs;
    if (phi) *phi = P->phi;
    if (far) *far = P->far;
    if (monopole_host) {
        const cudaError_t e = cudaMemcpyAsync(monopole_host, P->mono, sizeof(double) * 4, cudaMemcpyDeviceToHost, P->stream);
        if (e == cudaSuccess) cudaStreamSynchronize(P->stream);
        if (e != cudaSuccess) return pot_fail("pppm_potential_grids", e);
    }
    return PPPM_OK;
}
