// Curl of the vector potential fused with the far-field correction
// (HFS/GPU_kernel.cu:1750-1805 getCurl, 2487-2564 Step1, 1976-2001 diagonal
// potential, 2566-2630 diagonal subtraction, host table 2646-2692):
//
//   U(c)   = curl(psi)(c), central differences / (2h), clamped sampling
//   far(c) = U(c) - sum_{c' != c, |c'-c|_inf <= K, c' in grid} D[c'-c] x omega(c') h^3
//                 - curl(0.250580605913965 * omega * h^2)(c)     (clamped)
//
// D[off] is the central-difference gradient (step h) of 1/(4 pi |X - X'|)
// between the cell centre and the cell at offset `off`, a coincident pair
// reading 1/1e24 (HFS/GPU_kernel.cu:11-17).  Each block evaluates the
// (2K+1)^3 table in FP64 from the device cell size into shared memory, so the
// reference's per-call host build, cudaMalloc and copy disappear, as does the
// grid-velocity round trip through the host (HFS/BiotSavartSolverImp.cpp:
// 779-781, 811-813).  The curl reads the FP64 potential; the omega stencil
// runs in FP32.
#include "pppm_internal.cuh"

namespace pppm {

namespace {

constexpr int kFFThreads = 256;
constexpr int kMaxTable = (2 * kMaxK + 1) * (2 * kMaxK + 1) * (2 * kMaxK + 1);

__device__ double inv4pi_r(double ax, double ay, double az, double bx, double by, double bz) {
    const double r_sqr = (ax - bx) * (ax - bx) + (ay - by) * (ay - by) + (az - bz) * (az - bz);
    const double r = (r_sqr > 1e-12) ? kFourPi * sqrt(r_sqr) : 1e+24;
    return 1.0 / r;
}

__global__ void __launch_bounds__(kFFThreads)
farfield_kernel(const double *__restrict__ psi, const float *__restrict__ vort, float *__restrict__ far,
                const DevParams *__restrict__ P, int n, int K) {
    __shared__ float3 table[kMaxTable];
    const int W = 2 * K + 1;
    const int T = W * W * W;
    const double h = P->cell_h;
    for (int q = threadIdx.x; q < T; q += blockDim.x) {
        const int ii = q % W - K, jj = (q / W) % W - K, kk = q / (W * W) - K;
        float3 v = make_float3(0.f, 0.f, 0.f);
        if (ii || jj || kk) {
            const double Xpx = ((double)ii + 0.5) * h, Xpy = ((double)jj + 0.5) * h, Xpz = ((double)kk + 0.5) * h;
            const double X = 0.5 * h;
            v.x = (float)(0.5 * (inv4pi_r(X + h, X, X, Xpx, Xpy, Xpz) - inv4pi_r(X - h, X, X, Xpx, Xpy, Xpz)) / h);
            v.y = (float)(0.5 * (inv4pi_r(X, X + h, X, Xpx, Xpy, Xpz) - inv4pi_r(X, X - h, X, Xpx, Xpy, Xpz)) / h);
            v.z = (float)(0.5 * (inv4pi_r(X, X, X + h, Xpx, Xpy, Xpz) - inv4pi_r(X, X, X - h, Xpx, Xpy, Xpz)) / h);
        }
        table[q] = v;
    }
    __syncthreads();
    const uint32_t C = (uint32_t)n * n * n;
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    const int i = (int)(c % n), j = (int)((c / n) % n), k = (int)(c / ((uint32_t)n * n));
    const int im = max(i - 1, 0), ip = min(i + 1, n - 1);
    const int jm = max(j - 1, 0), jp = min(j + 1, n - 1);
    const int km = max(k - 1, 0), kp = min(k + 1, n - 1);
    auto at = [n](int x, int y, int z) { return ((size_t)z * n + y) * n + x; };
    const double *Fx = psi, *Fy = psi + C, *Fz = psi + 2 * (size_t)C;
    const float *Wx = vort, *Wy = vort + C, *Wz = vort + 2 * (size_t)C;

    // curl(psi), HFS/GPU_kernel.cu:1770-1793
    const double invh = P->invh;
    const double ux = 0.5 * invh * (Fz[at(i, jp, k)] - Fz[at(i, jm, k)] + Fy[at(i, j, km)] - Fy[at(i, j, kp)]);
    const double uy = 0.5 * invh * (Fx[at(i, j, kp)] - Fx[at(i, j, km)] + Fz[at(im, j, k)] - Fz[at(ip, j, k)]);
    const double uz = 0.5 * invh * (Fy[at(ip, j, k)] - Fy[at(im, j, k)] + Fx[at(i, jm, k)] - Fx[at(i, jp, k)]);

    // mesh's own near-field contribution, HFS/GPU_kernel.cu:2533-2556
    float mx = 0.f, my = 0.f, mz = 0.f;
    for (int dk = -K; dk <= K; dk++) {
        const int kk = k + dk;
        if (kk < 0 || kk >= n) continue;
        for (int dj = -K; dj <= K; dj++) {
            const int jj = j + dj;
            if (jj < 0 || jj >= n) continue;
            for (int di = -K; di <= K; di++) {
                const int ii = i + di;
                if (ii < 0 || ii >= n || (!di && !dj && !dk)) continue;
                const size_t s = at(ii, jj, kk);
                const float3 D = table[((dk + K) * W + (dj + K)) * W + (di + K)];
                const float ox = Wx[s], oy = Wy[s], oz = Wz[s];
                mx += D.y * oz - D.z * oy;
                my += D.z * ox - D.x * oz;
                mz += D.x * oy - D.y * ox;
            }
        }
    }
    const float vh3 = P->vh3_f;
    mx *= vh3;
    my *= vh3;
    mz *= vh3;

    // curl of the diagonal self-potential 0.250580605913965 * omega * h^2
    const float kd = P->kdiag_f;
    const float dx = kd * (Wz[at(i, jp, k)] - Wz[at(i, jm, k)] + Wy[at(i, j, km)] - Wy[at(i, j, kp)]);
    const float dy = kd * (Wx[at(i, j, kp)] - Wx[at(i, j, km)] + Wz[at(im, j, k)] - Wz[at(ip, j, k)]);
    const float dz = kd * (Wy[at(ip, j, k)] - Wy[at(im, j, k)] + Wx[at(i, jm, k)] - Wx[at(i, jp, k)]);

    far[c] = (float)(ux - (double)mx) - dx;
    far[C + c] = (float)(uy - (double)my) - dy;
    far[2 * (size_t)C + c] = (float)(uz - (double)mz) - dz;
}

__global__ void __launch_bounds__(kFFThreads)
curl_only_kernel(const double *__restrict__ psi, float *__restrict__ far, const DevParams *__restrict__ P, int n) {
    const uint32_t C = (uint32_t)n * n * n;
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    const int i = (int)(c % n), j = (int)((c / n) % n), k = (int)(c / ((uint32_t)n * n));
    const int im = max(i - 1, 0), ip = min(i + 1, n - 1);
    const int jm = max(j - 1, 0), jp = min(j + 1, n - 1);
    const int km = max(k - 1, 0), kp = min(k + 1, n - 1);
    auto at = [n](int x, int y, int z) { return ((size_t)z * n + y) * n + x; };
    const double *Fx = psi, *Fy = psi + C, *Fz = psi + 2 * (size_t)C;
    const double invh = P->invh;
    far[c] = (float)(0.5 * invh * (Fz[at(i, jp, k)] - Fz[at(i, jm, k)] + Fy[at(i, j, km)] - Fy[at(i, j, kp)]));
    far[C + c] = (float)(0.5 * invh * (Fx[at(i, j, kp)] - Fx[at(i, j, km)] + Fz[at(im, j, k)] - Fz[at(ip, j, k)]));
    far[2 * (size_t)C + c] =
        (float)(0.5 * invh * (Fy[at(ip, j, k)] - Fy[at(im, j, k)] + Fx[at(i, jm, k)] - Fx[at(i, jp, k)]));
}

}  // namespace

cudaError_t launch_farfield(pppm_scene *s) {
    const unsigned blocks = (s->C + kFFThreads - 1) / kFFThreads;
    ::pppm::note_launch();
    if (s->prm.K >= 0)
        farfield_kernel<<<blocks, kFFThreads, 0, s->stream>>>(s->psi, s->vort, s->far, s->dparams, (int)s->n,
                                                              s->prm.K);
    else  // BiotSavartComputeFarField is a no-op for K < 0: far = curl(psi)
        curl_only_kernel<<<blocks, kFFThreads, 0, s->stream>>>(s->psi, s->far, s->dparams, (int)s->n);
    return cudaGetLastError();
}

}  // namespace pppm
