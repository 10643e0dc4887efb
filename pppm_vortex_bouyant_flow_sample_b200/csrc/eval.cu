// Velocity evaluation: far-field interpolation + near-field smoothed
// Biot-Savart correction + scatter back to the caller's order, one fused
// kernel (HFS/GPU_kernel.cu:2886-2976 BiotSavartInterpolate_far_field_kernel2,
// :2262-2485 BiotSavartPPCorrScaleMN_kernel, PH/particle_hash_kernel.cu:
// 160-188 removeReorder).
//
// Evaluation points are visited in hash order (same grid as the vortices), so
// the threads of a warp walk the same neighbour cells and read the same
// vortex records.  Per point:
//   * relative position rounded to float from the FP64 difference with the
//     domain origin, NGP cell floor(rel * invh) in FP64 (reference rounding);
//   * far field: hat weights 1 - |cell centre - rel/h| on the 8 surrounding
//     cell centres, cells outside the grid skipped, no write when the point's
//     own cell is outside the grid;
//   * near field: hash cells [i-K-1, i+K+1]^3; a vortex counts when its float
//     coordinate differences are all below (K+0.5)h (the float test is exact:
//     |d| <= largest float below the double bound); contribution
//     (alpha x d) * phi((r/a)^3) / (4 pi a^3) with phi(t) = (1 - e^-t)/t,
//     which equals (1 - e^-(r/a)^3) / (4 pi r^3); pairs with r = 0, or (for
//     segments) a zero distance to the other end, are skipped.
// Pair arithmetic is FP32; phi uses its Taylor series below t = 0.5 (no
// cancellation) and 1 - exp(-t) above.
#include "pppm_internal.cuh"

namespace pppm {

namespace {

constexpr int kEvalThreads = 128;

__device__ __forceinline__ float phi_smooth(float t) {
    if (t < 0.5f) {
        float p = 1.0f / 362880.0f;
        p = fmaf(p, t, -1.0f / 40320.0f);
        p = fmaf(p, t, 1.0f / 5040.0f);
        p = fmaf(p, t, -1.0f / 720.0f);
        p = fmaf(p, t, 1.0f / 120.0f);
        p = fmaf(p, t, -1.0f / 24.0f);
        p = fmaf(p, t, 1.0f / 6.0f);
        p = fmaf(p, t, -0.5f);
        return fmaf(p, t, 1.0f);
    }
    return (1.0f - __expf(-t)) / t;
}

__device__ __forceinline__ float3 rel_pos(float4 p, const DevParams *__restrict__ P) {
    return make_float3((float)((double)p.x - P->origin[0]), (float)((double)p.y - P->origin[1]),
                       (float)((double)p.z - P->origin[2]));
}

__global__ void __launch_bounds__(kEvalThreads)
eval_kernel(const uint32_t *__restrict__ eidx, uint32_t M, const float4 *__restrict__ eval_a,
            const float4 *__restrict__ eval_b, int is_segment, const float *__restrict__ far,
            const uint32_t *__restrict__ start, const uint32_t *__restrict__ end, const float4 *__restrict__ vrec,
            const float4 *__restrict__ valf, const DevParams *__restrict__ P, int n, int K,
            double *__restrict__ u, double *__restrict__ v, double *__restrict__ w, float *__restrict__ uf,
            unsigned long long *__restrict__ pair_count) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long pairs = 0;
    if (s < M) {
        const uint32_t q = eidx[s];
        const float3 ra = rel_pos(eval_a[q], P);
        float3 rb = make_float3(0.f, 0.f, 0.f);
        if (is_segment == 1) rb = rel_pos(eval_b[q], P);
        const double invh = P->invh;
        const double qx = (double)ra.x * invh, qy = (double)ra.y * invh, qz = (double)ra.z * invh;
        const int i = (int)floor(qx), j = (int)floor(qy), k = (int)floor(qz);
        const uint32_t C = (uint32_t)n * n * n;
        float ux = 0.f, uy = 0.f, uz = 0.f;
        if (i >= 0 && i < n && j >= 0 && j < n && k >= 0 && k < n) {
            const double tx = qx - 0.5, ty = qy - 0.5, tz = qz - 0.5;
            const double fx0 = floor(tx), fy0 = floor(ty), fz0 = floor(tz);
            const int i0 = (int)fx0, j0 = (int)fy0, k0 = (int)fz0;
            const float fx = (float)(tx - fx0), fy = (float)(ty - fy0), fz = (float)(tz - fz0);
            const float wx[2] = {1.f - fx, fx}, wy[2] = {1.f - fy, fy}, wz[2] = {1.f - fz, fz};
#pragma unroll
            for (int c = 0; c < 8; c++) {
                const int ii = i0 + (c & 1), jj = j0 + ((c >> 1) & 1), kk = k0 + (c >> 2);
                if (ii < 0 || ii >= n || jj < 0 || jj >= n || kk < 0 || kk >= n) continue;
                const float wgt = wx[c & 1] * wy[(c >> 1) & 1] * wz[c >> 2];
                const size_t g = ((size_t)kk * n + jj) * n + ii;
                ux = fmaf(far[g], wgt, ux);
                uy = fmaf(far[C + g], wgt, uy);
                uz = fmaf(far[2 * (size_t)C + g], wgt, uz);
            }
        }
        if (K >= 0) {
            const float cr = P->cr_f;
            const float inv_a3 = P->inv_a3_f, inv4pia3 = P->inv4pia3_f;
            float px = 0.f, py = 0.f, pz = 0.f;
            const int k_lo = max(k - K - 1, 0), k_hi = min(k + K + 1, n - 1);
            const int j_lo = max(j - K - 1, 0), j_hi = min(j + K + 1, n - 1);
            const int i_lo = max(i - K - 1, 0), i_hi = min(i + K + 1, n - 1);
            for (int kk = k_lo; kk <= k_hi; kk++)
                for (int jj = j_lo; jj <= j_hi; jj++)
                    for (int ii = i_lo; ii <= i_hi; ii++) {
                        const uint32_t cell = ((uint32_t)kk * n + (uint32_t)jj) * n + (uint32_t)ii;
                        const uint32_t ps = start[cell];
                        if (ps == kEmpty) continue;
                        const uint32_t pe = end[cell];
                        for (uint32_t p = ps; p < pe; p++) {
                            const float4 r = vrec[p];
                            const float dx = ra.x - r.x, dy = ra.y - r.y, dz = ra.z - r.z;
                            if (!(fabsf(dx) <= cr && fabsf(dy) <= cr && fabsf(dz) <= cr)) continue;
                            pairs++;
                            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                            bool skip = r2 < 1e-24f;
                            if (is_segment == 1) {
                                const float ex = rb.x - r.x, ey = rb.y - r.y, ez = rb.z - r.z;
                                skip |= fmaf(ex, ex, fmaf(ey, ey, ez * ez)) < 1e-24f;
                            }
                            if (skip) continue;
                            const float rr = sqrtf(r2);
                            const float coeff = phi_smooth(r2 * rr * inv_a3) * inv4pia3;
                            const float4 al = valf[p];
                            px = fmaf(al.y * dz - al.z * dy, coeff, px);
                            py = fmaf(al.z * dx - al.x * dz, coeff, py);
                            pz = fmaf(al.x * dy - al.y * dx, coeff, pz);
                        }
                    }
            ux += px;
            uy += py;
            uz += pz;
        }
        if (u) {
            u[q] = (double)ux;
            v[q] = (double)uy;
            w[q] = (double)uz;
        }
        if (uf) {
            uf[3 * (size_t)q] = ux;
            uf[3 * (size_t)q + 1] = uy;
            uf[3 * (size_t)q + 2] = uz;
        }
    }
    if (pair_count) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
        if ((threadIdx.x & 31) == 0 && pairs) atomicAdd(pair_count, pairs);
    }
}

}  // namespace

cudaError_t launch_eval(pppm_scene *s, const float4 *eval_a, const float4 *eval_b, int is_segment, uint32_t M,
                        double *u, double *v, double *w, float *uf, int count_pairs) {
    uint32_t *skey = nullptr, *sidx = nullptr;
    PPPM_CUDA_TRY(launch_hash_sort(s, eval_a, M, s->ekey, s->eidx, &skey, &sidx));
    s->esorted_idx = sidx;
    if (count_pairs) PPPM_CUDA_TRY(cudaMemsetAsync(s->pair_count, 0, sizeof(unsigned long long), s->stream));
    eval_kernel<<<(M + kEvalThreads - 1) / kEvalThreads, kEvalThreads, 0, s->stream>>>(
        sidx, M, eval_a, eval_b, is_segment, s->far, s->cell_start, s->cell_end, s->vrec, s->valf, s->dparams,
        (int)s->n, s->prm.K, u, v, w, uf, count_pairs ? s->pair_count : nullptr);
    return cudaGetLastError();
}

}  // namespace pppm
