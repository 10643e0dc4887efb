// Spatial hash of the PPPM path on sm_100a.
//
//  * bounding box + domain parameters on the device
//    (HFS/BiotSavartSolverImp.cpp:379-409, PH/SpaceHashClass.h:46-54);
//  * cell keys bit-exact with PH/particle_hash_kernel.cu:32-70;
//  * a stable LSD radix sort of (key, index) replacing thrust::sort_by_key
//    (PH/SpaceHashFunctional.cu:97-102): 8-bit digits, per pass an upsweep
//    histogram, one scan, and a downsweep whose ranks are stable (warp
//    __match_any_sync, warps and item rounds in index order);
//  * cell start/end tables (PH/particle_hash_kernel.cu:74-126) fused with the
//    gather of positions and strengths into sorted order
//    (PH/particle_hash_kernel.cu:128-158), which also rounds positions to the
//    float relative coordinates the reference kernels use and computes each
//    vortex's nearest-grid-point cell in FP64.
#include <cfloat>
#include <cmath>

#include "pppm_internal.cuh"

namespace pppm {

namespace {

constexpr int kBBoxThreads = 256;
constexpr int kRsThreads = 256;
constexpr int kRsItems = 16;
constexpr int kRsTile = kRsThreads * kRsItems;
static_assert(kRsTile == (int)kRsTileHost, "tile size mismatch");
constexpr int kRsWarps = kRsThreads / 32;

__global__ void bbox_partial_kernel(const float4 *__restrict__ pos, uint32_t N,
                                    float *__restrict__ partial, int nblocks) {
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < N; t += gridDim.x * blockDim.x) {
        float4 p = pos[t];
        mn[0] = fminf(mn[0], p.x); mx[0] = fmaxf(mx[0], p.x);
        mn[1] = fminf(mn[1], p.y); mx[1] = fmaxf(mx[1], p.y);
        mn[2] = fminf(mn[2], p.z); mx[2] = fmaxf(mx[2], p.z);
    }
    __shared__ float sh[6][kBBoxThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int a = 0; a < 3; a++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
            mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
        }
    }
    if (lane == 0) {
        for (int a = 0; a < 3; a++) { sh[a][warp] = mn[a]; sh[3 + a][warp] = mx[a]; }
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int q = threadIdx.x;
        float v = sh[q][0];
        for (int w = 1; w < kBBoxThreads / 32; w++) v = (q < 3) ? fminf(v, sh[q][w]) : fmaxf(v, sh[q][w]);
        partial[q * nblocks + blockIdx.x] = v;
    }
}

// Largest float strictly below the double c (for x < c tests on floats).
__device__ float float_below(double c) {
    float f = (float)c;
    if ((double)f >= c) f = nextafterf(f, -FLT_MAX);
    return f;
}

__global__ void params_kernel(const float *__restrict__ partial, int nblocks, pppm_params prm,
                              DevParams *__restrict__ P) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double origin[3], L;
    if (prm.domain_mode == PPPM_DOMAIN_FIXED) {
        origin[0] = prm.fixed_origin[0];
        origin[1] = prm.fixed_origin[1];
        origin[2] = prm.fixed_origin[2];
        L = prm.fixed_length;
    }
    double mn[3], mx[3];
    for (int a = 0; a < 3; a++) {
        float lo = partial[a * nblocks], hi = partial[(3 + a) * nblocks];
        for (int b = 1; b < nblocks; b++) {
            lo = fminf(lo, partial[a * nblocks + b]);
            hi = fmaxf(hi, partial[(3 + a) * nblocks + b]);
        }
        mn[a] = lo;
        mx[a] = hi;
    }
    if (prm.domain_mode != PPPM_DOMAIN_FIXED) {
        // HFS/BiotSavartSolverImp.cpp:399-406
        L = 3 * fmax(fmax(mx[0] - mn[0], mx[1] - mn[1]), mx[2] - mn[2]);
        for (int a = 0; a < 3; a++) {
            double c = mn[a] + 0.5 * (mx[a] - mn[a]);
            origin[a] = c - 0.5 * L;
        }
    }
    const uint32_t n = prm.n;
    P->status = (L > 0.0 && isfinite(L)) ? 0 : PPPM_ERR_DOMAIN;
    for (int a = 0; a < 3; a++) {
        P->origin[a] = origin[a];
        P->origin_f[a] = (float)origin[a];
    }
    P->length = L;
    const float h_f = (float)(L / (double)n);  // setSpatialHashGrid(float h)
    P->h_f = h_f;
    const double h = (double)h_f;              // getCellSize().x
    P->cell_h = h;
    const double invh = 1.0 / h;
    P->invh = invh;
    P->h2f = __fmul_rn(h_f, h_f);
    P->invh3_f = (float)(invh * invh * invh);
    P->cr_f = float_below(((double)prm.K + 0.5) / invh);
    P->vh3_f = (float)(h * h * h);
    P->kdiag_f = (float)(0.5 * invh * kDiagPsi * (h * h));
    const double a = (prm.a_cells > 0.0) ? prm.a_cells * h : prm.a;
    P->a = a;
    P->inv_a3_f = (float)(1.0 / (a * a * a));
    P->inv4pia3_f = (float)(1.0 / (kFourPi * a * a * a));
    {
        // farthest pair the box admits: (K+0.5) h along each axis
        const double rmax = ((double)prm.K + 0.5) * h * 1.7320508075688772 * 1.001;
        const double tmax = (rmax / a) * (rmax / a) * (rmax / a);
        P->need_exp = !(tmax < 0.25);
        P->need_exp2 = !(tmax < 2.0);
    }
    // The FP32 hash coordinate fl(fl(p - o_f) / h_f) and the FP64 NGP coordinate
    // fl32(p - o) / h differ by at most a few float roundings of |p| + |o| over h;
    // 2^-20 covers them with a factor > 4 to spare.  The box test adds the
    // rounding of one float subtraction of relative coordinates.
    double pmax = 0.0, omax = 0.0;
    for (int a = 0; a < 3; a++) {
        pmax = fmax(pmax, fmax(fabs(mn[a]), fabs(mx[a])));
        omax = fmax(omax, fabs(origin[a]));
    }
    P->prune_cells = (h > 0.0) ? ldexp(pmax + omax + L, -20) / h + ldexp((double)prm.K + 0.5, -20) + 1e-6 : 1.0;
    P->n = n;
    P->K = prm.K;
}

__device__ __forceinline__ uint32_t umul24u(uint32_t a, uint32_t b) { return __umul24(a, b); }

// PH/particle_hash_kernel.cu:32-70: floor((p - o)/h) in FP32 (IEEE division),
// int % uint wrap, __umul24 address.
__device__ __forceinline__ uint32_t cell_key(float4 p, const float *of, float h, uint32_t n) {
    int gx = (int)floorf(__fdiv_rn(__fsub_rn(p.x, of[0]), h));
    int gy = (int)floorf(__fdiv_rn(__fsub_rn(p.y, of[1]), h));
    int gz = (int)floorf(__fdiv_rn(__fsub_rn(p.z, of[2]), h));
    uint32_t ux = (uint32_t)gx % n, uy = (uint32_t)gy % n, uz = (uint32_t)gz % n;
    return umul24u(umul24u(uz, n), n) + umul24u(uy, n) + ux;
}

// Reference cell keys (the order getSortPos / the ParticleManager tables use).
__global__ void keys_kernel(const float4 *__restrict__ pos, uint32_t N, const DevParams *__restrict__ P,
                            uint32_t *__restrict__ key, uint32_t *__restrict__ idx) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    const float of[3] = {P->origin_f[0], P->origin_f[1], P->origin_f[2]};
    key[t] = cell_key(pos[t], of, P->h_f, P->n);
    idx[t] = t;
}

// Near-field order: the reference cell key, then the octant of the vortex
// inside that cell (FP64 coordinate relative to the FP32 hash cell, so a
// vortex that rounding put in a neighbouring hash cell still lands in the
// sub-cell nearest to it).  Key = cell * 8 + octant.
__global__ void keys_octant_kernel(const float4 *__restrict__ pos, uint32_t N, const DevParams *__restrict__ P,
                                   uint32_t *__restrict__ key, uint32_t *__restrict__ idx) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    const float4 p = pos[t];
    const float h = P->h_f;
    const int gx = (int)floorf(__fdiv_rn(__fsub_rn(p.x, P->origin_f[0]), h));
    const int gy = (int)floorf(__fdiv_rn(__fsub_rn(p.y, P->origin_f[1]), h));
    const int gz = (int)floorf(__fdiv_rn(__fsub_rn(p.z, P->origin_f[2]), h));
    const uint32_t n = P->n;
    const uint32_t ux = (uint32_t)gx % n, uy = (uint32_t)gy % n, uz = (uint32_t)gz % n;
    const uint32_t ck = umul24u(umul24u(uz, n), n) + umul24u(uy, n) + ux;
    const double invh = P->invh;
    const double qx = (double)(float)((double)p.x - P->origin[0]) * invh;
    const double qy = (double)(float)((double)p.y - P->origin[1]) * invh;
    const double qz = (double)(float)((double)p.z - P->origin[2]) * invh;
    const uint32_t oct = (qx - (double)gx >= 0.5 ? 1u : 0u) | (qy - (double)gy >= 0.5 ? 2u : 0u) |
                         (qz - (double)gz >= 0.5 ? 4u : 0u);
    key[t] = (ck << 3) | oct;
    idx[t] = t;
}

__global__ void keys_explicit_kernel(const float4 *__restrict__ pos, uint32_t N, float h,
                                     float ox, float oy, float oz, uint32_t n,
                                     uint32_t *__restrict__ key, uint32_t *__restrict__ idx) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    const float of[3] = {ox, oy, oz};
    key[t] = cell_key(pos[t], of, h, n);
    idx[t] = t;
}

// Per-tile digit histogram, written digit-major: hist[d * nb + b].
__global__ void __launch_bounds__(kRsThreads)
radix_upsweep_kernel(const uint32_t *__restrict__ keys, uint32_t N, int shift, uint32_t *__restrict__ hist) {
    __shared__ uint32_t cnt[256];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t base = blockIdx.x * kRsTile;
#pragma unroll 4
    for (int j = 0; j < kRsItems; j++) {
        uint32_t i = base + j * kRsThreads + threadIdx.x;
        if (i < N) atomicAdd(&cnt[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[threadIdx.x * gridDim.x + blockIdx.x] = cnt[threadIdx.x];
}

// Block-wide exclusive scan of one value per thread (blockDim.x == 256).
__device__ __forceinline__ uint32_t block_excl_scan256(uint32_t v, uint32_t *warp_tot, uint32_t &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    uint32_t before = 0, all = 0;
#pragma unroll
    for (int w = 0; w < kRsWarps; w++) {
        const uint32_t t = warp_tot[w];
        if (w < warp) before += t;
        all += t;
    }
    __syncthreads();
    total = all;
    return x - v + before;
}

// Exclusive scan of each digit's row hist[d][0..nb) (one block per digit);
// the row total goes to totals[d].
__global__ void __launch_bounds__(kRsThreads)
radix_rowscan_kernel(uint32_t *__restrict__ hist, uint32_t nb, uint32_t *__restrict__ totals) {
    __shared__ uint32_t warp_tot[kRsWarps];
    uint32_t *row = hist + (size_t)blockIdx.x * nb;
    uint32_t run = 0;
    for (uint32_t base = 0; base < nb; base += kRsThreads) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = (i < nb) ? row[i] : 0u;
        uint32_t tot;
        const uint32_t ex = block_excl_scan256(v, warp_tot, tot);
        if (i < nb) row[i] = run + ex;
        run += tot;
    }
    if (threadIdx.x == 0) totals[blockIdx.x] = run;
}

// Stable scatter of one 8-bit digit.  Item order inside a tile is
// (round j, warp, lane) = index order, so ranks preserve input order.
__global__ void __launch_bounds__(kRsThreads)
radix_downsweep_kernel(const uint32_t *__restrict__ kin, const uint32_t *__restrict__ vin,
                       uint32_t *__restrict__ kout, uint32_t *__restrict__ vout, uint32_t N, int shift,
                       const uint32_t *__restrict__ hist, const uint32_t *__restrict__ totals) {
    __shared__ uint32_t goff[256];
    __shared__ uint32_t running[256];
    __shared__ uint32_t wcnt[kRsWarps][256];
    __shared__ uint32_t warp_tot[kRsWarps];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint32_t all;
    const uint32_t digit_base = block_excl_scan256(totals[tid], warp_tot, all);
    goff[tid] = digit_base + hist[tid * gridDim.x + blockIdx.x];
    running[tid] = 0;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint32_t base = blockIdx.x * kRsTile;
    for (int j = 0; j < kRsItems; j++) {
        for (int q = 0; q < kRsWarps; q++) wcnt[q][tid] = 0;
        __syncthreads();
        const uint32_t i = base + j * kRsThreads + tid;
        const bool valid = i < N;
        uint32_t k = 0, d = 256u + lane;  // invalid lanes form singleton groups
        if (valid) {
            k = kin[i];
            d = (k >> shift) & 255u;
        }
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t rank = __popc(peers & lt_mask);
        if (valid && rank == 0) wcnt[warp][d] = __popc(peers);
        __syncthreads();
        {
            uint32_t acc = running[tid];
#pragma unroll
            for (int q = 0; q < kRsWarps; q++) {
                uint32_t c = wcnt[q][tid];
                wcnt[q][tid] = acc;
                acc += c;
            }
            running[tid] = acc;
        }
        __syncthreads();
        if (valid) {
            const uint32_t p = goff[d] + wcnt[warp][d] + rank;
            kout[p] = k;
            vout[p] = vin[i];
        }
        __syncthreads();
    }
}

__device__ __forceinline__ uint32_t ngp_cell(float rx, float ry, float rz, double invh, uint32_t n) {
    // floor(pos * invh) with pos the float relative coordinate promoted to
    // double, as in HFS/GPU_kernel.cu:2300-2302 and the P2M weight test.
    const double qx = floor((double)rx * invh), qy = floor((double)ry * invh), qz = floor((double)rz * invh);
    const double dn = (double)n;
    if (!(qx >= 0.0 && qx < dn && qy >= 0.0 && qy < dn && qz >= 0.0 && qz < dn)) return kEmpty;
    return ((uint32_t)qz * n + (uint32_t)qy) * n + (uint32_t)qx;
}

// Cell and sub-cell tables + reorder + relative coordinates + NGP cell, one
// thread per sorted slot (keys are cell * 8 + octant).  All tables were set
// to kEmpty beforehand.
__global__ void cells_reorder_kernel(const uint32_t *__restrict__ skey, const uint32_t *__restrict__ sidx,
                                     uint32_t N, const float4 *__restrict__ pos,
                                     const double *__restrict__ alpha, uint32_t capN,
                                     const DevParams *__restrict__ P, uint32_t *__restrict__ start,
                                     uint32_t *__restrict__ end, uint32_t *__restrict__ sub_start,
                                     uint32_t *__restrict__ sub_end, uint32_t *__restrict__ mflag, uint32_t epoch,
                                     float4 *__restrict__ vrec, float4 *__restrict__ valf) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    const uint32_t skk = skey[s];
    const uint32_t prev = (s > 0) ? skey[s - 1] : 0u;
    const uint32_t key = skk >> 3;
    if (s == 0 || key != (prev >> 3)) {
        start[key] = s;
        if (s > 0) end[prev >> 3] = s;
    }
    if (s == N - 1) end[key] = N;
    if (s == 0 || skk != prev) {
        sub_start[skk] = s;
        if (s > 0) sub_end[prev] = s;
    }
    if (s == N - 1) sub_end[skk] = N;
    const uint32_t i = sidx[s];
    const float4 p = pos[i];
    const float rx = (float)((double)p.x - P->origin[0]);
    const float ry = (float)((double)p.y - P->origin[1]);
    const float rz = (float)((double)p.z - P->origin[2]);
    const uint32_t cell = ngp_cell(rx, ry, rz, P->invh, P->n);
    if (cell != kEmpty && cell != key) mflag[cell] = epoch;  // rare: rounding put it in a neighbour
    vrec[s] = make_float4(rx, ry, rz, __uint_as_float(cell));
    valf[s] = make_float4((float)alpha[i], (float)alpha[capN + i], (float)alpha[2 * (size_t)capN + i], 0.f);
}

__global__ void cells_only_kernel(const uint32_t *__restrict__ skey, uint32_t N, uint32_t *__restrict__ start,
                                  uint32_t *__restrict__ end) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    const uint32_t key = skey[s];
    if (s == 0 || key != skey[s - 1]) {
        start[key] = s;
        if (s > 0) end[skey[s - 1]] = s;
    }
    if (s == N - 1) end[key] = N;
}

__global__ void gather_sorted_kernel(const uint32_t *__restrict__ sidx, uint32_t N,
                                     const float4 *__restrict__ pos, const double *__restrict__ alpha,
                                     uint32_t capN, float4 *__restrict__ pos_out, double *__restrict__ ax,
                                     double *__restrict__ ay, double *__restrict__ az) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    const uint32_t i = sidx[s];
    if (pos_out) pos_out[s] = pos[i];
    if (ax) ax[s] = alpha[i];
    if (ay) ay[s] = alpha[capN + i];
    if (az) az[s] = alpha[2 * (size_t)capN + i];
}

template <typename T>
__global__ void permute_kernel(const uint32_t *__restrict__ idx, uint32_t N, const T *__restrict__ in,
                               T *__restrict__ out, uint32_t stride, int scatter) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    const size_t src = scatter ? (size_t)s * stride : (size_t)idx[s] * stride;
    const size_t dst = scatter ? (size_t)idx[s] * stride : (size_t)s * stride;
    for (uint32_t q = 0; q < stride; q++) out[dst + q] = in[src + q];
}

inline unsigned blocks_for(uint32_t n, int threads) { return (n + threads - 1) / threads; }

}  // namespace

uint32_t key_bits(uint32_t n) {
    const uint64_t cells = (uint64_t)n * n * n;
    uint32_t b = 0;
    while (b < 32 && (1ull << b) < cells) b++;
    return b == 0 ? 1 : b;
}

size_t radix_hist_entries(uint32_t N) { return 256ull * ((N + kRsTile - 1) / kRsTile) + 256ull; }

cudaError_t launch_bbox_and_params(pppm_scene *s) {
    const int nb = s->bbox_blocks;
    ::pppm::note_launch();
    bbox_partial_kernel<<<nb, kBBoxThreads, 0, s->stream>>>(s->vpos, s->N, s->bbox_partial, nb);
    PPPM_CUDA_TRY(cudaGetLastError());
    ::pppm::note_launch();
    params_kernel<<<1, 32, 0, s->stream>>>(s->bbox_partial, nb, s->prm, s->dparams);
    return cudaGetLastError();
}

// Sorts (key, index) of N points; key[0]/idx[0] hold the keys on entry.
// Returns pointers to the buffers holding the sorted result.
cudaError_t radix_sort_pairs(cudaStream_t st, uint32_t N, uint32_t bits, uint32_t *key[2],
                                    uint32_t *idx[2], uint32_t *hist, uint32_t **sorted_key,
                                    uint32_t **sorted_idx) {
    const uint32_t nb = (N + kRsTile - 1) / kRsTile;
    int cur = 0;
    for (uint32_t shift = 0; shift < bits; shift += 8) {
        ::pppm::note_launch();
        radix_upsweep_kernel<<<nb, kRsThreads, 0, st>>>(key[cur], N, (int)shift, hist);
        PPPM_CUDA_TRY(cudaGetLastError());
        ::pppm::note_launch();
        radix_rowscan_kernel<<<256, kRsThreads, 0, st>>>(hist, nb, hist + 256u * nb);
        PPPM_CUDA_TRY(cudaGetLastError());
        ::pppm::note_launch();
        radix_downsweep_kernel<<<nb, kRsThreads, 0, st>>>(key[cur], idx[cur], key[cur ^ 1], idx[cur ^ 1], N,
                                                          (int)shift, hist, hist + 256u * nb);
        PPPM_CUDA_TRY(cudaGetLastError());
        cur ^= 1;
    }
    *sorted_key = key[cur];
    *sorted_idx = idx[cur];
    return cudaSuccess;
}

cudaError_t launch_hash_sort(pppm_scene *s, const float4 *pos, uint32_t N, uint32_t *key[2], uint32_t *idx[2],
                             uint32_t **sorted_key, uint32_t **sorted_idx) {
    ::pppm::note_launch();
    keys_octant_kernel<<<blocks_for(N, 256), 256, 0, s->stream>>>(pos, N, s->dparams, key[0], idx[0]);
    PPPM_CUDA_TRY(cudaGetLastError());
    return radix_sort_pairs(s->stream, N, key_bits(s->n) + 3, key, idx, s->hist, sorted_key, sorted_idx);
}

// The reference's order (stable by original index inside each cell), built
// on request for the accessors; the near field uses the octant order.
cudaError_t launch_reference_order(pppm_scene *s) {
    ::pppm::note_launch();
    keys_kernel<<<blocks_for(s->N, 256), 256, 0, s->stream>>>(s->vpos, s->N, s->dparams, s->rkey[0], s->ridx[0]);
    PPPM_CUDA_TRY(cudaGetLastError());
    return radix_sort_pairs(s->stream, s->N, key_bits(s->n), s->rkey, s->ridx, s->hist, &s->ref_sorted_key,
                            &s->ref_sorted_idx);
}

cudaError_t launch_cells_reorder(pppm_scene *s) {
    const size_t tbytes = sizeof(uint32_t) * (size_t)s->C;
    PPPM_CUDA_TRY(cudaMemsetAsync(s->cell_start, 0xFF, tbytes, s->stream));
    PPPM_CUDA_TRY(cudaMemsetAsync(s->cell_end, 0xFF, tbytes, s->stream));
    PPPM_CUDA_TRY(cudaMemsetAsync(s->sub_start, 0xFF, 8 * tbytes, s->stream));
    PPPM_CUDA_TRY(cudaMemsetAsync(s->sub_end, 0xFF, 8 * tbytes, s->stream));
    s->epoch++;
    if (s->epoch == 0) {  // wrapped: restart the mismatch flags
        PPPM_CUDA_TRY(cudaMemsetAsync(s->mflag, 0, tbytes, s->stream));
        s->epoch = 1;
    }
    ::pppm::note_launch();
    cells_reorder_kernel<<<blocks_for(s->N, 256), 256, 0, s->stream>>>(
        s->vsorted_key, s->vsorted_idx, s->N, s->vpos, s->valpha, s->capN, s->dparams, s->cell_start,
        s->cell_end, s->sub_start, s->sub_end, s->mflag, s->epoch, s->vrec, s->valf);
    return cudaGetLastError();
}

cudaError_t launch_gather_sorted(pppm_scene *s, float4 *pos_out, double *alpha_out) {
    ::pppm::note_launch();
    gather_sorted_kernel<<<blocks_for(s->N, 256), 256, 0, s->stream>>>(
        s->ref_sorted_idx, s->N, s->vpos, s->valpha, s->capN, pos_out, alpha_out,
        alpha_out ? alpha_out + s->N : nullptr, alpha_out ? alpha_out + 2 * (size_t)s->N : nullptr);
    return cudaGetLastError();
}

cudaError_t launch_explicit_hash(cudaStream_t st, const float4 *pos, uint32_t N, float h, const float of[3],
                                 uint32_t n, uint32_t *key[2], uint32_t *idx[2], uint32_t *hist,
                                 uint32_t **skey, uint32_t **sidx, uint32_t *start, uint32_t *end) {
    ::pppm::note_launch();
    keys_explicit_kernel<<<blocks_for(N, 256), 256, 0, st>>>(pos, N, h, of[0], of[1], of[2], n, key[0], idx[0]);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = radix_sort_pairs(st, N, key_bits(n), key, idx, hist, skey, sidx);
    const size_t C = (size_t)n * n * n;
    if (e == cudaSuccess) e = cudaMemsetAsync(start, 0xFF, sizeof(uint32_t) * C, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(end, 0xFF, sizeof(uint32_t) * C, st);
    if (e == cudaSuccess) {
        ::pppm::note_launch();
        cells_only_kernel<<<blocks_for(N, 256), 256, 0, st>>>(*skey, N, start, end);
        e = cudaGetLastError();
    }
    return e;
}

}  // namespace pppm

// ---------------------------------------------------------------------------
// ParticleManager surface (PH/SpaceHashClass.h:10-84).
// ---------------------------------------------------------------------------
struct pppm_hasher {
    cudaStream_t stream = nullptr;
    uint32_t cap = 0, n = 0, C = 0, N = 0;
    uint32_t *key[2] = {nullptr, nullptr}, *idx[2] = {nullptr, nullptr};
    uint32_t *hist = nullptr;
    uint32_t *start = nullptr, *end = nullptr;
    uint32_t *skey = nullptr, *sidx = nullptr;
};

extern "C" __attribute__((visibility("hidden"))) void pppm_set_error(const char *fmt, ...);

extern "C" pppm_status pppm_hasher_create(uint32_t cap, uint32_t n, void *stream, pppm_hasher **out) {
    if (!out || cap == 0 || n < 2 || n > 1024) {
        pppm_set_error("pppm_hasher_create: invalid argument");
        return PPPM_ERR_INVALID;
    }
    std::lock_guard<std::recursive_mutex> lk(pppm::device_lock());
    pppm_hasher *h = new pppm_hasher();
    h->stream = (cudaStream_t)stream;
    h->cap = cap;
    h->n = n;
    h->C = n * n * n;
    cudaError_t e = cudaSuccess;
    for (int q = 0; q < 2 && e == cudaSuccess; q++) {
        e = ::pppm::device_malloc((void **)&h->key[q], sizeof(uint32_t) * cap);
        if (e == cudaSuccess) e = ::pppm::device_malloc((void **)&h->idx[q], sizeof(uint32_t) * cap);
    }
    if (e == cudaSuccess) e = ::pppm::device_malloc((void **)&h->hist, sizeof(uint32_t) * pppm::radix_hist_entries(cap));
    if (e == cudaSuccess) e = ::pppm::device_malloc((void **)&h->start, sizeof(uint32_t) * h->C);
    if (e == cudaSuccess) e = ::pppm::device_malloc((void **)&h->end, sizeof(uint32_t) * h->C);
    if (e != cudaSuccess) {
        pppm_set_error("pppm_hasher_create: %s", cudaGetErrorString(e));
        pppm_hasher_destroy(h);
        return PPPM_ERR_OOM;
    }
    *out = h;
    return PPPM_OK;
}

extern "C" pppm_status pppm_hasher_destroy(pppm_hasher *h) {
    if (!h) return PPPM_OK;
    std::lock_guard<std::recursive_mutex> lk(pppm::device_lock());
    for (int q = 0; q < 2; q++) {
        cudaFree(h->key[q]);
        cudaFree(h->idx[q]);
    }
    cudaFree(h->hist);
    cudaFree(h->start);
    cudaFree(h->end);
    delete h;
    return PPPM_OK;
}

extern "C" pppm_status pppm_hasher_run(pppm_hasher *h, uint32_t N, const float *pos4_dev, float cell_h,
                                       const float origin[3]) {
    if (!h || !pos4_dev || !origin || N == 0 || N > h->cap || !(cell_h > 0.f)) {
        pppm_set_error("pppm_hasher_run: invalid argument (N=%u cap=%u)", N, h ? h->cap : 0u);
        return PPPM_ERR_INVALID;
    }
    h->N = N;
    const float4 *pos = reinterpret_cast<const float4 *>(pos4_dev);
    ::pppm::note_launch();
    pppm::keys_explicit_kernel<<<(N + 255) / 256, 256, 0, h->stream>>>(pos, N, cell_h, origin[0], origin[1],
                                                                     origin[2], h->n, h->key[0], h->idx[0]);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = pppm::radix_sort_pairs(h->stream, N, pppm::key_bits(h->n), h->key, h->idx, h->hist, &h->skey, &h->sidx);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->start, 0xFF, sizeof(uint32_t) * h->C, h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->end, 0xFF, sizeof(uint32_t) * h->C, h->stream);
    if (e == cudaSuccess) {
        ::pppm::note_launch();
        pppm::cells_only_kernel<<<(N + 255) / 256, 256, 0, h->stream>>>(h->skey, N, h->start, h->end);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        pppm_set_error("pppm_hasher_run: %s", cudaGetErrorString(e));
        return PPPM_ERR_CUDA;
    }
    return PPPM_OK;
}

extern "C" pppm_status pppm_hasher_tables(pppm_hasher *h, const uint32_t **key, const uint32_t **idx,
                                          const uint32_t **start, const uint32_t **end) {
    if (!h || !h->skey) {
        pppm_set_error("pppm_hasher_tables: hash not run");
        return PPPM_ERR_STATE;
    }
    if (key) *key = h->skey;
    if (idx) *idx = h->sidx;
    if (start) *start = h->start;
    if (end) *end = h->end;
    return PPPM_OK;
}

static pppm_status hasher_permute(pppm_hasher *h, uint32_t N, const void *in, void *out, uint32_t stride,
                                  uint32_t precision, int scatter) {
    if (!h || !h->sidx || !in || !out || N > h->N || stride == 0 || (precision != 1 && precision != 2)) {
        pppm_set_error("pppm_hasher_%s: invalid argument", scatter ? "deorder" : "reorder");
        return PPPM_ERR_INVALID;
    }
    ::pppm::note_launch();
    if (precision == 1)
        pppm::permute_kernel<float><<<(N + 255) / 256, 256, 0, h->stream>>>(
            h->sidx, N, (const float *)in, (float *)out, stride, scatter);
    else
        pppm::permute_kernel<double><<<(N + 255) / 256, 256, 0, h->stream>>>(
            h->sidx, N, (const double *)in, (double *)out, stride, scatter);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        pppm_set_error("pppm_hasher permute: %s", cudaGetErrorString(e));
        return PPPM_ERR_CUDA;
    }
    return PPPM_OK;
}

extern "C" pppm_status pppm_hasher_reorder(pppm_hasher *h, uint32_t N, const void *in, void *out,
                                           uint32_t stride, uint32_t precision) {
    return hasher_permute(h, N, in, out, stride, precision, 0);
}

extern "C" pppm_status pppm_hasher_deorder(pppm_hasher *h, uint32_t N, const void *in, void *out,
                                           uint32_t stride, uint32_t precision) {
    return hasher_permute(h, N, in, out, stride, precision, 1);
}

// ---------------------------------------------------------------------------
// Spatial hash that allocates nothing.
//
// For callers that cannot call cudaMalloc on this path: a simulation loop with
// a fixed per-frame budget (cudaMalloc / cudaFree synchronise the device), a
// host whose device allocator must not grow, or a process whose device memory
// is handed out by another framework's pool.  The caller
// passes the positions and the four output arrays; the radix sort's second
// key/index buffer and its digit histograms live in the fixed device array
// below, which every GPU that loads this library holds until the process
// exits (PPPM_NOALLOC_SCRATCH_BYTES, about 8.3 MB).
// ---------------------------------------------------------------------------
#include <mutex>

namespace {

constexpr uint32_t kNoAllocMaxN = PPPM_NOALLOC_MAX_PARTICLES;
constexpr size_t kNoAllocHistWords = 256ull * ((kNoAllocMaxN + pppm::kRsTileHost - 1) / pppm::kRsTileHost) + 256ull;
constexpr size_t kNoAllocWords = 2ull * kNoAllocMaxN + kNoAllocHistWords;
static_assert(kNoAllocWords * 4 == PPPM_NOALLOC_SCRATCH_BYTES, "scratch size in pppm.h is stale");

// Shared by every call on a device; its contents are whatever the last call
// left.  Nothing in it needs to start at zero: each pass overwrites every
// histogram entry and every key/index slot it later reads.
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocWords];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
uint32_t *g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device.  The host-side symbol is only a stand-in and must never be
// passed to a kernel.
cudaError_t noalloc_scratch(uint32_t **out) {
    int dev = 0;
    PPPM_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        PPPM_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_addr[dev] = static_cast<uint32_t *>(p);
    }
    *out = g_noalloc_addr[dev];
    return cudaSuccess;
}

}  // namespace

extern "C" pppm_status pppm_spatial_hash_noalloc(uint32_t N, const float *pos4_dev, uint32_t n, float cell_h,
                                                 const float origin[3], uint32_t *sorted_key_dev,
                                                 uint32_t *sorted_idx_dev, uint32_t *cell_start_dev,
                                                 uint32_t *cell_end_dev, void *stream) {
    if (N > kNoAllocMaxN) {
        pppm_set_error("pppm_spatial_hash_noalloc: N=%u exceeds the fixed scratch limit of %u particles", N,
                       kNoAllocMaxN);
        return PPPM_ERR_INVALID;
    }
    if (N == 0 || !pos4_dev || !origin || !sorted_key_dev || !sorted_idx_dev || !cell_start_dev || !cell_end_dev ||
        n < 2 || n > 1024 || !(cell_h > 0.f)) {
        pppm_set_error("pppm_spatial_hash_noalloc: invalid argument");
        return PPPM_ERR_INVALID;
    }
    uint32_t *scratch = nullptr;
    cudaError_t e = noalloc_scratch(&scratch);
    if (e != cudaSuccess) {
        pppm_set_error("pppm_spatial_hash_noalloc: scratch set-up failed: %s", cudaGetErrorString(e));
        return PPPM_ERR_CUDA;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t bits = pppm::key_bits(n);
    const uint32_t passes = (bits + 7) / 8;
    // The result lands in key[passes % 2]; start in the scratch when the pass
    // count is odd so that it ends in the caller's arrays.
    uint32_t *bk = scratch, *bi = scratch + kNoAllocMaxN, *hist = scratch + 2ull * kNoAllocMaxN;
    uint32_t *key[2], *idx[2];
    if (passes & 1u) {
        key[0] = bk; idx[0] = bi; key[1] = sorted_key_dev; idx[1] = sorted_idx_dev;
    } else {
        key[0] = sorted_key_dev; idx[0] = sorted_idx_dev; key[1] = bk; idx[1] = bi;
    }
    const uint64_t C = (uint64_t)n * n * n;
    ::pppm::note_launch();
    pppm::keys_explicit_kernel<<<(N + 255) / 256, 256, 0, st>>>(reinterpret_cast<const float4 *>(pos4_dev), N,
                                                               cell_h, origin[0], origin[1], origin[2], n, key[0],
                                                               idx[0]);
    e = cudaGetLastError();
    uint32_t *sk = nullptr, *si = nullptr;
    if (e == cudaSuccess) e = pppm::radix_sort_pairs(st, N, bits, key, idx, hist, &sk, &si);
    if (e == cudaSuccess && sk != sorted_key_dev) e = cudaErrorUnknown;  // parity rule above broken
    if (e == cudaSuccess) e = cudaMemsetAsync(cell_start_dev, 0xFF, sizeof(uint32_t) * C, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(cell_end_dev, 0xFF, sizeof(uint32_t) * C, st);
    if (e == cudaSuccess) {
        ::pppm::note_launch();
        pppm::cells_only_kernel<<<(N + 255) / 256, 256, 0, st>>>(sorted_key_dev, N, cell_start_dev, cell_end_dev);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        pppm_set_error("pppm_spatial_hash_noalloc: %s", cudaGetErrorString(e));
        return PPPM_ERR_CUDA;
    }
    return PPPM_OK;
}
