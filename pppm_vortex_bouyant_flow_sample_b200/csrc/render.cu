// Headless particle splatting renderer: the reference's CPU renderer
// (Particle_renderer/particle_renderer/particle_renderer/shadow.cpp
// compute_shadows :56-145, render.cpp render_smoke :61-125) as tile-binned
// CUDA kernels.
//
// Both passes splat every particle, in a distance order, as a disc of weight
// (1 - d^2/r^2)^2 into a 2-D buffer:
//   shadows  nearest-to-the-light first; the shadow map starts at 1 and each
//            disc multiplies it by exp(-opacity * weight); a particle's
//            illumination is the map at its own centre pixel just before its
//            disc is applied;
//   smoke    farthest-from-the-camera first; each disc blends its colour over
//            the image with alpha exp(-opacity * weight).
// The order makes every pixel a sequential fold over the discs that cover it,
// so the kernels keep that fold and parallelise over pixels: particles are
// sorted by distance (stable radix sort on the float bits), each disc's
// bounding box is binned into 16x16-pixel tiles ((tile, rank) pairs, stably
// sorted by tile so ranks stay in order), and one thread block per tile walks
// its list in order with one thread per pixel.
//
// Every float operation that decides coverage or order (distances, the camera
// projection, the disc test) is written with round-to-nearest intrinsics in
// the reference's evaluation order, without contraction, so the sort order and
// the set of covered pixels match the reference compiled without FMA; only
// expf may differ from the host's in the last place.
#include <algorithm>
#include <cmath>
#include <vector>

#include "pppm_internal.cuh"

extern "C" __attribute__((visibility("hidden"))) void pppm_set_error(const char *fmt, ...);

struct pppm_renderer {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t capN = 0, capPairs = 0, capTiles = 0, capMap = 0;
    uint32_t *key[2] = {nullptr, nullptr};
    uint32_t *idx[2] = {nullptr, nullptr};
    uint32_t *hist = nullptr;
    size_t hist_cap = 0;
    float4 *splat = nullptr;       // per rank {x, y, r^2, opacity}
    float4 *rgb = nullptr;         // per rank colour (smoke pass)
    uint32_t *sid = nullptr;       // per rank particle id
    uint32_t *count = nullptr;     // per rank tiles covered, then their offsets
    uint32_t *tiles_of = nullptr;  // per rank tiles covered (kept through the scan)
    int4 *tbox = nullptr;          // per rank tile range {x0, x1, y0, y1}
    uint32_t *bsum = nullptr;      // scan block sums
    uint32_t *pkey[2] = {nullptr, nullptr};
    uint32_t *pval[2] = {nullptr, nullptr};
    uint32_t *tstart = nullptr, *tend = nullptr;
    float *red = nullptr;          // reduction partials
    float *host_red = nullptr;     // pinned
    uint32_t *host_u32 = nullptr;  // pinned
    float *map = nullptr;          // shadow map [npix^2]
    uint32_t npix = 0;
};

namespace pppm {
namespace {

constexpr int kTile = 16;
constexpr int kTileThreads = kTile * kTile;
constexpr int kRedBlocks = 296;
constexpr int kScanItems = 1024;   // 256 threads x 4

__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fdv(float a, float b) { return __fdiv_rn(a, b); }

// vec.h dist / dot: left-to-right sums of rounded products
__device__ __forceinline__ float dist3(float ax, float ay, float az, float bx, float by, float bz) {
    const float dx = fs(ax, bx), dy = fs(ay, by), dz = fs(az, bz);
    float d = fm(dx, dx);
    d = fa(d, fm(dy, dy));
    d = fa(d, fm(dz, dz));
    return __fsqrt_rn(d);
}
__device__ __forceinline__ float dot3(float ax, float ay, float az, const float *b) {
    float d = fm(ax, b[0]);
    d = fa(d, fm(ay, b[1]));
    d = fa(d, fm(az, b[2]));
    return d;
}

struct View {
    float from[3];     // light or camera position
    float cx[3], cy[3], cz[3];
    float scale;       // shadows: perspective scale; smoke: -perspective
    float radius, opacity;
    float half_w;      // shadows: 0.5f * npix; smoke: 0.5f * ni
    int ni, nj;
    int tiles_x;
};

__global__ void minmax_kernel(const float4 *__restrict__ x, uint32_t n, float *__restrict__ out) {
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const float4 p = x[t];
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

// Sort key = bits of dist(x, from) (non-negative floats order as unsigned);
// with `centre`, also the block maximum of dist(x, centre).
__global__ void dist_kernel(const float4 *__restrict__ x, uint32_t n, float fx, float fy, float fz,
                            uint32_t *__restrict__ key, uint32_t *__restrict__ idx, int with_centre, float cx,
                            float cy, float cz, float *__restrict__ maxout) {
    float m = 0.0f;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const float4 p = x[t];
        key[t] = __float_as_uint(dist3(p.x, p.y, p.z, fx, fy, fz));
        idx[t] = t;
        if (with_centre) m = fmaxf(m, dist3(p.x, p.y, p.z, cx, cy, cz));
    }
    if (!with_centre) return;
    __shared__ float sh[8];
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        float v = sh[0];
        for (int q = 1; q < (int)(blockDim.x >> 5); q++) v = fmaxf(v, sh[q]);
        maxout[blockIdx.x] = v;
    }
}

__device__ __forceinline__ int clamp_trunc(float v, int lo, int hi) {
    // (int)v clamped to [lo, hi]; values far outside never reach the int cast
    if (!(v > (float)(lo - 1))) return lo - 1;
    if (v > (float)(hi + 1)) return hi + 1;
    return (int)v;
}

// Per processing rank r: screen disc, colour, and the tile range its bounding
// box touches (blot's ilo = (int)(x - r), ihi = ceil(x + r), clamped to the
// image; an empty box touches none).
template <bool SHADOW>
__global__ void project_kernel(const float4 *__restrict__ x, const uint32_t *__restrict__ order, uint32_t n,
                               const View v, const float *__restrict__ dens, const float *__restrict__ illum,
                               const float *__restrict__ base_rgb, const float *__restrict__ lit_rgb,
                               float4 *__restrict__ splat, float4 *__restrict__ rgb, uint32_t *__restrict__ sid,
                               int4 *__restrict__ tbox, uint32_t *__restrict__ count) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    // shadows: nearest to the light first; smoke: farthest from the camera first
    const uint32_t j = SHADOW ? order[r] : order[n - 1 - r];
    sid[r] = j;
    const float4 p4 = x[j];
    const float px_ = fs(p4.x, v.from[0]), py_ = fs(p4.y, v.from[1]), pz_ = fs(p4.z, v.from[2]);
    const float u = dot3(px_, py_, pz_, v.cx), vv = dot3(px_, py_, pz_, v.cy), w = dot3(px_, py_, pz_, v.cz);
    float sx, sy, sr;
    if (SHADOW) {
        sx = fa(fdv(fm(v.scale, u), w), v.half_w);
        sy = fa(fdv(fm(v.scale, vv), w), v.half_w);
        sr = fdv(fm(v.scale, v.radius), w);
    } else {
        if (w >= 0.0f) {  // behind the camera: not drawn
            splat[r] = make_float4(0.f, 0.f, 0.f, 0.f);
            count[r] = 0;
            return;
        }
        sx = fa(fm(fdv(fm(v.scale, u), w), (float)v.nj), v.half_w);
        sy = fm(fa(fdv(fm(v.scale, vv), w), 0.5f), (float)v.nj);
        sr = fm(fdv(fm(v.scale, v.radius), w), (float)v.nj);
    }
    splat[r] = make_float4(sx, sy, fm(sr, sr), fm(v.opacity, dens[j]));
    if (!SHADOW) {
        const float il = illum[j];
        const float one = fs(1.0f, il);
        rgb[r] = make_float4(fa(fm(one, base_rgb[3 * j]), fm(il, lit_rgb[3 * j])),
                             fa(fm(one, base_rgb[3 * j + 1]), fm(il, lit_rgb[3 * j + 1])),
                             fa(fm(one, base_rgb[3 * j + 2]), fm(il, lit_rgb[3 * j + 2])), 0.f);
    }
    const int ilo = max(clamp_trunc(fs(sx, sr), 0, v.ni - 1), 0);
    const int ihi = min(clamp_trunc(ceilf(fa(sx, sr)), 0, v.ni - 1), v.ni - 1);
    const int jlo = max(clamp_trunc(fs(sy, sr), 0, v.nj - 1), 0);
    const int jhi = min(clamp_trunc(ceilf(fa(sy, sr)), 0, v.nj - 1), v.nj - 1);
    uint32_t tiles = 0;
    if (ilo <= ihi && jlo <= jhi) {
        const int4 b = make_int4(ilo / kTile, ihi / kTile, jlo / kTile, jhi / kTile);
        tbox[r] = b;
        tiles = (uint32_t)((b.y - b.x + 1) * (b.w - b.z + 1));
    }
    count[r] = tiles;
}

// Exclusive scan of counts in blocks of 1024, block totals to bsum.
__global__ void scan_block_kernel(uint32_t *__restrict__ data, uint32_t n, uint32_t *__restrict__ bsum) {
    __shared__ uint32_t wsum[8];
    const uint32_t base = blockIdx.x * kScanItems + threadIdx.x * 4;
    uint32_t v[4], s = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        v[q] = (base + q < n) ? data[base + q] : 0u;
        s += v[q];
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t incl = s;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    uint32_t wpre = 0;
    for (int q = 0; q < w; q++) wpre += wsum[q];
    uint32_t run = wpre + incl - s;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        if (base + q < n) data[base + q] = run;
        run += v[q];
    }
    if (threadIdx.x == blockDim.x - 1) bsum[blockIdx.x] = wpre + incl;
}

// Exclusive scan of the block totals in one block; the grand total goes to
// bsum[nb].
__global__ void scan_sums_kernel(uint32_t *__restrict__ bsum, uint32_t nb) {
    __shared__ uint32_t wsum[8];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t base = 0; base < nb; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t s = i < nb ? bsum[i] : 0u;
        uint32_t incl = s;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) wsum[w] = incl;
        __syncthreads();
        uint32_t wpre = 0;
        for (int q = 0; q < w; q++) wpre += wsum[q];
        const uint32_t c = carry;
        if (i < nb) bsum[i] = c + wpre + incl - s;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = c + wpre + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) bsum[nb] = carry;
}

__global__ void scan_add_kernel(uint32_t *__restrict__ data, uint32_t n, const uint32_t *__restrict__ bsum) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) data[i] += bsum[i / kScanItems];
}

// (tile, rank) pairs, written in rank order.
__global__ void emit_kernel(const int4 *__restrict__ tbox, const uint32_t *__restrict__ offset,
                            const uint32_t *__restrict__ tiles_of, uint32_t n, int tiles_x,
                            uint32_t *__restrict__ pkey, uint32_t *__restrict__ pval) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    if (tiles_of[r] == 0) return;
    const int4 b = tbox[r];
    uint32_t o = offset[r];
    for (int ty = b.z; ty <= b.w; ty++)
        for (int tx = b.x; tx <= b.y; tx++) {
            pkey[o] = (uint32_t)(ty * tiles_x + tx);
            pval[o] = r;
            o++;
        }
}

__global__ void tile_ranges_kernel(const uint32_t *__restrict__ skey, uint32_t n, uint32_t *__restrict__ start,
                                   uint32_t *__restrict__ end) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint32_t k = skey[s];
    if (s == 0 || k != skey[s - 1]) {
        start[k] = s;
        if (s > 0) end[skey[s - 1]] = s;
    }
    if (s == n - 1) end[k] = n;
}

__global__ void fill_kernel(float *__restrict__ p, uint32_t n, float v) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// One block per tile, one thread per pixel; the tile's discs in rank order.
//   shadows: T *= exp(-opacity * (1 - t/r^2)^2) where t = |pixel - centre|^2 < r^2;
//            a disc's own centre pixel ((int)x, (int)y) records T first
//   smoke:   c = a c + (1 - a) rgb with a = exp(-opacity * (1 - t/r^2)^2)
template <bool SHADOW>
__global__ void __launch_bounds__(kTileThreads) tile_kernel(
    const uint32_t *__restrict__ tstart, const uint32_t *__restrict__ tend, const uint32_t *__restrict__ prank,
    const float4 *__restrict__ splat, const float4 *__restrict__ rgb, const uint32_t *__restrict__ sid, int ni,
    int nj, int tiles_x, float bg0, float bg1, float bg2, float *__restrict__ out, float *__restrict__ illum) {
    __shared__ float4 s_sp[kTileThreads];
    __shared__ float4 s_col[kTileThreads];
    __shared__ uint32_t s_id[kTileThreads];
    const uint32_t tile = blockIdx.x;
    const int i = (int)(tile % tiles_x) * kTile + (int)(threadIdx.x % kTile);
    const int j = (int)(tile / tiles_x) * kTile + (int)(threadIdx.x / kTile);
    const bool inside = i < ni && j < nj;
    const float fi = (float)i, fj = (float)j;
    float tr = 1.0f, c0 = bg0, c1 = bg1, c2 = bg2;
    const uint32_t s0 = tstart[tile];
    const uint32_t s1 = (s0 == kEmpty) ? 0u : tend[tile];
    for (uint32_t base = (s0 == kEmpty ? 0u : s0); base < s1; base += kTileThreads) {
        const uint32_t k = base + threadIdx.x;
        if (k < s1) {
            const uint32_t r = prank[k];
            s_sp[threadIdx.x] = splat[r];
            if (SHADOW) s_id[threadIdx.x] = sid[r];
            else s_col[threadIdx.x] = rgb[r];
        }
        __syncthreads();
        const uint32_t cnt = min((uint32_t)kTileThreads, s1 - base);
        if (inside) {
            for (uint32_t q = 0; q < cnt; q++) {
                const float4 sp = s_sp[q];
                if (SHADOW && sp.x >= 0.0f && sp.y >= 0.0f && (int)sp.x == i && (int)sp.y == j) illum[s_id[q]] = tr;
                const float u = fs(sp.y, fj), v = fs(sp.x, fi);
                const float t = fa(fm(u, u), fm(v, v));
                if (t < sp.z) {
                    const float k1 = fs(1.0f, fdv(t, sp.z));
                    const float a = expf(fm(-sp.w, fm(k1, k1)));
                    if (SHADOW) {
                        tr = fm(tr, a);
                    } else {
                        const float4 cc = s_col[q];
                        const float oa = fs(1.0f, a);
                        c0 = fa(fm(a, c0), fm(oa, cc.x));
                        c1 = fa(fm(a, c1), fm(oa, cc.y));
                        c2 = fa(fm(a, c2), fm(oa, cc.z));
                    }
                }
            }
        }
        __syncthreads();
    }
    if (!inside) return;
    const size_t px = (size_t)i + (size_t)ni * j;
    if (SHADOW) {
        out[px] = tr;
    } else {
        out[3 * px] = c0;
        out[3 * px + 1] = c1;
        out[3 * px + 2] = c2;
    }
}

template <typename T>
cudaError_t grow(T **p, size_t count) {
    cudaFree(*p);
    *p = nullptr;
    return ::pppm::device_malloc((void **)p, sizeof(T) * (count ? count : 1));
}

// Capacities are raised only once every buffer they cover exists; a failed
// growth leaves capacity 0 so that the next call allocates again.
cudaError_t ensure_particles(pppm_renderer *R, uint32_t n) {
    if (n <= R->capN) return cudaSuccess;
    std::lock_guard<std::recursive_mutex> lk(device_lock());
    R->capN = 0;
    for (int q = 0; q < 2; q++) {
        PPPM_CUDA_TRY(grow(&R->key[q], n));
        PPPM_CUDA_TRY(grow(&R->idx[q], n));
    }
    PPPM_CUDA_TRY(grow(&R->splat, n));
    PPPM_CUDA_TRY(grow(&R->rgb, n));
    PPPM_CUDA_TRY(grow(&R->sid, n));
    PPPM_CUDA_TRY(grow(&R->count, (size_t)n + 1));
    PPPM_CUDA_TRY(grow(&R->tiles_of, n));
    PPPM_CUDA_TRY(grow(&R->tbox, n));
    PPPM_CUDA_TRY(grow(&R->bsum, (size_t)n / kScanItems + 2));
    R->capN = n;
    return cudaSuccess;
}

cudaError_t ensure_pairs(pppm_renderer *R, uint32_t pairs, uint32_t tiles) {
    std::lock_guard<std::recursive_mutex> lk(device_lock());
    if (pairs > R->capPairs) {
        R->capPairs = 0;
        for (int q = 0; q < 2; q++) {
            PPPM_CUDA_TRY(grow(&R->pkey[q], pairs));
            PPPM_CUDA_TRY(grow(&R->pval[q], pairs));
        }
        R->capPairs = pairs;
    }
    const size_t need = radix_hist_entries(std::max(pairs, R->capN));
    if (need > R->hist_cap) {
        R->hist_cap = 0;
        PPPM_CUDA_TRY(grow(&R->hist, need));
        R->hist_cap = need;
    }
    if (tiles > R->capTiles) {
        R->capTiles = 0;
        PPPM_CUDA_TRY(grow(&R->tstart, tiles));
        PPPM_CUDA_TRY(grow(&R->tend, tiles));
        R->capTiles = tiles;
    }
    return cudaSuccess;
}

uint32_t bits_for(uint32_t v) {
    uint32_t b = 1;
    while (b < 32 && (1ull << b) < (uint64_t)v) b++;
    return b;
}

// Host copies of the reference's float vector arithmetic (vec.h), for the
// camera frames; the host code is compiled without FMA contraction.
struct V3 {
    float v[3];
};
V3 sub(V3 a, V3 b) { return {{a.v[0] - b.v[0], a.v[1] - b.v[1], a.v[2] - b.v[2]}}; }
float dotv(V3 a, V3 b) {
    float d = a.v[0] * b.v[0];
    d += a.v[1] * b.v[1];
    d += a.v[2] * b.v[2];
    return d;
}
float magv(V3 a) { return std::sqrt(dotv(a, a)); }
V3 divs(V3 a, float s) { return {{a.v[0] / s, a.v[1] / s, a.v[2] / s}}; }
V3 crossv(V3 a, V3 b) {
    return {{a.v[1] * b.v[2] - a.v[2] * b.v[1], a.v[2] * b.v[0] - a.v[0] * b.v[2], a.v[0] * b.v[1] - a.v[1] * b.v[0]}};
}
float distv(V3 a, V3 b) {
    const V3 d = sub(a, b);
    float s = d.v[0] * d.v[0];
    s += d.v[1] * d.v[1];
    s += d.v[2] * d.v[2];
    return std::sqrt(s);
}

// Sort by distance to `from` (stable), project, bin into tiles, and run the
// tile kernel.  Returns the number of (tile, disc) pairs through *pairs_out.
template <bool SHADOW>
cudaError_t splat_pass(pppm_renderer *R, uint32_t n, const float4 *x, const View &v, const float *dens,
                       const float *illum, const float *base_rgb, const float *lit_rgb, uint32_t *order,
                       float bg0, float bg1, float bg2, float *out, float *illum_out, uint64_t *pairs_out) {
    cudaStream_t st = R->stream;
    const uint32_t tiles_x = (uint32_t)((v.ni + kTile - 1) / kTile), tiles_y = (uint32_t)((v.nj + kTile - 1) / kTile);
    const uint32_t tiles = tiles_x * tiles_y;
    note_launch();
    project_kernel<SHADOW><<<(n + 255) / 256, 256, 0, st>>>(x, order, n, v, dens, illum, base_rgb, lit_rgb,
                                                            R->splat, R->rgb, R->sid, R->tbox, R->count);
    PPPM_CUDA_TRY(cudaGetLastError());
    PPPM_CUDA_TRY(cudaMemcpyAsync(R->tiles_of, R->count, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
    const uint32_t nb = (n + kScanItems - 1) / kScanItems;
    note_launch();
    scan_block_kernel<<<nb, 256, 0, st>>>(R->count, n, R->bsum);
    note_launch();
    scan_sums_kernel<<<1, 256, 0, st>>>(R->bsum, nb);
    note_launch();
    scan_add_kernel<<<(n + 255) / 256, 256, 0, st>>>(R->count, n, R->bsum);
    PPPM_CUDA_TRY(cudaGetLastError());
    PPPM_CUDA_TRY(cudaMemcpyAsync(R->host_u32, R->bsum + nb, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    PPPM_CUDA_TRY(cudaStreamSynchronize(st));
    const uint32_t pairs = R->host_u32[0];
    if (pairs_out) *pairs_out = pairs;
    PPPM_CUDA_TRY(ensure_pairs(R, pairs, tiles));
    PPPM_CUDA_TRY(cudaMemsetAsync(R->tstart, 0xFF, sizeof(uint32_t) * tiles, st));
    PPPM_CUDA_TRY(cudaMemsetAsync(R->tend, 0xFF, sizeof(uint32_t) * tiles, st));
    uint32_t *skey = R->pkey[0], *sval = R->pval[0];
    if (pairs > 0) {
        note_launch();
        emit_kernel<<<(n + 255) / 256, 256, 0, st>>>(R->tbox, R->count, R->tiles_of, n, (int)tiles_x, R->pkey[0],
                                                     R->pval[0]);
        PPPM_CUDA_TRY(cudaGetLastError());
        PPPM_CUDA_TRY(radix_sort_pairs(st, pairs, bits_for(tiles), R->pkey, R->pval, R->hist, &skey, &sval));
        note_launch();
        tile_ranges_kernel<<<(pairs + 255) / 256, 256, 0, st>>>(skey, pairs, R->tstart, R->tend);
        PPPM_CUDA_TRY(cudaGetLastError());
    }
    note_launch();
    tile_kernel<SHADOW><<<tiles, kTileThreads, 0, st>>>(R->tstart, R->tend, sval, R->splat, R->rgb, R->sid, v.ni,
                                                        v.nj, (int)tiles_x, bg0, bg1, bg2, out, illum_out);
    return cudaGetLastError();
}

cudaError_t sort_by_distance(pppm_renderer *R, uint32_t n, const float4 *x, V3 from, bool with_centre, V3 centre,
                             uint32_t **order) {
    cudaStream_t st = R->stream;
    note_launch();
    dist_kernel<<<kRedBlocks, 256, 0, st>>>(x, n, from.v[0], from.v[1], from.v[2], R->key[0], R->idx[0],
                                            with_centre ? 1 : 0, centre.v[0], centre.v[1], centre.v[2], R->red);
    PPPM_CUDA_TRY(cudaGetLastError());
    uint32_t *skey = nullptr;
    const size_t need = radix_hist_entries(n);
    if (need > R->hist_cap) {
        std::lock_guard<std::recursive_mutex> lk(device_lock());
        PPPM_CUDA_TRY(grow(&R->hist, need));
        R->hist_cap = need;
    }
    return radix_sort_pairs(st, n, 32, R->key, R->idx, R->hist, &skey, order);
}

}  // namespace
}  // namespace pppm

using pppm::V3;

extern "C" pppm_status pppm_renderer_create(void *stream, pppm_renderer **out) {
    if (!out) {
        pppm_set_error("pppm_renderer_create: out is NULL");
        return PPPM_ERR_INVALID;
    }
    std::lock_guard<std::recursive_mutex> lk(pppm::device_lock());
    pppm_renderer *R = new pppm_renderer;
    R->stream = (cudaStream_t)stream;
    cudaGetDevice(&R->device);
    cudaError_t e = ::pppm::device_malloc((void **)&R->red, sizeof(float) * 6 * pppm::kRedBlocks);
    if (e == cudaSuccess) e = ::pppm::host_malloc((void **)&R->host_red, sizeof(float) * 6 * pppm::kRedBlocks);
    if (e == cudaSuccess) e = ::pppm::host_malloc((void **)&R->host_u32, sizeof(uint32_t) * 4);
    if (e != cudaSuccess) {
        pppm_set_error("pppm_renderer_create: %s", cudaGetErrorString(e));
        pppm_renderer_destroy(R);
        return PPPM_ERR_OOM;
    }
    *out = R;
    return PPPM_OK;
}

extern "C" pppm_status pppm_renderer_destroy(pppm_renderer *R) {
    if (!R) return PPPM_OK;
    std::lock_guard<std::recursive_mutex> lk(pppm::device_lock());
    for (int q = 0; q < 2; q++) {
        cudaFree(R->key[q]); cudaFree(R->idx[q]); cudaFree(R->pkey[q]); cudaFree(R->pval[q]);
    }
    cudaFree(R->hist); cudaFree(R->splat); cudaFree(R->rgb); cudaFree(R->sid); cudaFree(R->count);
    cudaFree(R->tiles_of); cudaFree(R->tbox); cudaFree(R->bsum); cudaFree(R->tstart); cudaFree(R->tend);
    cudaFree(R->red); cudaFree(R->map);
    if (R->host_red) cudaFreeHost(R->host_red);
    if (R->host_u32) cudaFreeHost(R->host_u32);
    delete R;
    return PPPM_OK;
}

static pppm_status render_fail(const char *where, cudaError_t e) {
    pppm_set_error("%s: %s", where, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? PPPM_ERR_OOM : PPPM_ERR_CUDA;
}

extern "C" pppm_status pppm_render_shadows(pppm_renderer *R, uint32_t n, const float *pos4, const float *dens,
                                           float radius, float opacity, const float light[3], float quality,
                                           float *illum, uint32_t *npix_out) {
    using namespace pppm;
    if (!R || !light || (n > 0 && (!pos4 || !dens || !illum)) || !(radius > 0.0f)) {
        pppm_set_error("pppm_render_shadows: invalid argument");
        return PPPM_ERR_INVALID;
    }
    if (npix_out) *npix_out = 0;
    if (n == 0) return PPPM_OK;
    cudaStream_t st = R->stream;
    cudaError_t e = ensure_particles(R, n);
    if (e != cudaSuccess) return render_fail("pppm_render_shadows (alloc)", e);
    const float4 *x = reinterpret_cast<const float4 *>(pos4);
    // bounding box, then the bounding sphere about its centre (two host reads)
    note_launch();
    minmax_kernel<<<kRedBlocks, 256, 0, st>>>(x, n, R->red);
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(R->host_red, R->red, sizeof(float) * 6 * kRedBlocks, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return render_fail("pppm_render_shadows (bbox)", e);
    V3 xmin, xmax;
    for (int c = 0; c < 3; c++) {
        float lo = R->host_red[c * kRedBlocks], hi = R->host_red[(3 + c) * kRedBlocks];
        for (int q = 1; q < kRedBlocks; q++) {
            lo = std::min(lo, R->host_red[c * kRedBlocks + q]);
            hi = std::max(hi, R->host_red[(3 + c) * kRedBlocks + q]);
        }
        xmin.v[c] = lo;
        xmax.v[c] = hi;
    }
    const V3 centre = {{(xmin.v[0] + xmax.v[0]) / 2, (xmin.v[1] + xmax.v[1]) / 2, (xmin.v[2] + xmax.v[2]) / 2}};
    const V3 L = {{light[0], light[1], light[2]}};
    uint32_t *order = nullptr;
    e = sort_by_distance(R, n, x, L, true, centre, &order);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(R->host_red, R->red, sizeof(float) * kRedBlocks, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return render_fail("pppm_render_shadows (sort)", e);
    float r = 0.0f;
    for (int q = 0; q < kRedBlocks; q++) r = std::max(r, R->host_red[q]);
    if (distv(L, centre) < 1.25f * r) {
        pppm_set_error("pppm_render_shadows: light is too close to the particles (inside 1.25 x the bounding sphere)");
        return PPPM_ERR_DOMAIN;
    }
    // orthogonal frame looking from the light at the centre (shadow.cpp:104-118)
    const V3 d0 = sub(centre, L);
    const V3 camz = divs(d0, magv(d0));
    V3 camy;
    if (std::fabs(camz.v[0]) >= std::fabs(camz.v[1]) && std::fabs(camz.v[0]) >= std::fabs(camz.v[2])) {
        camy = {{-camz.v[1], camz.v[0], 0}};
    } else {
        camy = {{0, -camz.v[2], camz.v[1]}};
    }
    camy = divs(camy, magv(camy));
    const V3 camx = crossv(camy, camz);
    const int npix = int(quality * r / radius);
    if (npix <= 0 || npix > 16384) {
        pppm_set_error("pppm_render_shadows: shadow map edge %d outside [1, 16384]", npix);
        return PPPM_ERR_INVALID;
    }
    const float scale = 0.4 * npix * distv(centre, L) / r;
    View v{};
    for (int c = 0; c < 3; c++) {
        v.from[c] = L.v[c]; v.cx[c] = camx.v[c]; v.cy[c] = camy.v[c]; v.cz[c] = camz.v[c];
    }
    v.scale = scale;
    v.radius = radius;
    v.opacity = opacity;
    v.half_w = 0.5f * npix;
    v.ni = v.nj = npix;
    v.tiles_x = (npix + kTile - 1) / kTile;
    const uint32_t cells = (uint32_t)npix * (uint32_t)npix;
    if (cells > R->capMap) {
        std::lock_guard<std::recursive_mutex> lk(device_lock());
        R->capMap = 0;
        R->npix = 0;   // no shadow map until this one is drawn
        e = grow(&R->map, cells);
        if (e != cudaSuccess) return render_fail("pppm_render_shadows (map)", e);
        R->capMap = cells;
    }
    note_launch();
    fill_kernel<<<(n + 255) / 256, 256, 0, st>>>(illum, n, 1.0f);
    e = cudaGetLastError();
    uint64_t pairs = 0;
    if (e == cudaSuccess)
        e = splat_pass<true>(R, n, x, v, dens, nullptr, nullptr, nullptr, order, 0.f, 0.f, 0.f, R->map, illum, &pairs);
    if (e != cudaSuccess) return render_fail("pppm_render_shadows", e);
    R->npix = (uint32_t)npix;
    if (npix_out) *npix_out = (uint32_t)npix;
    return PPPM_OK;
}

extern "C" pppm_status pppm_render_shadow_map(pppm_renderer *R, const float **map_dev, uint32_t *npix) {
    if (!R || R->npix == 0) {
        pppm_set_error("pppm_render_shadow_map: no shadow map rendered");
        return PPPM_ERR_STATE;
    }
    if (map_dev) *map_dev = R->map;
    if (npix) *npix = R->npix;
    return PPPM_OK;
}

extern "C" pppm_status pppm_render_smoke(pppm_renderer *R, uint32_t n, const float *pos4, const float *illum,
                                         const float *base_rgb, const float *lit_rgb, float radius, float opacity,
                                         const float *den, const float background[3], const float camera[3],
                                         const float target[3], float perspective, uint32_t width, uint32_t height,
                                         float *image) {
    using namespace pppm;
    if (!R || !background || !camera || !target || !image || width == 0 || height == 0 || width > 16384 ||
        height > 16384 || (n > 0 && (!pos4 || !illum || !base_rgb || !lit_rgb || !den))) {
        pppm_set_error("pppm_render_smoke: invalid argument");
        return PPPM_ERR_INVALID;
    }
    cudaStream_t st = R->stream;
    const V3 cam = {{camera[0], camera[1], camera[2]}}, tgt = {{target[0], target[1], target[2]}};
    // camera frame (render.cpp:88-91)
    const V3 d0 = sub(cam, tgt);
    const V3 camz = divs(d0, magv(d0));
    const V3 zc = crossv(V3{{0, 0, 1}}, camz);
    const V3 camx = divs(zc, magv(zc));
    const V3 camy = crossv(camz, camx);
    View v{};
    for (int c = 0; c < 3; c++) {
        v.from[c] = cam.v[c]; v.cx[c] = camx.v[c]; v.cy[c] = camy.v[c]; v.cz[c] = camz.v[c];
    }
    v.scale = -perspective;
    v.radius = radius;
    v.opacity = opacity;
    v.half_w = 0.5f * (float)width;
    v.ni = (int)width;
    v.nj = (int)height;
    v.tiles_x = (int)((width + kTile - 1) / kTile);
    if (n == 0) {
        const uint32_t tiles = (uint32_t)v.tiles_x * ((height + kTile - 1) / kTile);
        cudaError_t e = ensure_pairs(R, 0, tiles);
        if (e == cudaSuccess) e = cudaMemsetAsync(R->tstart, 0xFF, sizeof(uint32_t) * tiles, st);
        if (e == cudaSuccess) {
            note_launch();
            tile_kernel<false><<<tiles, kTileThreads, 0, st>>>(R->tstart, R->tend, nullptr, nullptr, nullptr,
                                                               nullptr, v.ni, v.nj, v.tiles_x, background[0],
                                                               background[1], background[2], image, nullptr);
            e = cudaGetLastError();
        }
        return e == cudaSuccess ? PPPM_OK : render_fail("pppm_render_smoke", e);
    }
    cudaError_t e = ensure_particles(R, n);
    if (e != cudaSuccess) return render_fail("pppm_render_smoke (alloc)", e);
    const float4 *x = reinterpret_cast<const float4 *>(pos4);
    uint32_t *order = nullptr;
    e = sort_by_distance(R, n, x, cam, false, cam, &order);
    uint64_t pairs = 0;
    if (e == cudaSuccess)
        e = splat_pass<false>(R, n, x, v, den, illum, base_rgb, lit_rgb, order, background[0], background[1],
                              background[2], image, nullptr, &pairs);
    if (e != cudaSuccess) return render_fail("pppm_render_smoke", e);
    return PPPM_OK;
}
