// Buoyancy source of the reference's plume: heat particles -> density grid ->
// baroclinic vorticity on the vortices (VortexSimulationSystem::
// addBaroclinicForce, HFS/VortexSimulationSystemImp.cpp:369-465).
//
//   setDensityDomain (:336-366)   1.2 x the heat particles' bounding box
//   grid edge                     min(floor(L / 0.2) + 1, 200), h = L / edge
//   hash                          the reference hash on that grid (float h, origin)
//   AssignDensity                 per grid cell, quartic-weighted mean of the
//     (HFS/GPU_kernel.cu:3655-3740)  heat of the particles in the 5^3 hash cells
//                                 around it; an empty hash cell adds its own
//                                 centre's weight with zero heat
//   GradDensity (:3742-3797)      periodic central differences
//   ParticleGetBaroclinic         grad rho interpolated at each vortex (hat
//     (:3800-3898)                 weights over 5^3 cells), crossed with
//                                 (0, 10, 0), times 5 dt * 0.1, added to alpha
//
// The quartic weight (1 - d^2)^4 vanishes for d >= 1 cell, so only particles in
// the 3^3 hash cells around a grid cell can carry weight, and an empty hash
// cell's centre weighs 1 only for the grid cell's own hash cell: the density
// kernel walks 3^3 cells and adds that 1, which gives the same terms as the
// reference's 5^3 walk.  Work item = (grid cell, slice of its particles); a
// warp per item, FP64 sums reduced in a fixed order, so the result does not
// depend on scheduling.  Small grids with many particles (a compact plume puts
// millions of particles in a handful of cells) split each cell's particles
// over up to 256 warps and combine the partial sums in a second pass.
//
// One deliberate difference: the reference launches ParticleGetBaroclinic with
// its block and grid sizes swapped (HFS/GPU_kernel.cu:3897), which fails for
// more than 262,144 vortices (more than 1024 threads per block) and then adds
// nothing.  Here the force is applied to every vortex.
#include <algorithm>
#include <cmath>
#include <cstdio>

#include "pppm_internal.cuh"

extern "C" __attribute__((visibility("hidden"))) void pppm_set_error(const char *fmt, ...);

namespace pppm {

struct Buoyancy {
    uint32_t capH = 0;
    size_t capC = 0, capPart = 0;
    uint32_t *key[2] = {nullptr, nullptr};
    uint32_t *idx[2] = {nullptr, nullptr};
    uint32_t *hist = nullptr;
    float4 *rec = nullptr;        // sorted {rel.x, rel.y, rel.z, heat}
    float *bbox = nullptr;        // [6][kBBoxBlocks] block partial min / max
    uint32_t *start = nullptr, *end = nullptr;
    float *rho = nullptr;         // [C]
    float *grad = nullptr;        // [3][C]
    double2 *part = nullptr;      // [C * S] partial (sum, weight)
    float *host_bbox = nullptr;   // pinned [6][kBBoxBlocks]
    // last run, for the accessors
    uint32_t dim = 0;
    double origin[3] = {0, 0, 0};
    double h = 0.0;
};

namespace {

constexpr int kBBoxBlocks = 296;
constexpr int kMaxSplit = 256;

__global__ void heat_bbox_kernel(const float4 *__restrict__ pos, uint32_t N, float *__restrict__ out) {
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

// Sorted heat records: position relative to the FP64 origin rounded to float
// (the reference's `ppos.x -= origin.x` on a float4), and the heat value.
__global__ void heat_records_kernel(const float4 *__restrict__ pos, const float *__restrict__ heat,
                                    const uint32_t *__restrict__ sidx, uint32_t N, double ox, double oy, double oz,
                                    float4 *__restrict__ rec) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    const uint32_t i = sidx[s];
    const float4 p = pos[i];
    rec[s] = make_float4((float)((double)p.x - ox), (float)((double)p.y - oy), (float)((double)p.z - oz), heat[i]);
}

__device__ __forceinline__ double quartic(double r) {
    const double rr = fabs(r);
    const double r1 = 1.0 - rr;
    const double r2 = r1 * r1;
    const double r4 = r2 * r2;
    return rr < 1.0 ? r4 : 0.0;
}

// One warp per (grid cell, slice).  Lanes take the slice's particles of the
// 3^3 hash cells around the grid cell in (k, j, i, p) order; the warp then
// reduces its FP64 sums with a fixed butterfly.
template <bool FINAL>
__global__ void assign_density_kernel(
    const uint32_t *__restrict__ start, const uint32_t *__restrict__ end, const float4 *__restrict__ rec,
    uint32_t dim, uint32_t S, double invh, float *__restrict__ rho, double2 *__restrict__ part) {
    const uint64_t item = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t cells = (uint64_t)dim * dim * dim;
    if (item >= cells * S) return;
    const int lane = threadIdx.x & 31;
    const uint32_t c = (uint32_t)(item / S), sl = (uint32_t)(item % S);
    const int d = (int)dim;
    const int i = (int)(c % dim), j = (int)((c / dim) % dim), k = (int)(c / (dim * dim));
    const double gx = i + 0.5, gy = j + 0.5, gz = k + 0.5;
    double sum = 0.0, tw = 0.0;
    const uint32_t stride = 32u * S;
    for (int kk = max(k - 1, 0); kk <= min(k + 1, d - 1); kk++)
        for (int jj = max(j - 1, 0); jj <= min(j + 1, d - 1); jj++)
            for (int ii = max(i - 1, 0); ii <= min(i + 1, d - 1); ii++) {
                const uint32_t r = ((uint32_t)kk * dim + (uint32_t)jj) * dim + (uint32_t)ii;
                const uint32_t s0 = start[r];
                if (s0 == kEmpty) continue;
                const uint32_t s1 = end[r];
                for (uint32_t p = s0 + sl * 32u + (uint32_t)lane; p < s1; p += stride) {
                    const float4 q = rec[p];
                    const double dx = gx - (double)q.x * invh, dy = gy - (double)q.y * invh,
                                 dz = gz - (double)q.z * invh;
                    const double w = quartic(dx * dx + dy * dy + dz * dz);
                    sum += w * (double)q.w;
                    tw += w;
                }
            }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
        tw += __shfl_xor_sync(0xffffffffu, tw, o);
    }
    if (lane != 0) return;
    if (FINAL) {
        if (start[c] == kEmpty) tw += 1.0;  // the empty own hash cell's centre
        if (tw < 1e-12) tw = 1e+24;
        rho[c] = (float)(sum / tw);
    } else {
        part[item] = make_double2(sum, tw);
    }
}

__global__ void density_finish_kernel(const double2 *__restrict__ part, const uint32_t *__restrict__ start,
                                      uint32_t cells, uint32_t S, float *__restrict__ rho) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cells) return;
    double sum = 0.0, tw = 0.0;
    for (uint32_t s = 0; s < S; s++) {
        const double2 v = part[(size_t)c * S + s];
        sum += v.x;
        tw += v.y;
    }
    if (start[c] == kEmpty) tw += 1.0;
    if (tw < 1e-12) tw = 1e+24;
    rho[c] = (float)(sum / tw);
}

// GradDensity: periodic central differences, written as three planes.
__global__ void grad_density_kernel(const float *__restrict__ phi, uint32_t dim, double invh,
                                    float *__restrict__ grad) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t cells = dim * dim * dim;
    if (c >= cells) return;
    const uint32_t i = c % dim, j = (c / dim) % dim, k = c / (dim * dim);
    const uint32_t im = (i + dim - 1) % dim, ip = (i + 1) % dim;
    const uint32_t jm = (j + dim - 1) % dim, jp = (j + 1) % dim;
    const uint32_t km = (k + dim - 1) % dim, kp = (k + 1) % dim;
    const uint32_t sl = dim * dim;
    const double t = phi[k * sl + jp * dim + i], dn = phi[k * sl + jm * dim + i];
    const double l = phi[k * sl + j * dim + im], r = phi[k * sl + j * dim + ip];
    const double f = phi[km * sl + j * dim + i], b = phi[kp * sl + j * dim + i];
    grad[c] = (float)((r - l) * 0.5 * invh);
    grad[cells + c] = (float)((t - dn) * 0.5 * invh);
    grad[2 * (size_t)cells + c] = (float)((b - f) * 0.5 * invh);
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

// ParticleGetBaroclinic: hat-weighted grad rho over the 5^3 grid cells around
// the vortex's cell (only cells with a non-zero weight are read), crossed with
// (0, 10, 0), times dt_beta * 0.1, added to the strength.
__global__ void baroclinic_kernel(const float4 *__restrict__ cent, uint32_t N, const float *__restrict__ grad,
                                  uint32_t dim, double inv_h, double ox, double oy, double oz, double dt_beta,
                                  double *__restrict__ vx, double *__restrict__ vy, double *__restrict__ vz) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    const float4 p = cent[t];
    const float px = (float)((double)p.x - ox), py = (float)((double)p.y - oy), pz = (float)((double)p.z - oz);
    const double qx = (double)px * inv_h, qy = (double)py * inv_h, qz = (double)pz * inv_h;
    const int d = (int)dim;
    const int i = clamp_cell(floor(qx), d), j = clamp_cell(floor(qy), d), k = clamp_cell(floor(qz), d);
    double hx[5], hy[5], hz[5];
#pragma unroll
    for (int q = 0; q < 5; q++) {
        hx[q] = hat((double)(i - 2 + q) + 0.5 - qx);
        hy[q] = hat((double)(j - 2 + q) + 0.5 - qy);
        hz[q] = hat((double)(k - 2 + q) + 0.5 - qz);
    }
    const size_t cells = (size_t)dim * dim * dim;
    double sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll
    for (int c = 0; c < 5; c++) {
        const int kk = k - 2 + c;
        if (kk < 0 || kk >= d || hz[c] == 0.0) continue;
#pragma unroll
        for (int b = 0; b < 5; b++) {
            const int jj = j - 2 + b;
            if (jj < 0 || jj >= d || hy[b] == 0.0) continue;
#pragma unroll
            for (int a = 0; a < 5; a++) {
                const int ii = i - 2 + a;
                if (ii < 0 || ii >= d || hx[a] == 0.0) continue;
                const double w = hx[a] * hy[b] * hz[c];
                const size_t g = ((size_t)kk * dim + jj) * dim + ii;
                sx += (double)grad[g] * w;
                sy += (double)grad[cells + g] * w;
                sz += (double)grad[2 * cells + g] * w;
            }
        }
    }
    const double v0 = 0.0, v1 = 10.0, v2 = 0.0;
    const double bx = sy * v2 - sz * v1, by = sz * v0 - sx * v2, bz = sx * v1 - sy * v0;
    vx[t] += dt_beta * 0.1 * bx;
    vy[t] += dt_beta * 0.1 * by;
    vz[t] += dt_beta * 0.1 * bz;
}

template <typename T>
cudaError_t grow(T **p, size_t count) {
    cudaFree(*p);
    *p = nullptr;
    return ::pppm::device_malloc((void **)p, sizeof(T) * (count ? count : 1));
}

// Capacities are raised only once every buffer they cover exists; a failed
// growth leaves capacity 0 so that the next call allocates again.
cudaError_t ensure_heat(Buoyancy *b, uint32_t H) {
    if (H <= b->capH) return cudaSuccess;
    std::lock_guard<std::recursive_mutex> lk(device_lock());
    b->capH = 0;
    for (int q = 0; q < 2; q++) {
        PPPM_CUDA_TRY(grow(&b->key[q], H));
        PPPM_CUDA_TRY(grow(&b->idx[q], H));
    }
    PPPM_CUDA_TRY(grow(&b->hist, radix_hist_entries(H)));
    PPPM_CUDA_TRY(grow(&b->rec, H));
    b->capH = H;
    return cudaSuccess;
}

cudaError_t ensure_grid(Buoyancy *b, size_t cells, size_t parts) {
    std::lock_guard<std::recursive_mutex> lk(device_lock());
    if (cells > b->capC) {
        b->capC = 0;
        b->dim = 0;   // the last density grid went with the old buffers
        PPPM_CUDA_TRY(grow(&b->start, cells));
        PPPM_CUDA_TRY(grow(&b->end, cells));
        PPPM_CUDA_TRY(grow(&b->rho, cells));
        PPPM_CUDA_TRY(grow(&b->grad, 3 * cells));
        b->capC = cells;
    }
    if (parts > b->capPart) {
        b->capPart = 0;
        PPPM_CUDA_TRY(grow(&b->part, parts));
        b->capPart = parts;
    }
    return cudaSuccess;
}

}  // namespace

void free_buoyancy(Buoyancy *b) {
    if (!b) return;
    std::lock_guard<std::recursive_mutex> lk(device_lock());
    for (int q = 0; q < 2; q++) { cudaFree(b->key[q]); cudaFree(b->idx[q]); }
    cudaFree(b->hist);
    cudaFree(b->rec);
    cudaFree(b->bbox);
    cudaFree(b->start);
    cudaFree(b->end);
    cudaFree(b->rho);
    cudaFree(b->grad);
    cudaFree(b->part);
    if (b->host_bbox) cudaFreeHost(b->host_bbox);
    delete b;
}

}  // namespace pppm

extern "C" pppm_status pppm_baroclinic(pppm_scene *s, uint32_t H, const float *heat4, const float *heat,
                                       uint32_t N, const float *cent4, double *ax, double *ay, double *az,
                                       double dt) {
    using namespace pppm;
    if (!s || (H > 0 && (!heat4 || !heat)) || (N > 0 && (!cent4 || !ax || !ay || !az)) || !std::isfinite(dt)) {
        pppm_set_error("pppm_baroclinic: invalid argument");
        return PPPM_ERR_INVALID;
    }
    if (H == 0 || N == 0) return PPPM_OK;
    cudaStream_t st = s->stream;
    cudaError_t e = cudaSuccess;
    if (!s->buoy) {
        std::lock_guard<std::recursive_mutex> lk(device_lock());
        Buoyancy *nb = new Buoyancy;
        e = ::pppm::device_malloc((void **)&nb->bbox, sizeof(float) * 6 * kBBoxBlocks);
        if (e == cudaSuccess) e = ::pppm::host_malloc((void **)&nb->host_bbox, sizeof(float) * 6 * kBBoxBlocks);
        if (e == cudaSuccess) {
            s->buoy = nb;
        } else {
            free_buoyancy(nb);   // the next call starts over
            pppm_set_error("pppm_baroclinic (alloc): %s", cudaGetErrorString(e));
            return PPPM_ERR_OOM;
        }
    }
    Buoyancy *b = s->buoy;
    if (e == cudaSuccess) e = ensure_heat(b, H);
    if (e != cudaSuccess) {
        pppm_set_error("pppm_baroclinic (alloc): %s", cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? PPPM_ERR_OOM : PPPM_ERR_CUDA;
    }
    const float4 *hp = reinterpret_cast<const float4 *>(heat4);
    // setDensityDomain: the grid size depends on the box, so the box comes back
    // to the host once
    note_launch();
    heat_bbox_kernel<<<kBBoxBlocks, 256, 0, st>>>(hp, H, b->bbox);
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->host_bbox, b->bbox, sizeof(float) * 6 * kBBoxBlocks, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        pppm_set_error("pppm_baroclinic (bbox): %s", cudaGetErrorString(e));
        return PPPM_ERR_CUDA;
    }
    double mn[3], mx[3];
    for (int c = 0; c < 3; c++) {
        float lo = b->host_bbox[c * kBBoxBlocks], hi = b->host_bbox[(3 + c) * kBBoxBlocks];
        for (int q = 1; q < kBBoxBlocks; q++) {
            lo = fminf(lo, b->host_bbox[c * kBBoxBlocks + q]);
            hi = fmaxf(hi, b->host_bbox[(3 + c) * kBBoxBlocks + q]);
        }
        mn[c] = lo;
        mx[c] = hi;
    }
    const double L = 1.2 * std::max(std::max(mx[0] - mn[0], mx[1] - mn[1]), mx[2] - mn[2]);
    if (!(L > 0.0) || !std::isfinite(L)) return PPPM_OK;  // one point, or all coincident: no gradient
    double origin[3];
    for (int c = 0; c < 3; c++) origin[c] = (mn[c] + 0.5 * (mx[c] - mn[c])) - 0.5 * L;
    double h = 0.2;
    uint32_t dim = (uint32_t)(std::floor(L / h) + 1);
    dim = std::min(dim, (uint32_t)200);
    h = L / (double)dim;
    const float h_f = (float)(L / (double)dim);
    const float of[3] = {(float)origin[0], (float)origin[1], (float)origin[2]};
    const uint32_t cells = dim * dim * dim;
    // slices per cell: enough warps to fill the GPU when the grid is small
    uint32_t S = (uint32_t)std::min<uint64_t>(kMaxSplit, std::max<uint64_t>(1, (148ull * 32) / cells));
    e = ensure_grid(b, cells, S > 1 ? (size_t)cells * S : 0);
    if (e != cudaSuccess) {
        pppm_set_error("pppm_baroclinic (grid alloc): %s", cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? PPPM_ERR_OOM : PPPM_ERR_CUDA;
    }
    uint32_t *skey = nullptr, *sidx = nullptr;
    e = launch_explicit_hash(st, hp, H, h_f, of, dim, b->key, b->idx, b->hist, &skey, &sidx, b->start, b->end);
    if (e == cudaSuccess) {
        note_launch();
        heat_records_kernel<<<(H + 255) / 256, 256, 0, st>>>(hp, heat, sidx, H, origin[0], origin[1], origin[2],
                                                               b->rec);
        e = cudaGetLastError();
    }
    const double invh = 1.0 / h;
    if (e == cudaSuccess) {
        const uint64_t warps = (uint64_t)cells * S;
        const uint32_t blocks = (uint32_t)((warps * 32 + 255) / 256);
        note_launch();
        if (S == 1)
            assign_density_kernel<true><<<blocks, 256, 0, st>>>(b->start, b->end, b->rec, dim, 1, invh, b->rho,
                                                                nullptr);
        else
            assign_density_kernel<false><<<blocks, 256, 0, st>>>(b->start, b->end, b->rec, dim, S, invh, nullptr,
                                                                 b->part);
        e = cudaGetLastError();
        if (e == cudaSuccess && S > 1) {
            note_launch();
            density_finish_kernel<<<(cells + 255) / 256, 256, 0, st>>>(b->part, b->start, cells, S, b->rho);
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess) {
        note_launch();
        grad_density_kernel<<<(cells + 255) / 256, 256, 0, st>>>(b->rho, dim, invh, b->grad);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        note_launch();
        baroclinic_kernel<<<(N + 255) / 256, 256, 0, st>>>(reinterpret_cast<const float4 *>(cent4), N, b->grad,
                                                           dim, 1.0 / (double)h_f, origin[0], origin[1],
                                                           origin[2], dt * 5.0, ax, ay, az);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        pppm_set_error("pppm_baroclinic: %s", cudaGetErrorString(e));
        return PPPM_ERR_CUDA;
    }
    b->dim = dim;
    for (int c = 0; c < 3; c++) b->origin[c] = origin[c];
    b->h = h;
    return PPPM_OK;
}

extern "C" pppm_status pppm_get_density(pppm_scene *s, uint32_t *dim, double origin[3], double *h,
                                        const float **rho_dev, const float **grad_dev) {
    if (!s || !s->buoy || s->buoy->dim == 0) {
        pppm_set_error("pppm_get_density: no density grid built");
        return PPPM_ERR_STATE;
    }
    const pppm::Buoyancy *b = s->buoy;
    if (dim) *dim = b->dim;
    if (origin) for (int c = 0; c < 3; c++) origin[c] = b->origin[c];
    if (h) *h = b->h;
    if (rho_dev) *rho_dev = b->rho;
    if (grad_dev) *grad_dev = b->grad;
    return PPPM_OK;
}
