// One vortex-segment time step of the reference's VortexSimulationSystem
// (HFS/VortexSimulationSystemImp.cpp:90-125 solveTimeStep) for a system
// without solid boundary or shedding (the buoyancy source is pppm_baroclinic,
// called before the step as solveTimeStep calls addBaroclinicForce):
//
//   convertVortToSeg   each blob becomes a segment through its centre along
//                      its strength, of length min(|alpha|, h_seg)
//                      (ComputePosb, HFS/GPU_kernel.cu:3184-3229)
//   computeURotation   far field of the blobs, then the velocity at both
//                      segment ends with the centre as the other end, and at
//                      the passive points (tracers, heat particles), which
//                      move with it (HFS/VortexSimulationSystemImp.cpp:142-228,
//                      evaluateBiotSavart :1195-1244)
//   applyFlow          both ends move, the centre is their midpoint
//                      (move_particle / ComputePosa, HFS/GPU_kernel.cu:3118-3254)
//   convertSegToVort   dalpha = kappa * (endb - enda) - alpha
//                      (ComputeVortex, HFS/GPU_kernel.cu:3143-3180)
//   computeStretching  alpha + dalpha is smoothed with a Gaussian of width nu
//                      over the 5^3 hash cells around each centre
//                      (HFS/VortexSimulationSystemImp.cpp:466-525,
//                      ParticleGaussianSmooth HFS/GPU_kernel.cu:3327-3438)
//
// The two end evaluations run as one launch over 2N points.  The segment
// conversion, the move, the midpoint and the strength update are fused into
// two elementwise kernels.  The smoothing walks the vortices in hash order, a
// warp at a time, staging 32 records of a cell in shared memory as 16 record
// pairs that Blackwell's packed f32x2 instructions process two at a time, in
// coordinates scaled so that the squared distance is the exponent of 2^x, and
// sums the weights in FP32 per staged chunk and in FP64 across chunks.
#include <cmath>

#include "pppm_internal.cuh"

namespace pppm {
namespace {

constexpr int kSmoothThreads = 128;
// A warp walks the union of its lanes' 5^3 boxes when that union holds at most
// this many cells; otherwise (sparse vortices) each lane walks its own box.
constexpr int kSmoothUnionMax = 250;

// ComputePosb: endb = c + s/2, enda = c - s/2 with s = alpha capped to length
// h_seg; kappa = max(|alpha| / h_seg, 1).  ends[0, N) = endb, ends[N, 2N) =
// enda; other[] holds the centre for both halves (the segment's other end).
__global__ void segment_kernel(const float4 *__restrict__ cent, const double *__restrict__ alpha, size_t stride,
                               double h_seg, uint32_t N, float4 *__restrict__ ends, float4 *__restrict__ other,
                               double *__restrict__ kappa) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    const float4 c = cent[t];
    const double sx = alpha[t], sy = alpha[stride + t], sz = alpha[2 * stride + t];
    const double l = sqrt(sx * sx + sy * sy + sz * sz);
    float4 b = c, a = c;
    double k;
    if (l < h_seg) {
        k = 1.0;
        b.x = (float)(c.x + 0.5 * sx); b.y = (float)(c.y + 0.5 * sy); b.z = (float)(c.z + 0.5 * sz);
        a.x = (float)(c.x - 0.5 * sx); a.y = (float)(c.y - 0.5 * sy); a.z = (float)(c.z - 0.5 * sz);
    } else {
        k = l / h_seg;
        b.x = (float)(c.x + 0.5 * sx / l * h_seg);
        b.y = (float)(c.y + 0.5 * sy / l * h_seg);
        b.z = (float)(c.z + 0.5 * sz / l * h_seg);
        a.x = (float)(c.x - 0.5 * sx / l * h_seg);
        a.y = (float)(c.y - 0.5 * sy / l * h_seg);
        a.z = (float)(c.z - 0.5 * sz / l * h_seg);
    }
    ends[t] = b;
    ends[N + t] = a;
    other[t] = c;
    other[N + t] = c;
    kappa[t] = k;
}

__device__ __forceinline__ float4 moved(float4 p, double ux, double uy, double uz, double dt) {
    const double x = (double)p.x + ux * dt;
    const double y = (double)p.y + uy * dt;
    const double z = (double)p.z + uz * dt;
    return make_float4((float)x, (float)y, (float)z, 0.0f);
}

// applyFlow + convertSegToVort + the first VectorAdd of computeStretching:
// both ends move with their velocities (u[0, N) at endb, u[N, 2N) at enda),
// the centre becomes their midpoint (w kept), and the scene's strength copy
// becomes alpha + (kappa * (endb - enda) - alpha).
__global__ void segment_to_blob_kernel(const float4 *__restrict__ ends, const double *__restrict__ u, size_t ustride,
                                       const double *__restrict__ kappa, double dt, uint32_t N,
                                       float4 *__restrict__ cent, float4 *__restrict__ vpos,
                                       double *__restrict__ alpha, size_t astride, float4 *__restrict__ enda_out,
                                       float4 *__restrict__ endb_out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    const float4 b = moved(ends[t], u[t], u[ustride + t], u[2 * ustride + t], dt);
    const float4 a = moved(ends[N + t], u[N + t], u[ustride + N + t], u[2 * ustride + N + t], dt);
    float4 c = cent[t];
    c.x = (float)(0.5 * (double)(b.x + a.x));
    c.y = (float)(0.5 * (double)(b.y + a.y));
    c.z = (float)(0.5 * (double)(b.z + a.z));
    cent[t] = c;
    vpos[t] = c;
    const double k = kappa[t];
    const double s[3] = {(double)(b.x - a.x), (double)(b.y - a.y), (double)(b.z - a.z)};
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const double v = alpha[q * astride + t];
        const double d = k * s[q] - v;
        alpha[q * astride + t] = 1.0 * v + 1.0 * d;
    }
    if (enda_out) enda_out[t] = a;
    if (endb_out) endb_out[t] = b;
}

// move_particle (HFS/GPU_kernel.cu:3118-3140) with the velocity in three arrays.
__global__ void move3_kernel(float4 *__restrict__ pos, const double *__restrict__ u, const double *__restrict__ v,
                             const double *__restrict__ w, double dt, uint32_t N) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    pos[t] = moved(pos[t], u[t], v[t], w[t], dt);
}

// 2^x by the MUFU.EX2 instruction (PTX ex2.approx.ftz.f32, relative error about
// 2^-22; results below 2^-126 flush to zero, weights negligible beside the
// vortex's own weight 1).
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Shared staging of a chunk of 32 records as 16 pairs: slot p holds records
// 2p (.x, .z halves) and 2p+1 (.y, .w halves).  Planes: {-x, -y}, {-z, ax},
// {ay, az}.
constexpr int kSlots = 16;
__device__ __forceinline__ void stage_pair(float *__restrict__ pk, int slot, int half, float nx, float ny, float nz,
                                           float ax, float ay, float az) {
    float *A = pk + 4 * slot, *B = pk + 4 * (kSlots + slot), *Cc = pk + 4 * (2 * kSlots + slot);
    A[half] = nx; A[2 + half] = ny;
    B[half] = nz; B[2 + half] = ax;
    Cc[half] = ay; Cc[2 + half] = az;
}

__device__ __forceinline__ int clamp_cell(double q, int n) {
    // cells more than two outside the grid see no in-grid cell: any value past
    // that behaves the same, so clamp before converting to int
    if (!(q >= -3.0)) return -3;
    if (q > (double)(n + 2)) return n + 2;
    return (int)q;
}

// ParticleGaussianSmooth over the hash-sorted vortices.  Lane t (sorted slot)
// finds its NGP cell (i, j, k) from the FP64 origin as the reference does,
// then sums exp(-|x_p - x_t|^2 / (2 nu^2)) and that weight times the strength
// over every vortex p hashed into cells [i-2, i+2] x [j-2, j+2] x [k-2, k+2]
// inside the grid.  The result, divided by the weight sum (1e24 when that sum
// is below 1e-12), replaces the strength: out = 0 * out_old + smoothed.
__global__ void __launch_bounds__(kSmoothThreads) gaussian_smooth_kernel(
    const float4 *__restrict__ vrec, const float4 *__restrict__ valf, const uint32_t *__restrict__ sidx,
    const uint32_t *__restrict__ cstart, const uint32_t *__restrict__ cend, const DevParams *__restrict__ P,
    float wscale, uint32_t N, double *__restrict__ ox, double *__restrict__ oy, double *__restrict__ oz) {
    __shared__ float4 s_pk[(kSmoothThreads / 32) * 3 * kSlots];
    const int lane = threadIdx.x & 31;
    const int wbase = threadIdx.x & ~31;
    const int wpk = (threadIdx.x >> 5) * 3 * kSlots;
    const uint32_t t0 = (blockIdx.x * blockDim.x) + wbase;
    if (t0 >= N) return;
    const uint32_t t = t0 + lane;
    const bool live = t < N;
    const int n = (int)P->n;
    const double invh = P->invh;
    float3 ra = make_float3(0.f, 0.f, 0.f);
    int ci = 0, cj = 0, ck = 0;
    if (live) {
        const float4 r = vrec[t];
        ra = make_float3(r.x, r.y, r.z);
        ci = clamp_cell(floor((double)r.x * invh), n);
        cj = clamp_cell(floor((double)r.y * invh), n);
        ck = clamp_cell(floor((double)r.z * invh), n);
    }
    // idle lanes of the last warp copy lane 0 (always live) so the union stays
    // tight; every lane takes part in the shuffles
    {
        const int i0 = __shfl_sync(0xffffffffu, ci, 0);
        const int j0 = __shfl_sync(0xffffffffu, cj, 0);
        const int k0 = __shfl_sync(0xffffffffu, ck, 0);
        if (!live) { ci = i0; cj = j0; ck = k0; }
    }
    const int xlo = max(__reduce_min_sync(0xffffffffu, ci) - 2, 0);
    const int xhi = min(__reduce_max_sync(0xffffffffu, ci) + 2, n - 1);
    const int ylo = max(__reduce_min_sync(0xffffffffu, cj) - 2, 0);
    const int yhi = min(__reduce_max_sync(0xffffffffu, cj) + 2, n - 1);
    const int zlo = max(__reduce_min_sync(0xffffffffu, ck) - 2, 0);
    const int zhi = min(__reduce_max_sync(0xffffffffu, ck) + 2, n - 1);

    double tw = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
    // the staged walk works in coordinates scaled by sg = sqrt(-wscale), so
    // that the squared scaled distance is the (negated) exponent itself
    const float sg = sqrtf(-wscale);
    const float2 tx = make_float2(ra.x * sg, ra.x * sg), ty = make_float2(ra.y * sg, ra.y * sg),
                 tz = make_float2(ra.z * sg, ra.z * sg);
    auto walk = [&](int x0, int x1, int y0, int y1, int z0, int z1, bool member) {
        for (int z = z0; z <= z1; z++)
            for (int y = y0; y <= y1; y++)
                for (int x = x0; x <= x1; x++) {
                    const uint32_t c = ((uint32_t)z * (uint32_t)n + (uint32_t)y) * (uint32_t)n + (uint32_t)x;
                    const uint32_t s0 = cstart[c];
                    if (s0 == kEmpty) continue;
                    const uint32_t s1 = cend[c];
                    const bool ok = member && abs(x - ci) <= 2 && abs(y - cj) <= 2 && abs(z - ck) <= 2;
                    if (!__any_sync(0xffffffffu, ok)) continue;
                    for (uint32_t base = s0; base < s1; base += 32) {
                        const uint32_t cnt = min(32u, s1 - base);
                        // stage the chunk as 16 record pairs (records 2p, 2p+1 in
                        // the .x / .y halves) for packed f32x2 arithmetic; an odd
                        // chunk is padded with a record at 1e18 and zero strength
                        float *pk = reinterpret_cast<float *>(s_pk + wpk);
                        if ((uint32_t)lane < cnt) {
                            const float4 b = vrec[base + lane];
                            const float4 al = valf[base + lane];
                            stage_pair(pk, lane >> 1, lane & 1, -b.x * sg, -b.y * sg, -b.z * sg, al.x, al.y, al.z);
                        } else if ((uint32_t)lane == cnt && (cnt & 1u)) {
                            stage_pair(pk, lane >> 1, 1, 1e18f, 1e18f, 1e18f, 0.f, 0.f, 0.f);
                        }
                        __syncwarp();
                        if (ok) {
                            float2 pw = make_float2(0.f, 0.f), px = pw, py = pw, pz = pw;
                            const uint32_t np = (cnt + 1) >> 1;
#pragma unroll 4
                            for (uint32_t p = 0; p < np; p++) {
                                const float4 A = s_pk[wpk + p], B = s_pk[wpk + kSlots + p];
                                const float4 Cc = s_pk[wpk + 2 * kSlots + p];
                                const float2 dx = __fadd2_rn(tx, make_float2(A.x, A.y));
                                const float2 dy = __fadd2_rn(ty, make_float2(A.z, A.w));
                                const float2 dz = __fadd2_rn(tz, make_float2(B.x, B.y));
                                const float2 dsq = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
                                const float2 w = make_float2(ex2_approx(-dsq.x), ex2_approx(-dsq.y));
                                pw = __fadd2_rn(pw, w);
                                px = __ffma2_rn(w, make_float2(B.z, B.w), px);
                                py = __ffma2_rn(w, make_float2(Cc.x, Cc.y), py);
                                pz = __ffma2_rn(w, make_float2(Cc.z, Cc.w), pz);
                            }
                            tw += (double)pw.x + (double)pw.y;
                            wx += (double)px.x + (double)px.y;
                            wy += (double)py.x + (double)py.y;
                            wz += (double)pz.x + (double)pz.y;
                        }
                        __syncwarp();
                    }
                }
    };

    if (xlo <= xhi && ylo <= yhi && zlo <= zhi) {
        const int vol = (xhi - xlo + 1) * (yhi - ylo + 1) * (zhi - zlo + 1);
        if (vol <= kSmoothUnionMax) {
            walk(xlo, xhi, ylo, yhi, zlo, zhi, live);
        } else if (live) {
            // sparse warp (its lanes' boxes far apart): each lane walks its own
            // 5^3 box with the same arithmetic, one record at a time
            for (int z = max(ck - 2, 0); z <= min(ck + 2, n - 1); z++)
                for (int y = max(cj - 2, 0); y <= min(cj + 2, n - 1); y++)
                    for (int x = max(ci - 2, 0); x <= min(ci + 2, n - 1); x++) {
                        const uint32_t c = ((uint32_t)z * (uint32_t)n + (uint32_t)y) * (uint32_t)n + (uint32_t)x;
                        const uint32_t s0 = cstart[c];
                        if (s0 == kEmpty) continue;
                        const uint32_t s1 = cend[c];
                        float pw = 0.f, px = 0.f, py = 0.f, pz = 0.f;
                        for (uint32_t p = s0; p < s1; p++) {
                            const float4 b = vrec[p];
                            const float4 al = valf[p];
                            const float dx = ra.x + (-b.x), dy = ra.y + (-b.y), dz = ra.z + (-b.z);
                            const float dsq = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                            const float w = ex2_approx(dsq * wscale);
                            pw += w;
                            px = fmaf(w, al.x, px);
                            py = fmaf(w, al.y, py);
                            pz = fmaf(w, al.z, pz);
                        }
                        tw += (double)pw;
                        wx += (double)px;
                        wy += (double)py;
                        wz += (double)pz;
                    }
        }
    }
    if (!live) return;
    if (tw < 1e-12) tw = 1e+24;
    const uint32_t q = sidx[t];
    ox[q] = 0.0 * ox[q] + 1.0 * (wx / tw);
    oy[q] = 0.0 * oy[q] + 1.0 * (wy / tw);
    oz[q] = 0.0 * oz[q] + 1.0 * (wz / tw);
}

}  // namespace

cudaError_t launch_segments(pppm_scene *s, double h_seg, uint32_t N, float4 *ends, float4 *other, double *kappa) {
    ::pppm::note_launch();
    segment_kernel<<<(N + 255) / 256, 256, 0, s->stream>>>(s->vpos, s->valpha, s->capN, h_seg, N, ends, other,
                                                           kappa);
    return cudaGetLastError();
}

cudaError_t launch_segment_to_blob(pppm_scene *s, const float4 *ends, const double *u, size_t ustride,
                                   const double *kappa, double dt, uint32_t N, float4 *cent, float4 *enda_out,
                                   float4 *endb_out) {
    ::pppm::note_launch();
    segment_to_blob_kernel<<<(N + 255) / 256, 256, 0, s->stream>>>(ends, u, ustride, kappa, dt, N, cent, s->vpos,
                                                                   s->valpha, s->capN, enda_out, endb_out);
    return cudaGetLastError();
}

cudaError_t launch_move3(pppm_scene *s, float4 *pos, const double *u, const double *v, const double *w, double dt,
                         uint32_t N) {
    ::pppm::note_launch();
    move3_kernel<<<(N + 255) / 256, 256, 0, s->stream>>>(pos, u, v, w, dt, N);
    return cudaGetLastError();
}

cudaError_t launch_gaussian_smooth(pppm_scene *s, double nu, uint32_t N, double *ox, double *oy, double *oz) {
    // exp(-d^2 / (2 nu^2)) = 2^(d^2 * wscale)
    const float wscale = (float)(-1.0 / (2.0 * nu * nu * std::log(2.0)));
    ::pppm::note_launch();
    const uint32_t blocks = (uint32_t)(((uint64_t)N + kSmoothThreads - 1) / kSmoothThreads);
    gaussian_smooth_kernel<<<blocks, kSmoothThreads, 0, s->stream>>>(s->vrec, s->valf, s->vsorted_idx,
                                                                     s->cell_start, s->cell_end, s->dparams, wscale,
                                                                     N, ox, oy, oz);
    return cudaGetLastError();
}

}  // namespace pppm
