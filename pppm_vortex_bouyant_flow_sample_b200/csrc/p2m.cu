// Particle-to-mesh vorticity spreading (HFS/GPU_kernel.cu:218-294 with the
// nearest-grid-point weight of :31-50, then ComputeRHS :524-543 called with
// G = -1 at HFS/BiotSavartSolverImp.cpp:552-559).
//
// The reference gathers, for every grid cell, over the 5^3 hash cells around
// it and keeps the particles whose NGP cell is that cell.  Here the vortices
// are already sorted by hash cell, so a cell's particles are one contiguous
// run: one warp takes 32 consecutive cells, walks the non-empty runs with
// coalesced loads, reduces with a fixed xor-butterfly (deterministic, no
// atomics), and the owning lane writes the cell.  A particle whose FP64 NGP
// cell differs from its FP32 hash cell (a rounding tie at a cell face) has
// flagged its NGP cell; only flagged cells also walk their 26 neighbouring
// runs, which is the exact set the reference's 5^3 window can reach.
#include "pppm_internal.cuh"

namespace pppm {

namespace {

constexpr int kP2MThreads = 256;

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ void run_sum(const float4 *__restrict__ vrec, const float4 *__restrict__ valf,
                                        uint32_t s, uint32_t e, uint32_t cell, int lane, float &ax, float &ay,
                                        float &az) {
    // unrolled so that a dense cell's loads are in flight together (each
    // lane's records are still added in order)
#pragma unroll 4
    for (uint32_t p = s + lane; p < e; p += 32) {
        const float4 r = vrec[p];
        if (__float_as_uint(r.w) == cell) {
            const float4 a = valf[p];
            ax += a.x;
            ay += a.y;
            az += a.z;
        }
    }
}

__global__ void __launch_bounds__(kP2MThreads)
p2m_kernel(const uint32_t *__restrict__ start, const uint32_t *__restrict__ end,
           const float4 *__restrict__ vrec, const float4 *__restrict__ valf, const uint32_t *__restrict__ mflag,
           uint32_t epoch, const DevParams *__restrict__ P, uint32_t n, float *__restrict__ vort,
           float *__restrict__ rhs) {
    const uint32_t C = n * n * n;
    const int lane = threadIdx.x & 31;
    const uint32_t cell = (blockIdx.x * blockDim.x + threadIdx.x);
    const uint32_t wbase = cell - lane;
    if (wbase >= C) return;
    const bool inb = cell < C;
    const uint32_t s = inb ? start[cell] : kEmpty;
    const uint32_t e = inb ? end[cell] : kEmpty;
    const bool flagged = inb && mflag[cell] == epoch;
    float ox = 0.f, oy = 0.f, oz = 0.f;  // this lane's cell
    uint32_t busy = __ballot_sync(0xffffffffu, s != kEmpty);
    while (busy) {
        const int b = __ffs(busy) - 1;
        busy &= busy - 1;
        const uint32_t cs = __shfl_sync(0xffffffffu, s, b);
        const uint32_t ce = __shfl_sync(0xffffffffu, e, b);
        float ax = 0.f, ay = 0.f, az = 0.f;
        run_sum(vrec, valf, cs, ce, wbase + b, lane, ax, ay, az);
        ax = warp_sum(ax);
        ay = warp_sum(ay);
        az = warp_sum(az);
        if (lane == b) { ox = ax; oy = ay; oz = az; }
    }
    uint32_t fl = __ballot_sync(0xffffffffu, flagged);
    while (fl) {
        const int b = __ffs(fl) - 1;
        fl &= fl - 1;
        const uint32_t c = wbase + b;
        const int ci = (int)(c % n), cj = (int)((c / n) % n), ck = (int)(c / (n * n));
        float ax = 0.f, ay = 0.f, az = 0.f;
        for (int dk = -1; dk <= 1; dk++)
            for (int dj = -1; dj <= 1; dj++)
                for (int di = -1; di <= 1; di++) {
                    if (!di && !dj && !dk) continue;
                    const int ii = ci + di, jj = cj + dj, kk = ck + dk;
                    if (ii < 0 || jj < 0 || kk < 0 || ii >= (int)n || jj >= (int)n || kk >= (int)n) continue;
                    const uint32_t nb = ((uint32_t)kk * n + (uint32_t)jj) * n + (uint32_t)ii;
                    const uint32_t ns = start[nb];
                    if (ns == kEmpty) continue;
                    run_sum(vrec, valf, ns, end[nb], c, lane, ax, ay, az);
                }
        ax = warp_sum(ax);
        ay = warp_sum(ay);
        az = warp_sum(az);
        if (lane == b) { ox += ax; oy += ay; oz += az; }
    }
    if (inb) {
        const float s3 = P->invh3_f, h2 = P->h2f;
        const float wx = ox * s3, wy = oy * s3, wz = oz * s3;
        vort[cell] = wx;
        vort[C + cell] = wy;
        vort[2 * (size_t)C + cell] = wz;
        rhs[cell] = -(wx * h2);
        rhs[C + cell] = -(wy * h2);
        rhs[2 * (size_t)C + cell] = -(wz * h2);
    }
}

}  // namespace

cudaError_t launch_p2m(pppm_scene *s) {
    const unsigned blocks = (s->C + kP2MThreads - 1) / kP2MThreads;
    ::pppm::note_launch();
    p2m_kernel<<<blocks, kP2MThreads, 0, s->stream>>>(s->cell_start, s->cell_end, s->vrec, s->valf, s->mflag,
                                                      s->epoch, s->dparams, s->n, s->vort, s->lv[0].b);
    return cudaGetLastError();
}

}  // namespace pppm
