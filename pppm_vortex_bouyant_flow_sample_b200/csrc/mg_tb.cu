// Temporally blocked red-black SOR smoother for the multigrid levels that
// stream from HBM (edge >= 256; opt-in through PPPM_MG_TB, since the plain
// half sweeps on groups of 4 cells measured faster inside a whole solve):
// T half sweeps — T/2 of the
// reference's red-black iterations (MG/Multigrid.cu:202-239, odd cells first,
// omega = 1.43f) — in one pass over the level, optionally fused with the
// prolongation by injection that precedes the post-smoothing
// (MG/MultiGrid_kernel.cu, mg_ProlongationPeriodic3D2).
//
// Each CTA owns an output tile of TX x TY cells in (x, y) and a chunk of z
// planes.  It streams planes of x and b through a ring of T + 2 + PF slots (PF planes loaded ahead) in
// shared memory, each slot a (TX + 2H) x (TY + 2T) box loaded by one TMA
// tensor copy (cp.async.bulk.tensor.4d, completion on an mbarrier; H = T
// rounded up to 4 so that the box's x coordinate stays 16-byte aligned).  The
// box's cells beyond the grid arrive as zeros (the tensor map's out-of-bounds
// fill), which are exactly the zero ghost values of the reference's operator;
// they are never updated.  At step s, half sweep t (colour 1 for odd t, 0 for
// even t) updates plane s - t + 1 in the box shrunk by t cells on each side,
// in place: a half sweep reads only the other colour, which the previous half
// sweep of the same plane and its two neighbours left final.  Plane s - T + 1
// is then final and its TX x TY interior is stored with 128-bit stores into a
// second array (x_out != x_in: the boxes of neighbouring tiles overlap).  A
// z-chunk starts T planes early and ends T planes late, updating a plane at
// half sweep t only where its whole dependency cone lies inside the chunk's
// loaded planes, so the stored planes equal T plain half sweeps bit for bit.
//
// Every wait on an mbarrier is bounded; on running out the kernel records
// kTbErrTimeout in *err, waits (again bounded) for its copies in flight and
// returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstring>

#include "pppm_internal.cuh"

namespace pppm {

namespace {

constexpr float kOmegaF = 1.43f;
constexpr float kOneMinusOmegaF = 1.0f - 1.43f;  // formed in float, MG/MultiGrid_kernel.cu:766
constexpr uint32_t kWaitLimit = 1u << 22;         // polls of one mbarrier phase (each poll itself blocks a while)

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// One 4-D tiled tensor copy global -> shared (no multicast), completing on bar.
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ float sor(float x, float nb, float b) {
    const float r = nb - b;
    return kOneMinusOmegaF * x + (kOmegaF * r) * (1.0f / 6.0f);
}

}  // namespace

// Shared-memory bytes of one configuration (ring of x, and of b unless BG,
// plus barriers).  PF: planes loaded ahead of the one a step needs (copies in
// flight).  BG: b is read from global memory where a cell is updated instead
// of being staged (each b value is read once per pass either way).
template <int T, int TX, int TY, int PF, bool BG>
struct TbShape {
    static constexpr int H = (T + 3) / 4 * 4;  // x halo, a multiple of 4 floats
    static constexpr int BX = TX + 2 * H;
    static constexpr int BY = TY + 2 * T;
    static constexpr int R = T + 2 + PF;
    static constexpr int PLANE = BX * BY;                    // floats per slot
    static constexpr uint32_t PLANE_BYTES = PLANE * 4u;
    static constexpr size_t SMEM = (BG ? 1ull : 2ull) * R * PLANE_BYTES + 8ull * R + 128;
    static_assert(PLANE_BYTES % 128 == 0, "slots must stay 128-byte aligned");
    static_assert(BX <= 256 && BY <= 256, "TMA box edge above 256");
    static_assert(T % 2 == 0, "whole red-black iterations only");
};

// G4: a thread takes a group of 4 consecutive cells of a row (a 16-byte word of
// the slot) and, in a half sweep, updates the 2 of them that have the sweep's
// colour, reading its own row, the rows above and below and the planes before
// and after with 128-bit shared loads (conflict free) plus one scalar either
// side; the group is written back whole, the other colour's cells with the
// values just read (no other thread writes them in that half sweep, and the
// half sweep's readers of them read the same value either way).  Otherwise a
// thread takes a pair of cells and updates the one of the sweep's colour.
template <int T, int TX, int TY, int NT, int PF, bool BG, bool G4>
__global__ void __launch_bounds__(NT)
tb_smooth_kernel(const __grid_constant__ CUtensorMap map_x, const __grid_constant__ CUtensorMap map_b,
                 int load_x, const float *__restrict__ xc, float *__restrict__ x_out, int d, int zchunk,
                 int zchunks, uint32_t *__restrict__ err, const float *__restrict__ bg) {
    using S = TbShape<T, TX, TY, PF, BG>;
    constexpr int H = S::H, BX = S::BX, BY = S::BY, R = S::R, PLANE = S::PLANE;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    float *ring_x = reinterpret_cast<float *>(smem_raw);
    float *ring_b = ring_x + R * PLANE;  // (BG: no b ring)
    uint64_t *bars = reinterpret_cast<uint64_t *>(ring_x + (BG ? 1 : 2) * R * PLANE);
    const float *bgc = BG ? bg + (size_t)(blockIdx.z / zchunks) * d * d * d : nullptr;
    __shared__ int s_abort;
    __shared__ uint32_t s_issued[R];  // loads issued per slot (thread 0)

    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int comp = blockIdx.z / zchunks, chunk = blockIdx.z % zchunks;
    const int zc0 = chunk * zchunk, zc1 = min(d, zc0 + zchunk);
    const int p_first = zc0 - T, p_last = zc1 + T - 1;
    const size_t cells = (size_t)d * d * d;
    const int dc = d >> 1;
    const float *xcc = xc ? xc + (size_t)comp * dc * dc * dc : nullptr;
    float *xo = x_out + (size_t)comp * cells;

    if (tid == 0) {
        for (int r = 0; r < R; r++) {
            mbar_init(&bars[r], 1);
            s_issued[r] = 0;
        }
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // this thread's (row, pair) or (row, group of 4) slots of the box, the same
    // for every half sweep
    static_assert(!G4 || (!BG && BX % 4 == 0), "groups of 4 need b in the ring and whole words");
    constexpr int PAIRS = G4 ? BX / 4 : BX / 2;
    constexpr int ITEMS = (BY * PAIRS + NT - 1) / NT;
    int it_sy[ITEMS], it_px[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
        const int q = tid + i * NT;
        it_sy[i] = (q < BY * PAIRS) ? q / PAIRS : -1;
        it_px[i] = q % PAIRS;
    }

    const uint32_t tx_bytes = ((load_x ? 1u : 0u) + (BG ? 0u : 1u)) * S::PLANE_BYTES;
    auto slot_of = [&](int p) { return (p - p_first) % R; };
    auto issue = [&](int p) {  // thread 0 only
        const int sl = slot_of(p);
        s_issued[sl]++;
        mbar_expect_tx(&bars[sl], tx_bytes);
        if (load_x) tma_load_4d(ring_x + sl * PLANE, &map_x, x0 - H, y0 - T, p, comp, &bars[sl]);
        if (!BG) tma_load_4d(ring_b + sl * PLANE, &map_b, x0 - H, y0 - T, p, comp, &bars[sl]);
    };
    // Waits for plane p, then applies the start value: x as loaded, zero
    // (load_x = 0), plus the injected coarse correction xc[parent] (xc set);
    // cells outside the grid stay zero.
    auto wait_prep = [&](int p) -> bool {
        const int sl = slot_of(p);
        const uint32_t parity = (uint32_t)((p - p_first) / R) & 1u;
        uint32_t it = 0;
        while (!mbar_try_wait(&bars[sl], parity)) {
            if (++it > kWaitLimit) {
                atomicExch(err, kTbErrTimeout);
                s_abort = 1;
                break;
            }
        }
        if (load_x && !xcc) return true;
        float *X = ring_x + sl * PLANE;
        const bool zin = (p >= 0 && p < d);
        for (int q = tid; q < PLANE; q += NT) {
            const int gy = y0 - T + q / BX, gx = x0 - H + q % BX;
            float v = load_x ? X[q] : 0.0f;
            if (xcc && zin && gx >= 0 && gx < d && gy >= 0 && gy < d)
                v += xcc[((size_t)(p >> 1) * dc + (gy >> 1)) * dc + (gx >> 1)];
            X[q] = v;
        }
        return true;
    };

    const bool prep = !(load_x && !xcc);  // the start value is written by the threads
    if (tid == 0) {
        for (int p = p_first; p <= min(p_first + 1 + PF, p_last); p++) issue(p);
    }
    wait_prep(p_first);
    wait_prep(p_first + 1);
    fence_proxy_async();
    __syncthreads();

    const int s_begin = zc0 - T + 1, s_end = zc1 + T - 2;
    for (int s = s_begin; s <= s_end; s++) {
        // The slot refilled now held plane s - T - 1, whose last reads and
        // writes (half sweep T of the step before) every thread ordered before
        // the asynchronous proxy (fence) and the barrier that closed that step.
        if (tid == 0 && s + 1 + PF <= p_last) issue(s + 1 + PF);
        wait_prep(s + 1);
        if (prep) __syncthreads();
#pragma unroll
        for (int t = 1; t <= T; t++) {
            const int p = s - t + 1;
            if (p >= max(0, zc0 - T + t) && p < min(d, zc1 + T - t)) {
                const int c = t & 1;  // odd half sweeps: colour 1 (odd cells) first
                float *X = ring_x + slot_of(p) * PLANE;
                const float *Xm = ring_x + slot_of(p - 1) * PLANE;
                const float *Xp = ring_x + slot_of(p + 1) * PLANE;
                const float *B = BG ? nullptr : ring_b + slot_of(p) * PLANE;
                const float *Bg = BG ? bgc + (size_t)p * d * d : nullptr;
                const int ya = max(0, y0 - T + t), yb = min(d, y0 + TY + T - t);
                const int xa = max(0, x0 - T + t), xb = min(d, x0 + TX + T - t);
                if constexpr (G4) {
#pragma unroll
                    for (int i = 0; i < ITEMS; i++) {
                        const int sy = it_sy[i];
                        const int gy = y0 - T + sy;
                        // rows outside [ya, yb) include the box's first and
                        // last, so the rows above and below stay in the slot
                        if (sy < 0 || gy < ya || gy >= yb) continue;
                        const int sx = 4 * it_px[i];
                        const int gx = x0 - H + sx;  // a multiple of 4
                        const int a = (c - gy - p) & 1;  // the colour's cells: sx + a, sx + a + 2
                        const bool m_lo = gx + a >= xa && gx + a < xb;
                        const bool m_hi = gx + a + 2 >= xa && gx + a + 2 < xb;
                        if (!m_lo && !m_hi) continue;
                        const int o = sy * BX + sx;
                        const float4 v = *reinterpret_cast<const float4 *>(X + o);
                        const float4 un = *reinterpret_cast<const float4 *>(X + o + BX);
                        const float4 dn = *reinterpret_cast<const float4 *>(X + o - BX);
                        const float4 zm = *reinterpret_cast<const float4 *>(Xm + o);
                        const float4 zp = *reinterpret_cast<const float4 *>(Xp + o);
                        const float4 bb = *reinterpret_cast<const float4 *>(B + o);
                        const float xl = sx > 0 ? X[o - 1] : 0.0f;
                        const float xr = sx + 4 < BX ? X[o + 4] : 0.0f;
                        const bool odd = a != 0;
                        // the same sums in the same order as one cell of the
                        // pair mapping (left + right) + (y+1 + y-1) + (z-1 + z+1)
                        const float nb_lo = (((odd ? v.x : xl) + (odd ? v.z : v.y)) + ((odd ? un.y : un.x) + (odd ? dn.y : dn.x))) +
                                            ((odd ? zm.y : zm.x) + (odd ? zp.y : zp.x));
                        const float nb_hi = (((odd ? v.z : v.y) + (odd ? xr : v.w)) + ((odd ? un.w : un.z) + (odd ? dn.w : dn.z))) +
                                            ((odd ? zm.w : zm.z) + (odd ? zp.w : zp.z));
                        const float n_lo = sor(odd ? v.y : v.x, nb_lo, odd ? bb.y : bb.x);
                        const float n_hi = sor(odd ? v.w : v.z, nb_hi, odd ? bb.w : bb.z);
                        float4 w = v;
                        if (odd) {
                            if (m_lo) w.y = n_lo;
                            if (m_hi) w.w = n_hi;
                        } else {
                            if (m_lo) w.x = n_lo;
                            if (m_hi) w.z = n_hi;
                        }
                        *reinterpret_cast<float4 *>(X + o) = w;
                    }
                } else {
#pragma unroll
                for (int i = 0; i < ITEMS; i++) {
                    const int sy = it_sy[i];
                    const int gy = y0 - T + sy;
                    // box x origin x0 - H is even, so box and grid parities agree
                    const int sx = 2 * it_px[i] + ((c - gy - p) & 1);
                    const int gx = x0 - H + sx;
                    if (sy < 0 || gy < ya || gy >= yb || gx < xa || gx >= xb) continue;
                    const int o = sy * BX + sx;
                    const float nb = ((X[o - 1] + X[o + 1]) + (X[o + BX] + X[o - BX])) + (Xm[o] + Xp[o]);
                    X[o] = sor(X[o], nb, BG ? __ldg(Bg + (size_t)gy * d + gx) : B[o]);
                }
                }
            }
            if (t == T) fence_proxy_async();
            __syncthreads();
            if (t == 1 && s_abort) break;
        }
        if (s_abort) break;
        const int p = s - T + 1;
        if (p >= zc0 && p < zc1) {
            // 128-bit stores of the final TX x TY interior (x0, d multiples of 4)
            const float *X = ring_x + slot_of(p) * PLANE;
            constexpr int V = TX / 4;
            for (int q = tid; q < TY * V; q += NT) {
                const int ry = q / V, rx = 4 * (q % V);
                const int gy = y0 + ry, gx = x0 + rx;
                if (gy < d && gx < d) {
                    const float4 v = *reinterpret_cast<const float4 *>(X + (ry + T) * BX + rx + H);
                    *reinterpret_cast<float4 *>(xo + ((size_t)p * d + gy) * d + gx) = v;
                }
            }
        }
    }
    if (s_abort && tid == 0) {
        // let copies still in flight land before the CTA's shared memory goes
        // away: the last phase of every slot that was loaded, bounded again
        for (int r = 0; r < R; r++) {
            if (!s_issued[r]) continue;
            const uint32_t parity = (s_issued[r] - 1u) & 1u;
            uint32_t it = 0;
            while (!mbar_try_wait(&bars[r], parity) && ++it < kWaitLimit) {
            }
        }
    }
}

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// The configurations built; TbConfig::variant indexes this table.
struct TbVariant {
    int T, TX, TY, NT, PF;
    bool BG, G4;
    size_t smem;
    const void *kernel;
};

template <int T, int TX, int TY, int NT, int PF, bool BG, bool G4 = false>
TbVariant make_variant() {
    return TbVariant{T, TX, TY, NT, PF, BG, G4, TbShape<T, TX, TY, PF, BG>::SMEM,
                     (const void *)tb_smooth_kernel<T, TX, TY, NT, PF, BG, G4>};
}

const TbVariant *variants(int *count) {
    // Measured on B200 (256^3, three components, 8 half sweeps): 0.89 ms
    // (T2 64x16), 0.81 ms (T2 128x32), 0.94 ms for the plain half sweeps;
    // staging b through the ring beat reading it from global memory, and T = 4
    // lost to its larger halo.
    static const TbVariant v[] = {
        make_variant<2, 64, 16, 384, 4, false>(),
        make_variant<2, 128, 32, 1024, 1, false>(),
        make_variant<4, 64, 16, 384, 4, false>(),
        // groups of 4 cells per thread (one item per thread, or two for 128 x 32)
        make_variant<2, 64, 16, 384, 4, false, true>(),
        make_variant<2, 128, 16, 704, 1, false, true>(),
        make_variant<2, 128, 32, 640, 1, false, true>(),
        make_variant<4, 64, 16, 448, 4, false, true>(),
    };
    *count = (int)(sizeof(v) / sizeof(v[0]));
    return v;
}

}  // namespace

int tb_variant_count() {
    int c = 0;
    variants(&c);
    return c;
}

void tb_variant_shape(int variant, int *T, int *TX, int *TY, int *G4) {
    int c = 0;
    const TbVariant *v = variants(&c);
    const TbVariant &w = v[(variant >= 0 && variant < c) ? variant : 0];
    *T = w.T;
    *TX = w.TX;
    *TY = w.TY;
    if (G4) *G4 = w.G4 ? 1 : 0;
}

// 4-D tensor map {d, d, d, comps} of FP32 over `base`, box {BX, BY, 1, 1}.
cudaError_t tb_make_map(CUtensorMap *map, float *base, int d, int comps, int variant) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn) return cudaErrorNotSupported;
    int c = 0;
    const TbVariant &w = variants(&c)[variant];
    const int H = (w.T + 3) / 4 * 4;
    const cuuint64_t dims[4] = {(cuuint64_t)d, (cuuint64_t)d, (cuuint64_t)d, (cuuint64_t)comps};
    const cuuint64_t strides[3] = {(cuuint64_t)d * 4, (cuuint64_t)d * d * 4, (cuuint64_t)d * d * d * 4};
    const cuuint32_t box[4] = {(cuuint32_t)(w.TX + 2 * H), (cuuint32_t)(w.TY + 2 * w.T), 1, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    memset(map, 0, sizeof(*map));
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// Opts the variant's kernel into its dynamic shared memory (once, at set-up,
// outside any stream capture) and returns how many of its CTAs fit on an SM.
cudaError_t tb_prepare(int variant, int *blocks_per_sm) {
    int c = 0;
    const TbVariant &w = variants(&c)[variant];
    PPPM_CUDA_TRY(cudaFuncSetAttribute(w.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)w.smem));
    PPPM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, w.kernel, w.NT, w.smem));
    return cudaSuccess;
}

// One pass of T half sweeps over a level: x_out = S^T(x_in [+ P xc], b).
// map_x describes x_in (ignored when load_x = 0, start from zero); xc is the
// coarser level's x for a fused prolongation, or null.
cudaError_t tb_smooth(int variant, const CUtensorMap &map_x, const CUtensorMap &map_b, const float *b_dev, int load_x,
                      const float *xc, float *x_out, int d, int comps, int zchunk, uint32_t *err, cudaStream_t st) {
    int c = 0;
    const TbVariant &w = variants(&c)[variant];
    const int zchunks = (d + zchunk - 1) / zchunk;
    const dim3 grid((d + w.TX - 1) / w.TX, (d + w.TY - 1) / w.TY, comps * zchunks);
    const float *bg = b_dev;
    void *args[] = {(void *)&map_x, (void *)&map_b, &load_x, (void *)&xc, &x_out, &d, &zchunk, (void *)&zchunks,
                    &err, (void *)&bg};
    ::pppm::note_launch();
    return cudaLaunchKernel(w.kernel, grid, dim3(w.NT), args, w.smem, st);
}

}  // namespace pppm
