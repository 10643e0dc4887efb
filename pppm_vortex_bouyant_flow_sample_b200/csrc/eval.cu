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
// Pair arithmetic is FP32 (r^3 = r^2 sqrt.approx(r^2) in the warp-uniform walk,
// r^2 rsqrt(r^2) in a lane's own walk; ~1 ulp).  phi: when no pair of the
// scene can reach t = 0.25, a degree-4 polynomial (Chebyshev interpolant on
// [0, 0.25], relative error 5e-9); otherwise a degree-7 one on [0, 2] (relative
// error 2e-7, below that of the exp form near t = 0.25) and (1 - exp(-t)) / t
// above t = 2.  No cancellation in either polynomial.  When some pair can
// reach t = 2 (a smoothing radius of about a cell or less), the warp-uniform
// walk takes the exp form (1 - e^-t) / (4 pi r^3) for every pair, r^-1 from
// rsqrt.approx and e^-t from ex2.approx, with a degree-5 polynomial of phi
// below t = 1/64, where 1 - e^-t would cancel.
#include <climits>
#include <cstring>
#include <cmath>
#include <type_traits>
#include <utility>

#include "pppm_internal.cuh"

namespace pppm {

namespace {

constexpr int kEvalThreads = 128;
// Resident blocks per SM the evaluation kernels are compiled for: 9 (56
// registers, a few bytes of spill outside the pair loop) measured 12.85 ms on
// the 1M-ring headline against 13.05 ms with 8 (64 registers) and 13.77 ms
// with 10 (48 registers).
constexpr int kEvalBlocksPerSM = 9;

__device__ __forceinline__ float3 rel_pos(float4 p, const DevParams *__restrict__ P) {
    return make_float3((float)((double)p.x - P->origin[0]), (float)((double)p.y - P->origin[1]),
                       (float)((double)p.z - P->origin[2]));
}

// Evaluation order: NGP cell, then the Gray rank of the point's octant inside
// the cell, then (fine = 1) the Gray rank of its quarter-cell inside the
// octant (points outside the grid last).  A warp of consecutive points then
// covers about a quarter of a cell, so the union of its lanes' near-field
// boxes, over which it walks, exceeds each lane's own box by little and few
// staged candidates fail the lane's box test.  The order is internal: results
// return in caller order.
__global__ void eval_keys_kernel(const float4 *__restrict__ eval_a, uint32_t M, const DevParams *__restrict__ P,
                                 int fine, uint32_t *__restrict__ key, uint32_t *__restrict__ idx) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M) return;
    const float3 r = rel_pos(eval_a[t], P);
    const double invh = P->invh;
    const uint32_t n = P->n;
    const double qx = (double)r.x * invh, qy = (double)r.y * invh, qz = (double)r.z * invh;
    const double fx = floor(qx), fy = floor(qy), fz = floor(qz);
    const double dn = (double)n;
    const int sh = fine ? 6 : 3;
    uint32_t k = (n * n * n) << sh;
    if (fx >= 0.0 && fx < dn && fy >= 0.0 && fy < dn && fz >= 0.0 && fz < dn) {
        // quarter-cell coordinates 0..3 per axis (clamped against rounding)
        const uint32_t ux = min(3u, (uint32_t)(4.0 * (qx - fx))), uy = min(3u, (uint32_t)(4.0 * (qy - fy))),
                       uz = min(3u, (uint32_t)(4.0 * (qz - fz)));
        const uint32_t oct = (ux >> 1) | ((uy >> 1) << 1) | ((uz >> 1) << 2);
        // groups in Gray-code order (0,1,3,2,6,7,5,4): neighbouring groups differ
        // along one axis, so a warp spanning two groups widens its walk on one
        // axis only
        const uint32_t rank = (0x54672310u >> (4 * oct)) & 7u;
        const uint32_t cell = ((uint32_t)fz * n + (uint32_t)fy) * n + (uint32_t)fx;
        if (fine) {
            const uint32_t sub = (ux & 1u) | ((uy & 1u) << 1) | ((uz & 1u) << 2);
            k = (cell << 6) | (rank << 3) | ((0x54672310u >> (4 * sub)) & 7u);
        } else {
            k = (cell << 3) | rank;
        }
    }
    key[t] = k;
    idx[t] = t;
}

struct PairAcc {
    float x = 0.f, y = 0.f, z = 0.f;
    unsigned long long n = 0;
};

// phi(t) = (1 - e^-t) / t, scaled by 1/(4 pi a^3).  Below t = 0.25 a degree-4
// polynomial (the interpolant at the 5 Chebyshev nodes of [0, 0.25], relative
// error below 5e-9 with float coefficients) needs no special function; its
// coefficients arrive pre-scaled by 1/(4 pi a^3) in cf[0..4].  Above t = 0.25,
// (1 - exp(-t)) / t.  The exp branch runs only when the scene can reach it
// and some lane of the warp needs it (UNIFORM: the whole warp executes this
// call together; otherwise each lane branches on its own t).
template <bool UNIFORM>
__device__ __forceinline__ float smooth_coeff(float t, const float *cf, float inv4pia3, bool need_exp) {
    float p = cf[4];
    p = fmaf(p, t, cf[3]);
    p = fmaf(p, t, cf[2]);
    p = fmaf(p, t, cf[1]);
    p = fmaf(p, t, cf[0]);
    if (need_exp) {
        const bool big = t >= 0.25f;
        if (UNIFORM ? __any_sync(0xffffffffu, big) : big) {
            const float e = __fdividef(1.0f - __expf(-t), fmaxf(t, 0.25f)) * inv4pia3;
            p = big ? e : p;
        }
    }
    return p;
}

// One candidate pair, branch free: the box test, the lane's cell range and
// the zero-distance exclusions become a zero coefficient.  SEG: test the
// segment's other end; COUNT: count the pairs inside the box.
template <bool SEG, bool COUNT, bool UNIFORM>
__device__ __forceinline__ void pair_term(const float4 r, const float4 al, bool lane_ok, const float3 ra,
                                          const float3 rb, float cr, float inv_a3, const float *cf, float inv4pia3,
                                          bool need_exp, PairAcc &acc) {
    const float dx = ra.x - r.x, dy = ra.y - r.y, dz = ra.z - r.z;
    const float m = fmaxf(fabsf(dx), fmaxf(fabsf(dy), fabsf(dz)));
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    const bool inbox = lane_ok && m <= cr;
    if (COUNT) acc.n += inbox ? 1ull : 0ull;
    bool ok = inbox && !(r2 < 1e-24f);
    if (SEG) {
        const float ex = rb.x - r.x, ey = rb.y - r.y, ez = rb.z - r.z;
        ok = ok && !(fmaf(ex, ex, fmaf(ey, ey, ez * ez)) < 1e-24f);
    }
    const float rr = r2 * rsqrtf(fmaxf(r2, 1e-30f));
    const float c = smooth_coeff<UNIFORM>(r2 * rr * inv_a3, cf, inv4pia3, need_exp);
    const float coeff = ok ? c : 0.0f;
    acc.x = fmaf(al.y * dz - al.z * dy, coeff, acc.x);
    acc.y = fmaf(al.z * dx - al.x * dz, coeff, acc.y);
    acc.z = fmaf(al.x * dy - al.y * dx, coeff, acc.z);
}

// Near-field sum over one hash cell's vortices for one point (own walk).
template <bool SEG, bool COUNT>
__device__ __forceinline__ void cell_pairs(const float4 *__restrict__ vrec, const float4 *__restrict__ valf,
                                           uint32_t ps, uint32_t pe, bool lane_ok, const float3 ra, const float3 rb,
                                           float cr, float inv_a3, const float *cf, float inv4pia3, bool need_exp,
                                           PairAcc &acc) {
    for (uint32_t p = ps; p < pe; p++)
        pair_term<SEG, COUNT, false>(vrec[p], valf[p], lane_ok, ra, rb, cr, inv_a3, cf, inv4pia3, need_exp, acc);
}

// Packed accumulators of the warp-uniform walk (.x half: even records of a
// staged chunk, .y half: odd ones).  The near-field sum
//   sum_p c_p alpha_p x (ra - r_p)
// is kept as  A x (ra - o) - B  with  A = sum_p c_p alpha_p  and
// B = sum_p c_p alpha_p x (r_p - o), o a point of the warp's neighbourhood
// (lane 0's position): the per-source moment alpha_p x (r_p - o) is formed
// once when the record is staged, so a pair costs 6 multiply-adds for the
// accumulation instead of 9 for a cross product per pair.  With o within a few
// cells of both points, the two terms are of the size of the result (no
// cancellation beyond a few ulp).
struct PairAcc2 {
    float2 ax = {0.f, 0.f}, ay = {0.f, 0.f}, az = {0.f, 0.f};
    float2 bx = {0.f, 0.f}, by = {0.f, 0.f}, bz = {0.f, 0.f};
    unsigned long long n = 0;
};

// Per-warp ring of staged vortex records: 64 records as 32 record pairs, so
// that one Blackwell f32x2 instruction (FADD2 / FMUL2 / FFMA2) works on two
// records: slot p holds records 2p (.x, .z halves) and 2p+1 (.y, .w halves).
// Planes: A {-x, -y}, B {-z, alpha_x}, C {alpha_y, alpha_z}, D {m_x, m_y},
// E {m_z} with m = alpha x (r - o).  Records kept from successive runs are
// appended (record i at slot (i / 2) mod 32) and evaluated 32 at a time, so
// the pair loop runs whole blocks of 16 slots whatever the lengths of the
// runs; only the last block of a walk is partial.
constexpr int kPackSlots = 32;
constexpr int kPackPlanes = 5;
constexpr uint32_t kBlockRecs = 32;  // records per block of the pair loop

struct Ring {
    uint32_t fill = 0;  // records staged so far
    uint32_t head = 0;  // records evaluated so far (a multiple of kBlockRecs)
    bool near = false;  // a waiting record may lie within a / 4 of a lane (exp form)
};

// max(|a|, |b|, |c|) in one instruction: the three-input max.abs of PTX ISA 8.8
// (sm_100 and later).
__device__ __forceinline__ float max3_abs(float a, float b, float c) {
    float r;
    asm("max.abs.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// sqrt.approx.ftz.f32: one special-function op, sqrt(+0) = +0, so
// r^3 = r^2 sqrt(r^2) needs no guard at r = 0 (where rsqrt would give infinity);
// a subnormal r^2 (r < 1e-19) flushes to 0, where phi is its value at 0.
__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// rsqrt.approx.ftz.f32 and ex2.approx.ftz.f32: one special-function op each.
__device__ __forceinline__ float rsqrt_approx(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float ex2_approx(float x) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Exp-form constants of the warp-uniform walk for scenes whose pairs reach
// t = (r/a)^3 >= 2 (smoothing radius of about a cell or less).
struct ExpForm {
    float2 inv_a3;   // {1/a^3, 1/a^3}
    float2 nl2a3;    // {-log2(e)/a^3, ...}: the exponent of e^-t in base 2, per r^3
    float tsmall;    // below it phi comes from the polynomial (1 - e^-t cancels)
    float r3small;   // r^3 above tsmall * a^3 by a margin: the warp's trigger
};

// Switch point of the exp form to the polynomial.  ex2.approx has a relative
// error of about 2^-22 (the PTX ISA's bound), so near 1 the absolute error of
// e^-t is about 2^-22 and 1 - e^-t carries a relative error of about
// 2^-22 / t: 1.5e-5 at t = 1/64 (r = a / 4), falling as 1 / t, on pairs whose
// terms are a small part of the sum.  A low switch point keeps the polynomial
// branch rare: with a = h and K = 1 about 0.2 % of a lane's pairs have
// t < 1/64, against 5 % below t = 0.5, where some lane of the warp needed the
// branch on nearly every step.
constexpr float kExpSmallT = 1.0f / 64.0f;

// WIDX: the record's index into the sorted vortices goes to E's spare half
// (the index test of segment evaluation).
template <bool WIDX = false>
__device__ __forceinline__ void stage_record(float *__restrict__ pk, int slot, int half, float4 r, float4 a,
                                             float3 o, uint32_t ridx = 0xFFFFFFFFu) {
    float *A = pk + 4 * (0 * kPackSlots + slot), *B = pk + 4 * (1 * kPackSlots + slot);
    float *Cc = pk + 4 * (2 * kPackSlots + slot), *D = pk + 4 * (3 * kPackSlots + slot);
    float *E = pk + 4 * (4 * kPackSlots + slot);
    const float sx = r.x - o.x, sy = r.y - o.y, sz = r.z - o.z;
    A[half] = -r.x; A[2 + half] = -r.y;
    B[half] = -r.z; B[2 + half] = a.x;
    Cc[half] = a.y; Cc[2 + half] = a.z;
    D[half] = fmaf(a.y, sz, -(a.z * sy)); D[2 + half] = fmaf(a.z, sx, -(a.x * sz));
    E[half] = fmaf(a.x, sy, -(a.y * sx));
    if (WIDX) E[2 + half] = __uint_as_float(ridx);
}

// The pair loop over np slots of the ring from slot s0 (FULL: one whole block
// of 16 slots, unrolled into straight-line code with constant offsets): every
// lane takes the records two at a time from shared memory (broadcast reads)
// and evaluates both pairs with packed f32x2 arithmetic.  cr_lane is the box
// half-width, or -1 for an inactive lane.  The r = 0 exclusion needs no test:
// the pair's (ra - r_p) is zero.  SEG: the other-end test, 1 by position
// (|rb - r_p|^2 < 1e-24), 2 by record index (the one vortex at rb, pstar, found
// beforehand), 0 none.  phi is the
// degree-DEG polynomial cf (DEG 4: the scene never leaves [0, 0.25]; DEG 7:
// valid on [0, 2], the exp form above tbig when need_exp; DEG 0: the exp form,
// the polynomial only for small t, looked for only when CHECK).  FOLD: the
// coefficients carry the powers of 1/a^3, so the polynomial takes r^3
// directly and tbig is in r^3 too.
template <int SEG, bool COUNT, bool FOLD, int DEG, bool FULL, bool CHECK>
__device__ __forceinline__ void pair_slots(const float4 *__restrict__ pk4, uint32_t s0, uint32_t np, float cr_lane,
                                           const float3 ra, const float3 rb, uint32_t pstar, float2 inv_a3,
                                           const float2 *cf, float tbig, float inv4pia3, bool need_exp,
                                           PairAcc2 &acc, const ExpForm &xf) {
    const float2 tx = make_float2(ra.x, ra.x), ty = make_float2(ra.y, ra.y), tz = make_float2(ra.z, ra.z);
    const uint32_t cnt = FULL ? kBlockRecs / 2 : np;
#pragma unroll (FULL ? kBlockRecs / 2 : 2)
    for (uint32_t i = 0; i < cnt; i++) {
        const uint32_t p = s0 + i;
        const float4 A = pk4[0 * kPackSlots + p], B = pk4[1 * kPackSlots + p], Cc = pk4[2 * kPackSlots + p];
        const float4 D = pk4[3 * kPackSlots + p], E = pk4[4 * kPackSlots + p];
        const float2 nx = make_float2(A.x, A.y), ny = make_float2(A.z, A.w), nz = make_float2(B.x, B.y);
        const float2 dx = __fadd2_rn(tx, nx), dy = __fadd2_rn(ty, ny), dz = __fadd2_rn(tz, nz);
        const float m0 = max3_abs(dx.x, dy.x, dz.x);
        const float m1 = max3_abs(dx.y, dy.y, dz.y);
        // (the exp form adds 1e-30 to r^2 in the chain, so that rsqrt stays
        // finite at r = 0; that pair takes the polynomial below)
        const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, make_float2(DEG == 0 ? 1e-30f : 0.f,
                                                                                    DEG == 0 ? 1e-30f : 0.f))));
        bool ok0 = m0 <= cr_lane, ok1 = m1 <= cr_lane;
        if (COUNT) acc.n += (ok0 ? 1ull : 0ull) + (ok1 ? 1ull : 0ull);
        if (SEG == 2) {
            ok0 = ok0 && __float_as_uint(E.z) != pstar;
            ok1 = ok1 && __float_as_uint(E.w) != pstar;
        }
        if (SEG == 1) {
            const float2 ex = __fadd2_rn(make_float2(rb.x, rb.x), nx);
            const float2 ey = __fadd2_rn(make_float2(rb.y, rb.y), ny);
            const float2 ez = __fadd2_rn(make_float2(rb.z, rb.z), nz);
            const float2 e2 = __ffma2_rn(ex, ex, __ffma2_rn(ey, ey, __fmul2_rn(ez, ez)));
            ok0 = ok0 && !(e2.x < 1e-24f);
            ok1 = ok1 && !(e2.y < 1e-24f);
        }
        float2 c;
        if constexpr (DEG == 0) {
            // exp form, c * 4 pi = (1 - e^-t) / r^3 with t = r^3 / a^3: r^-1
            // from rsqrt, e^-t from ex2 (two special-function ops); where
            // some lane has t < tsmall (1 - e^-t cancels, or r = 0) the
            // degree-5 polynomial phi(t) / a^3 replaces it
            const float2 rs = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
            const float2 r3 = __fmul2_rn(r2, __fmul2_rn(r2, rs));
            const float2 ri3 = __fmul2_rn(__fmul2_rn(rs, rs), rs);
            const float2 ex = __fmul2_rn(r3, xf.nl2a3);
            const float2 e = make_float2(ex2_approx(ex.x), ex2_approx(ex.y));
            c = __ffma2_rn(make_float2(-e.x, -e.y), ri3, ri3);
            // the trigger r^3 < r3small is a superset of t < tsmall, and
            // a lane outside its box may trigger it (its coefficient is
            // dropped below either way)
            if (CHECK && __any_sync(0xffffffffu, fminf(r3.x, r3.y) < xf.r3small)) {
                const float2 t = __fmul2_rn(r3, xf.inv_a3);
                float2 p = __ffma2_rn(cf[5], t, cf[4]);
#pragma unroll
                for (int q = 3; q >= 0; q--) p = __ffma2_rn(p, t, cf[q]);
                p = __fmul2_rn(p, xf.inv_a3);
                c.x = t.x < xf.tsmall ? p.x : c.x;
                c.y = t.y < xf.tsmall ? p.y : c.y;
            }
        } else {
            const float2 r3 = __fmul2_rn(r2, make_float2(sqrt_approx(r2.x), sqrt_approx(r2.y)));
            const float2 t = FOLD ? r3 : __fmul2_rn(r3, inv_a3);
            c = __ffma2_rn(cf[DEG], t, cf[DEG - 1]);
#pragma unroll
            for (int q = DEG - 2; q >= 0; q--) c = __ffma2_rn(c, t, cf[q]);
            if (DEG > 4 && need_exp) {
                const bool big0 = ok0 && t.x >= tbig, big1 = ok1 && t.y >= tbig;
                if (__any_sync(0xffffffffu, big0 || big1)) {
                    const float v0 = FOLD ? t.x * inv_a3.x : t.x, v1 = FOLD ? t.y * inv_a3.y : t.y;
                    const float e0 = __fdividef(1.0f - __expf(-v0), fmaxf(v0, 1.0f)) * inv4pia3;
                    const float e1 = __fdividef(1.0f - __expf(-v1), fmaxf(v1, 1.0f)) * inv4pia3;
                    c.x = big0 ? e0 : c.x;
                    c.y = big1 ? e1 : c.y;
                }
            }
        }
        // the exp form's c is finite for every pair of an active lane (r = 0
        // lies inside the box and takes the polynomial), so the box mask can
        // multiply it; the polynomials can overflow on the padding record
        const float2 coeff = (DEG == 0 && SEG != 1 && !COUNT)
                                 ? __fmul2_rn(c, make_float2(ok0 ? 1.0f : 0.0f, ok1 ? 1.0f : 0.0f))
                                 : make_float2(ok0 ? c.x : 0.0f, ok1 ? c.y : 0.0f);
        acc.ax = __ffma2_rn(coeff, make_float2(B.z, B.w), acc.ax);
        acc.ay = __ffma2_rn(coeff, make_float2(Cc.x, Cc.y), acc.ay);
        acc.az = __ffma2_rn(coeff, make_float2(Cc.z, Cc.w), acc.az);
        acc.bx = __ffma2_rn(coeff, make_float2(D.x, D.y), acc.bx);
        acc.by = __ffma2_rn(coeff, make_float2(D.z, D.w), acc.by);
        acc.bz = __ffma2_rn(coeff, make_float2(E.x, E.y), acc.bz);
    }
}

// Appends one run of vortex records [ps, pe) to the ring, 32 at a time (one
// coalesced load per stream).  Records outside the warp's box [blo, bhi]
// (every lane's box, widened beyond float rounding) cannot pass any lane's
// test and are dropped.  Whenever 32 records wait, the warp evaluates them.
// The ring never overwrites a record still waiting: before a chunk fewer than
// 32 wait, a chunk adds at most 32, and the ring holds 64.
// Exp form: a record farther than dnear inside the warp's box [blo, bhi] on
// some axis is more than a / 4 (with a margin) from every lane's point, so no
// pair with it needs the small-t polynomial; a block of 32 records with no
// other record skips the warp's test for it.  The records still waiting after
// a block all come from the chunk just staged (fewer than 32 waited before
// it), so that chunk's flag carries over.
template <int SEG, bool COUNT, bool FOLD, int DEG>
__device__ __forceinline__ void stage_run(const float4 *__restrict__ vrec, const float4 *__restrict__ valf,
                                          uint32_t ps, uint32_t pe, float cr_lane, const float3 ra,
                                          const float3 rb, uint32_t pstar, float3 o, const float3 blo,
                                          const float3 bhi,
                                          float dnear, float2 inv_a3, const float2 *cf, float tbig,
                                          float inv4pia3, bool need_exp, float4 *__restrict__ pk4, int lane,
                                          Ring &ring, PairAcc2 &acc, const ExpForm &xf) {
    float *pk = reinterpret_cast<float *>(pk4);
    for (uint32_t base = ps; base < pe; base += 32) {
        const uint32_t cnt = min(32u, pe - base);
        // the strength is loaded with the position (one latency per chunk,
        // not two), also for records the box test then drops
        bool keep = false;
        float4 r = make_float4(0.f, 0.f, 0.f, 0.f), al = r;
        if ((uint32_t)lane < cnt) {
            r = vrec[base + lane];
            al = valf[base + lane];
            keep = r.x >= blo.x && r.x <= bhi.x && r.y >= blo.y && r.y <= bhi.y && r.z >= blo.z && r.z <= bhi.z;
        }
        const unsigned kept = __ballot_sync(0xffffffffu, keep);
        if (kept == 0u) continue;
        bool near_chunk = true;
        if (DEG == 0) {
            const bool nr = keep && r.x >= blo.x + dnear && r.x <= bhi.x - dnear && r.y >= blo.y + dnear &&
                            r.y <= bhi.y - dnear && r.z >= blo.z + dnear && r.z <= bhi.z - dnear;
            near_chunk = __any_sync(0xffffffffu, nr);
        }
        if (keep) {
            const uint32_t dst = ring.fill + (uint32_t)__popc(kept & ((1u << lane) - 1u));
            stage_record<SEG == 2>(pk, (int)((dst >> 1) & (kPackSlots - 1)), (int)(dst & 1u), r, al, o, base + lane);
        }
        ring.fill += (uint32_t)__popc(kept);
        ring.near = ring.near || near_chunk;
        if (ring.fill - ring.head >= kBlockRecs) {
            __syncwarp();
            const uint32_t s0 = (ring.head >> 1) & (kPackSlots - 1);
            if (DEG != 0 || ring.near)
                pair_slots<SEG, COUNT, FOLD, DEG, true, true>(pk4, s0, 0, cr_lane, ra, rb, pstar, inv_a3, cf, tbig,
                                                              inv4pia3, need_exp, acc, xf);
            else
                pair_slots<SEG, COUNT, FOLD, DEG, true, false>(pk4, s0, 0, cr_lane, ra, rb, pstar, inv_a3, cf,
                                                               tbig, inv4pia3, need_exp, acc, xf);
            ring.head += kBlockRecs;
            ring.near = near_chunk && ring.fill != ring.head;
            __syncwarp();  // the next records may take the slots just read
        }
    }
}

// Evaluates the records left in the ring after the walk (fewer than 32); an
// odd count is padded with a record at (-1e18, -1e18, -1e18) and zero
// strength, outside every box.
template <int SEG, bool COUNT, bool FOLD, int DEG>
__device__ __forceinline__ void finish_ring(float cr_lane, const float3 ra, const float3 rb, uint32_t pstar,
                                            float2 inv_a3,
                                            const float2 *cf, float tbig, float inv4pia3, bool need_exp,
                                            float4 *__restrict__ pk4, int lane, const Ring &ring, PairAcc2 &acc,
                                            const ExpForm &xf) {
    const uint32_t rem = ring.fill - ring.head;
    if (rem == 0) return;
    if (lane == 0 && (rem & 1u))
        stage_record<SEG == 2>(reinterpret_cast<float *>(pk4), (int)((ring.fill >> 1) & (kPackSlots - 1)), 1,
                     make_float4(-1e18f, -1e18f, -1e18f, 0.f), make_float4(0.f, 0.f, 0.f, 0.f),
                     make_float3(0.f, 0.f, 0.f));
    __syncwarp();
    pair_slots<SEG, COUNT, FOLD, DEG, false, true>(pk4, (ring.head >> 1) & (kPackSlots - 1), (rem + 1) >> 1, cr_lane,
                                                   ra, rb, pstar, inv_a3, cf, tbig, inv4pia3, need_exp, acc, xf);
    __syncwarp();
}

constexpr int kUniformMaxSub = 1000;  // warp-uniform walk up to 10^3 half-cells

// SEG: is_segment == 1 with a distinct other-end array (with eval_b == eval_a
// the other-end test is the r = 0 test itself, so SEG is off).
// Series coefficients of the smoothing kernel, known on the host from a alone;
// passed by value so they sit in the constant bank.
// Polynomials of phi, scaled by 1/(4 pi a^3).  The packed forms hold each
// coefficient twice ({c, c}): the f32x2 multiply-add then reads them straight
// from the kernel's parameter bank.  With fold they are in r^3 (c_q / a^(3q)),
// otherwise in t = (r/a)^3.
struct SmoothSeries {
    float c[5];    // degree 4 on [0, 0.25], in t (a lane's own walk)
    float2 p4[5];  // degree 4 on [0, 0.25], packed
    float2 p7[8];  // degree 7 on [0, 2], packed
    float2 p5[6];  // degree 5 on [0, 0.5] in t, unit scale (exp-form walk)
    float t7;      // 2 in the packed polynomials' variable: where the exp form takes over
};

// One block of evaluation points (kEvalThreads consecutive points in the
// evaluation order) of one scene.
template <bool SEG, bool COUNT, bool FOLD>
__device__ __forceinline__ void eval_points(const SmoothSeries &sc, const EvalArgs &ea, uint32_t block,
                                            float4 *__restrict__ stage) {
    const uint32_t *__restrict__ eidx = ea.eidx;
    const uint32_t M = ea.M;
    const float4 *__restrict__ eval_a = ea.eval_a;
    const float4 *__restrict__ eval_b = ea.eval_b;
    const float *__restrict__ far = ea.far;
    const uint32_t *__restrict__ start = ea.start;
    const uint32_t *__restrict__ end = ea.end;
    const uint32_t *__restrict__ sub_start = ea.sub_start;
    const uint32_t *__restrict__ sub_end = ea.sub_end;
    const float4 *__restrict__ vrec = ea.vrec;
    const float4 *__restrict__ valf = ea.valf;
    const DevParams *__restrict__ P = ea.P;
    const int n = ea.n, K = ea.K;
    double *__restrict__ u = ea.u;
    double *__restrict__ v = ea.v;
    double *__restrict__ w = ea.w;
    float *__restrict__ uf = ea.uf;
    unsigned long long *__restrict__ pair_count = ea.pair_count;
    const int lane = threadIdx.x & 31;
    float4 *pk = stage + (threadIdx.x >> 5) * (kPackPlanes * kPackSlots);
    const uint32_t s = block * blockDim.x + threadIdx.x;
    const bool act = s < M;
    const uint32_t q = act ? eidx[s] : 0u;
    float3 ra = make_float3(0.f, 0.f, 0.f), rb = make_float3(0.f, 0.f, 0.f);
    if (act) {
        ra = rel_pos(eval_a[q], P);
        if (SEG) rb = rel_pos(eval_b[q], P);
    }
    const double invh = P->invh;
    const double qx = (double)ra.x * invh, qy = (double)ra.y * invh, qz = (double)ra.z * invh;
    const int i = (int)floor(qx), j = (int)floor(qy), k = (int)floor(qz);
    const uint32_t C = (uint32_t)n * n * n;
    float ux = 0.f, uy = 0.f, uz = 0.f;
    if (act && i >= 0 && i < n && j >= 0 && j < n && k >= 0 && k < n) {
        const double tx = qx - 0.5, ty = qy - 0.5, tz = qz - 0.5;
        const double fx0 = floor(tx), fy0 = floor(ty), fz0 = floor(tz);
        const int i0 = (int)fx0, j0 = (int)fy0, k0 = (int)fz0;
        const float fx = (float)(tx - fx0), fy = (float)(ty - fy0), fz = (float)(tz - fz0);
#pragma unroll
        for (int c = 0; c < 8; c++) {
            const int ii = i0 + (c & 1), jj = j0 + ((c >> 1) & 1), kk = k0 + (c >> 2);
            const float wgt = ((c & 1) ? fx : 1.f - fx) * ((c & 2) ? fy : 1.f - fy) * ((c & 4) ? fz : 1.f - fz);
            if (ii >= 0 && ii < n && jj >= 0 && jj < n && kk >= 0 && kk < n) {
                const size_t g = ((size_t)kk * n + jj) * n + ii;
                ux = fmaf(far[g], wgt, ux);
                uy = fmaf(far[C + g], wgt, uy);
                uz = fmaf(far[2 * (size_t)C + g], wgt, uz);
            }
        }
    }
    PairAcc acc;
    PairAcc2 acc2;
    float3 o_w = make_float3(0.f, 0.f, 0.f);
    // some pair can reach t = 2: the exp-form walk (its sums carry 4 pi)
    const bool tier0 = P->need_exp2 != 0;
    if (K >= 0) {
        // FOLD: coefficients carry 1/(4 pi a^3); otherwise they have unit
        // scale and the sums are scaled once per point below
        const float cr = P->cr_f, inv_a3 = P->inv_a3_f, inv4pia3 = FOLD ? P->inv4pia3_f : 1.0f;
        const bool need_exp = P->need_exp != 0;
        const float *cf = sc.c;
        // some pair can reach t = 0.25 (but not 2): the degree-7 polynomial
        const bool tier7 = need_exp && !tier0;
        const bool need_exp2 = P->need_exp2 != 0;
        ExpForm xf;
        xf.inv_a3 = make_float2(inv_a3, inv_a3);
        xf.nl2a3 = make_float2(-1.4426950408889634f * inv_a3, -1.4426950408889634f * inv_a3);
        xf.tsmall = kExpSmallT;
        xf.r3small = 1.001f * kExpSmallT / inv_a3;
        // warp origin of the packed accumulation: lane 0's position
        const float3 o = make_float3(__shfl_sync(0xffffffffu, ra.x, 0), __shfl_sync(0xffffffffu, ra.y, 0),
                                     __shfl_sync(0xffffffffu, ra.z, 0));
        o_w = o;
        // the warp's box: every active lane's box, widened by far more than
        // the rounding of these float bounds (2^-18 of the coordinates' size)
        float3 blo, bhi;
        {
            float lx = act ? ra.x : INFINITY, ly = act ? ra.y : INFINITY, lz = act ? ra.z : INFINITY;
            float hx = act ? ra.x : -INFINITY, hy = act ? ra.y : -INFINITY, hz = act ? ra.z : -INFINITY;
#pragma unroll
            for (int s2 = 16; s2 > 0; s2 >>= 1) {
                lx = fminf(lx, __shfl_xor_sync(0xffffffffu, lx, s2));
                ly = fminf(ly, __shfl_xor_sync(0xffffffffu, ly, s2));
                lz = fminf(lz, __shfl_xor_sync(0xffffffffu, lz, s2));
                hx = fmaxf(hx, __shfl_xor_sync(0xffffffffu, hx, s2));
                hy = fmaxf(hy, __shfl_xor_sync(0xffffffffu, hy, s2));
                hz = fmaxf(hz, __shfl_xor_sync(0xffffffffu, hz, s2));
            }
            const float mx = ldexpf(fabsf(lx) + fabsf(hx) + cr, -18), my = ldexpf(fabsf(ly) + fabsf(hy) + cr, -18),
                        mz = ldexpf(fabsf(lz) + fabsf(hz) + cr, -18);
            blo = make_float3(lx - cr - mx, ly - cr - my, lz - cr - mz);
            bhi = make_float3(hx + cr + mx, hy + cr + my, hz + cr + mz);
        }
        const float2 inv_a3_2 = make_float2(inv_a3, inv_a3);
        // The reference walks hash cells [i-K-1, i+K+1]^3.  Only the half-cells
        // (cell, octant runs of the vortex order) that can hold a vortex inside
        // the point's box are visited: the box spans K+0.5 cells either side,
        // widened by the hash/NGP rounding bound.  Coordinates below are in
        // half cells.
        const double R = (double)K + 0.5 + P->prune_cells;
        int lo[3], hi[3], rlo[3], rhi[3];
        const double qq[3] = {qx, qy, qz};
        const int cc[3] = {i, j, k};
#pragma unroll
        for (int a = 0; a < 3; a++) {
            rlo[a] = cc[a] - K - 1;
            rhi[a] = cc[a] + K + 1;
            lo[a] = max(max(2 * rlo[a], 0), (int)floor(2.0 * (qq[a] - R)));
            hi[a] = min(min(2 * rhi[a] + 1, 2 * n - 1), (int)floor(2.0 * (qq[a] + R)));
            if (!act || lo[a] > hi[a]) { lo[a] = INT_MAX; hi[a] = INT_MIN; }
        }
        int ulo[3], uhi[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            ulo[a] = __reduce_min_sync(0xffffffffu, lo[a]);
            uhi[a] = __reduce_max_sync(0xffffffffu, hi[a]);
        }
        long long vol = 1;
#pragma unroll
        for (int a = 0; a < 3; a++) vol *= (uhi[a] >= ulo[a]) ? (long long)(uhi[a] - ulo[a] + 1) : 0ll;
        // warp-uniform walk over half-cells: every lane sees the same vortex at
        // once; DEG picks phi's polynomial (one walk per polynomial, so that
        // only one pair loop is live at a time).  The walk does not test a
        // lane's hash-cell range [i-K-1, i+K+1]^3 per run: a vortex inside the
        // lane's box, (K+0.5)h either side of a point of cell i, lies in that
        // range whenever its hash cell differs from its coordinate by less
        // than half a cell, which the rounding bound prune_cells < 1/4 (far
        // beyond float rounding of the relative coordinates) guarantees;
        // otherwise every lane takes its own walk below.
        const float cr_lane = act ? cr : -1.0f;
        // exp form: records inside [blo + dnear, bhi - dnear] may lie within
        // a / 4 of a lane (1 % margin on a / 4, far above the trigger's)
        const float dnear = cr - (float)(0.2525 * P->a);
        // Segments: the pair test on the other end only ever drops a vortex
        // that sits at this lane's other end (|rb - r_p|^2 < 1e-24).  Each lane
        // looks for them among the records of the hash cells its other end can
        // fall in (widened by the rounding bound prune_cells), with the pair
        // loop's own arithmetic.  None: the walk needs no test.  Exactly one
        // (the time step's segments: the other end is the segment's own
        // centre): the pair loop drops that record by its index.  More, or an
        // other end near or beyond the grid's faces (vortices hashed from
        // outside wrap around): the position test.
        int seg_mode = 0;
        uint32_t pstar = 0xFFFFFFFFu;
        if (SEG) {
            int found = 0;
            if (act) {
                const double pr = P->prune_cells + 1e-6;
                const double qb[3] = {(double)rb.x * invh, (double)rb.y * invh, (double)rb.z * invh};
                int clo[3], chi[3];
                bool edge = false;
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    // inside: floor(qb - pr) >= 0 and floor(qb + pr) <= n - 1
                    edge = edge || !(qb[a] >= pr && qb[a] < (double)n - pr);
                    clo[a] = (int)floor(qb[a] - pr);
                    chi[a] = (int)floor(qb[a] + pr);
                }
                if (edge) {
                    found = 2;
                } else {
                    for (int kk = clo[2]; kk <= chi[2] && found < 2; kk++)
                        for (int jj = clo[1]; jj <= chi[1] && found < 2; jj++)
                            for (int ii = clo[0]; ii <= chi[0] && found < 2; ii++) {
                                const uint32_t cell = ((uint32_t)kk * n + (uint32_t)jj) * n + (uint32_t)ii;
                                const uint32_t ps = start[cell];
                                if (ps == kEmpty) continue;
                                const uint32_t pe = end[cell];
                                for (uint32_t p = ps; p < pe && found < 2; p++) {
                                    const float4 r = vrec[p];
                                    const float ex = rb.x + (-r.x), ey = rb.y + (-r.y), ez = rb.z + (-r.z);
                                    if (fmaf(ex, ex, fmaf(ey, ey, ez * ez)) < 1e-24f) {
                                        found++;
                                        pstar = p;
                                    }
                                }
                            }
                }
            }
            seg_mode = __any_sync(0xffffffffu, found >= 2) ? 1 : (__any_sync(0xffffffffu, found == 1) ? 2 : 0);
        }
        auto uniform_walk = [&](auto deg, auto segc) {
            constexpr int D = decltype(deg)::value;
            constexpr int S = decltype(segc)::value;
            const float2 *cfd = D == 0 ? sc.p5 : (D == 7 ? sc.p7 : sc.p4);
            Ring ring;
            for (int k2 = ulo[2]; k2 <= uhi[2]; k2++)
                for (int j2 = ulo[1]; j2 <= uhi[1]; j2++)
                    for (int i2 = ulo[0]; i2 <= uhi[0];) {
                        // the two x-halves of a cell are adjacent runs: walk them as one
                        const bool both = ((i2 & 1) == 0) && (i2 + 1 <= uhi[0]);
                        const int ci = i2 >> 1, cj = j2 >> 1, ck = k2 >> 1;
                        const uint32_t cell = ((uint32_t)ck * n + (uint32_t)cj) * n + (uint32_t)ci;
                        const uint32_t k0 = (cell << 3) | ((uint32_t)(j2 & 1) << 1) | ((uint32_t)(k2 & 1) << 2) |
                                            (uint32_t)(i2 & 1);
                        uint32_t ps = sub_start[k0], pe = sub_end[k0];
                        if (both) {
                            const uint32_t s1 = sub_start[k0 | 1u];
                            if (s1 != kEmpty) {
                                if (ps == kEmpty) ps = s1;
                                pe = sub_end[k0 | 1u];
                            }
                        }
                        i2 += both ? 2 : 1;
                        if (ps == kEmpty) continue;
                        stage_run<S, COUNT, FOLD, D>(vrec, valf, ps, pe, cr_lane, ra, rb, pstar, o, blo, bhi,
                                                     dnear, inv_a3_2, cfd, sc.t7, inv4pia3, D == 7 && need_exp2, pk,
                                                     lane, ring, acc2, xf);
                    }
            finish_ring<S, COUNT, FOLD, D>(cr_lane, ra, rb, pstar, inv_a3_2, cfd, sc.t7, inv4pia3,
                                           D == 7 && need_exp2, pk, lane, ring, acc2, xf);
        };
        auto walk = [&](auto deg) {
            if constexpr (SEG) {
                if (seg_mode == 1) uniform_walk(deg, std::integral_constant<int, 1>{});
                else if (seg_mode == 2) uniform_walk(deg, std::integral_constant<int, 2>{});
                else uniform_walk(deg, std::integral_constant<int, 0>{});
            } else {
                uniform_walk(deg, std::integral_constant<int, 0>{});
            }
        };
        if (vol > 0 && vol <= kUniformMaxSub && P->prune_cells < 0.25) {
            if (tier0) walk(std::integral_constant<int, 0>{});
            else if (tier7) walk(std::integral_constant<int, 7>{});
            else walk(std::integral_constant<int, 4>{});
        } else if (act && lo[0] <= hi[0]) {
            // scattered warp (points outside the grid, sparse regions): own walk
            for (int kk = lo[2] >> 1; kk <= (hi[2] >> 1); kk++)
                for (int jj = lo[1] >> 1; jj <= (hi[1] >> 1); jj++)
                    for (int ii = lo[0] >> 1; ii <= (hi[0] >> 1); ii++) {
                        const uint32_t cell = ((uint32_t)kk * n + (uint32_t)jj) * n + (uint32_t)ii;
                        const uint32_t ps = start[cell];
                        if (ps == kEmpty) continue;
                        cell_pairs<SEG, COUNT>(vrec, valf, ps, end[cell], true, ra, rb, cr, inv_a3, cf, inv4pia3, need_exp, acc);
                    }
        }
    }
    if (act) {
        // packed walk: A x (ra - o) - B
        const float Ax = acc2.ax.x + acc2.ax.y, Ay = acc2.ay.x + acc2.ay.y, Az = acc2.az.x + acc2.az.y;
        const float Bx = acc2.bx.x + acc2.bx.y, By = acc2.by.x + acc2.by.y, Bz = acc2.bz.x + acc2.bz.y;
        const float sx = ra.x - o_w.x, sy = ra.y - o_w.y, sz = ra.z - o_w.z;
        if (tier0) {
            // exp-form sums carry 4 pi (the reference's literal); the lane's
            // own walk carries the scale of its coefficients
            const float kown = FOLD ? 1.0f : P->inv4pia3_f;
            const float k4 = (float)(1.0 / kFourPi);
            ux = fmaf(fmaf(Ay, sz, -(Az * sy)) - Bx, k4, fmaf(acc.x, kown, ux));
            uy = fmaf(fmaf(Az, sx, -(Ax * sz)) - By, k4, fmaf(acc.y, kown, uy));
            uz = fmaf(fmaf(Ax, sy, -(Ay * sx)) - Bz, k4, fmaf(acc.z, kown, uz));
        } else if (FOLD) {
            ux += acc.x + (fmaf(Ay, sz, -(Az * sy)) - Bx);
            uy += acc.y + (fmaf(Az, sx, -(Ax * sz)) - By);
            uz += acc.z + (fmaf(Ax, sy, -(Ay * sx)) - Bz);
        } else {
            const float k = P->inv4pia3_f;
            ux = fmaf(acc.x + (fmaf(Ay, sz, -(Az * sy)) - Bx), k, ux);
            uy = fmaf(acc.y + (fmaf(Az, sx, -(Ax * sz)) - By), k, uy);
            uz = fmaf(acc.z + (fmaf(Ax, sy, -(Ay * sx)) - Bz), k, uz);
        }
        if (P->status != 0) {
            // zero or non-finite domain edge (one vortex, or all coincident):
            // the cell size is 0 and the sums above are meaningless; the
            // velocity is defined as 0 and pppm_get_domain reports the domain
            ux = 0.f;
            uy = 0.f;
            uz = 0.f;
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
    if (COUNT) {
        unsigned long long pairs = acc.n + acc2.n;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
        if ((threadIdx.x & 31) == 0 && pairs) atomicAdd(pair_count, pairs);
    }
}

// One scene: block b evaluates points [128 b, 128 b + 128) of the order.
template <bool SEG, bool COUNT, bool FOLD>
__global__ void __launch_bounds__(kEvalThreads, kEvalBlocksPerSM) eval_kernel(const SmoothSeries sc, const EvalArgs ea) {
    __shared__ float4 stage[(kEvalThreads / 32) * kPackPlanes * kPackSlots];
    eval_points<SEG, COUNT, FOLD>(sc, ea, blockIdx.x, stage);
}

// Several scenes in one launch: block b takes work item work[b] = (scene,
// block of that scene).  The host orders the list so that the blocks of the
// scenes with the most pairs per point come first, which the block scheduler
// then hands out first (longest work first); each point's arithmetic is the
// one-scene kernel's, so results do not depend on the batch.
template <bool SEG, bool COUNT, bool FOLD>
__global__ void __launch_bounds__(kEvalThreads, kEvalBlocksPerSM)
eval_batch_kernel(const SmoothSeries sc, const EvalArgs *__restrict__ scenes, const uint2 *__restrict__ work) {
    __shared__ float4 stage[(kEvalThreads / 32) * kPackPlanes * kPackSlots];
    __shared__ EvalArgs sa;  // the block's scene, read from shared memory where used
    const uint2 it = work[blockIdx.x];
    if (threadIdx.x == 0) sa = scenes[it.x];
    __syncthreads();
    eval_points<SEG, COUNT, FOLD>(sc, sa, it.y, stage);
}

// Monomial coefficients of the degree-deg polynomial that interpolates
// phi(t) = (1 - e^-t) / t at the deg + 1 Chebyshev nodes of [0, T] (a near-best
// uniform approximation: relative error 2.6e-9 for degree 4 on [0, 0.25],
// 2e-8 for degree 7 on [0, 2]), by solving the Vandermonde system in FP64.
void phi_chebyshev(int deg, double T, double *c) {
    const double pi = 3.14159265358979323846;
    const int m = deg + 1;
    double V[8][9];
    for (int k = 0; k < m; k++) {
        const double t = 0.5 * T + 0.5 * T * std::cos((2 * k + 1) * pi / (2.0 * m));
        double pw = 1.0;
        for (int q = 0; q < m; q++) { V[k][q] = pw; pw *= t; }
        V[k][m] = -std::expm1(-t) / t;
    }
    for (int col = 0; col < m; col++) {  // Gauss-Jordan elimination, partial pivoting
        int piv = col;
        for (int r = col + 1; r < m; r++)
            if (std::fabs(V[r][col]) > std::fabs(V[piv][col])) piv = r;
        for (int q = 0; q <= m; q++) std::swap(V[col][q], V[piv][q]);
        for (int r = 0; r < m; r++) {
            if (r == col) continue;
            const double f = V[r][col] / V[col][col];
            for (int q = col; q <= m; q++) V[r][q] -= f * V[col][q];
        }
    }
    for (int q = 0; q < m; q++) c[q] = V[q][m] / V[q][q];
}

}  // namespace

// Evaluation keys of M points and their radix sort (the order the eval
// kernel walks); the sorted original indices land in s->esorted_idx.
cudaError_t launch_eval_sort(pppm_scene *s, const float4 *eval_a, uint32_t M) {
    uint32_t *skey = nullptr, *sidx = nullptr;
    prof_begin(s, kStageEvalSort);
    ::pppm::note_launch();
    // quarter-cell order while the key fits 32 bits (n <= 256), else octants
    const int fine = (64ull * s->C < (1ull << 32)) ? 1 : 0;
    eval_keys_kernel<<<(M + 255) / 256, 256, 0, s->stream>>>(eval_a, M, s->dparams, fine, s->ekey[0], s->eidx[0]);
    PPPM_CUDA_TRY(cudaGetLastError());
    uint32_t bits = 1;
    while (bits < 32 && (1ull << bits) <= (fine ? 64ull : 8ull) * s->C) bits++;
    PPPM_CUDA_TRY(radix_sort_pairs(s->stream, M, bits, s->ekey, s->eidx, s->hist, &skey, &sidx));
    prof_end(s, kStageEvalSort);
    s->esorted_idx = sidx;
    return cudaSuccess;
}

// The smoothing series of a scene and whether its coefficients are folded.
// With an absolute a (known here) the packed polynomials are in r^3
// (c_q / a^(3q), scaled by 1/(4 pi a^3)) while every coefficient stays a
// normal float far from overflow.  Otherwise (a tied to the cell size of the
// build, known only on the device, or extreme a) they are in t = (r/a)^3 with
// unit scale, and the kernel applies 1/(4 pi a^3) from the device parameters
// once per point.
static bool make_series(const pppm_scene *s, SmoothSeries &sc) {
    memset(&sc, 0, sizeof(sc));
    bool fold = s->prm.a_cells <= 0.0;
    double f4[5], f7[8], f5[6];
    phi_chebyshev(4, 0.25, f4);
    phi_chebyshev(7, 2.0, f7);
    phi_chebyshev(5, 0.5, f5);
    for (int q = 0; q < 6; q++) sc.p5[q] = make_float2((float)f5[q], (float)f5[q]);
    double u4[5], u7[8], k = 1.0;
    if (fold) {
        const double a = s->prm.a;
        k = 1.0 / (kFourPi * a * a * a);
        const double ia3 = 1.0 / (a * a * a);
        double pw = 1.0;
        for (int q = 0; q < 8; q++, pw *= ia3) {
            if (q < 5) u4[q] = k * f4[q] * pw;
            u7[q] = k * f7[q] * pw;
            for (double x : {q < 5 ? u4[q] : 1.0, u7[q]})
                if (!(std::fabs(x) <= 1e30 && std::fabs(x) >= 1e-30)) fold = false;
        }
    }
    if (!fold) k = 1.0;
    for (int q = 0; q < 8; q++) {
        if (q < 5) {
            sc.c[q] = (float)(k * f4[q]);
            const float v4 = fold ? (float)u4[q] : sc.c[q];
            sc.p4[q] = make_float2(v4, v4);
        }
        const float v7 = fold ? (float)u7[q] : (float)(k * f7[q]);
        sc.p7[q] = make_float2(v7, v7);
    }
    sc.t7 = fold ? (float)(2.0 * s->prm.a * s->prm.a * s->prm.a) : 2.0f;
    return fold;
}

static EvalArgs make_args(pppm_scene *s, const float4 *eval_a, const float4 *eval_b, uint32_t M, double *u, double *v,
                          double *w, float *uf, unsigned long long *pc) {
    EvalArgs a;
    a.eidx = s->esorted_idx;
    a.M = M;
    a.eval_a = eval_a;
    a.eval_b = eval_b;
    a.far = s->far;
    a.start = s->cell_start;
    a.end = s->cell_end;
    a.sub_start = s->sub_start;
    a.sub_end = s->sub_end;
    a.vrec = s->vrec;
    a.valf = s->valf;
    a.P = s->dparams;
    a.n = (int)s->n;
    a.K = s->prm.K;
    a.u = u;
    a.v = v;
    a.w = w;
    a.uf = uf;
    a.pair_count = pc;
    return a;
}

cudaError_t launch_eval(pppm_scene *s, const float4 *eval_a, const float4 *eval_b, int is_segment, uint32_t M,
                        double *u, double *v, double *w, float *uf, int count_pairs) {
    PPPM_CUDA_TRY(launch_eval_sort(s, eval_a, M));
    if (count_pairs) PPPM_CUDA_TRY(cudaMemsetAsync(s->pair_count, 0, sizeof(unsigned long long), s->stream));
    prof_begin(s, kStageEval);
    ::pppm::note_launch();
    const bool seg = (is_segment == 1) && (eval_b != eval_a);
    const unsigned grid = (M + kEvalThreads - 1) / kEvalThreads;
    SmoothSeries sc;
    const bool fold = make_series(s, sc);
    const EvalArgs ea = make_args(s, eval_a, eval_b, M, u, v, w, uf, count_pairs ? s->pair_count : nullptr);
#define PPPM_EVAL_LAUNCH(SEG_, COUNT_)                                                              \
    do {                                                                                              \
        if (fold) eval_kernel<SEG_, COUNT_, true><<<grid, kEvalThreads, 0, s->stream>>>(sc, ea);      \
        else eval_kernel<SEG_, COUNT_, false><<<grid, kEvalThreads, 0, s->stream>>>(sc, ea);         \
    } while (0)
    if (seg) {
        if (count_pairs) PPPM_EVAL_LAUNCH(true, true);
        else PPPM_EVAL_LAUNCH(true, false);
    } else {
        if (count_pairs) PPPM_EVAL_LAUNCH(false, true);
        else PPPM_EVAL_LAUNCH(false, false);
    }
#undef PPPM_EVAL_LAUNCH
    prof_end(s, kStageEval);
    return cudaGetLastError();
}

// Batched evaluation (pppm_batch_run): the arguments of each item's scene
// after its sort, and whether all items can share one launch (the same
// series, segment mode and folding).
cudaError_t eval_batch_prepare(pppm_scene *s, const float4 *eval_a, const float4 *eval_b, int is_segment, uint32_t M,
                               double *u, double *v, double *w, EvalArgs *args, EvalMode *mode) {
    PPPM_CUDA_TRY(launch_eval_sort(s, eval_a, M));
    SmoothSeries sc;
    mode->fold = make_series(s, sc);
    static_assert(sizeof(SmoothSeries) <= sizeof(mode->series), "series bytes");
    memcpy(mode->series, &sc, sizeof(sc));
    mode->seg = (is_segment == 1) && (eval_b != eval_a);
    *args = make_args(s, eval_a, eval_b, M, u, v, w, nullptr, nullptr);
    return cudaSuccess;
}

// One launch over a device work list of `blocks` (scene, block) items for
// scenes that share `mode`.
cudaError_t launch_eval_batch(const EvalMode &mode, const EvalArgs *args_dev, const uint2 *work_dev, uint32_t blocks,
                              cudaStream_t st) {
    if (!blocks) return cudaSuccess;
    SmoothSeries sc;
    memcpy(&sc, mode.series, sizeof(sc));
    ::pppm::note_launch();
    if (mode.seg) {
        if (mode.fold) eval_batch_kernel<true, false, true><<<blocks, kEvalThreads, 0, st>>>(sc, args_dev, work_dev);
        else eval_batch_kernel<true, false, false><<<blocks, kEvalThreads, 0, st>>>(sc, args_dev, work_dev);
    } else {
        if (mode.fold) eval_batch_kernel<false, false, true><<<blocks, kEvalThreads, 0, st>>>(sc, args_dev, work_dev);
        else eval_batch_kernel<false, false, false><<<blocks, kEvalThreads, 0, st>>>(sc, args_dev, work_dev);
    }
    return cudaGetLastError();
}

}  // namespace pppm
