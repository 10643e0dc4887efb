/*
 * CPU oracle for the PPPM vortex-particle velocity evaluation — TEST
 * INFRASTRUCTURE ONLY (see pppm_oracle.h for scope and pinning status).
 *
 * Build: oracle/Makefile (g++ -O3 -fopenmp -ffp-contract=off).  FP contraction
 * is off so every expression rounds exactly as written here; where the
 * reference mixes float and double the casts below reproduce its promotions.
 */
#include "pppm_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct F4 { float x, y, z, w; };

inline const F4 *as_f4(const float *p) { return reinterpret_cast<const F4 *>(p); }

/* __umul24: product of the low 24 bits of each operand (low 32 bits kept). */
inline uint32_t umul24(uint32_t a, uint32_t b) {
    return (uint32_t)((uint64_t)(a & 0xFFFFFFu) * (uint64_t)(b & 0xFFFFFFu));
}

/* The reference keeps the MG relaxation weight as the float literal 1.43f
 * (MG/MultiGrid_kernel.cu:36) and forms (1-omega) in float before promoting. */
const double kOmega = (double)1.43f;
const double kOneMinusOmega = (double)(1.0f - 1.43f);
/* Literal 4*pi of HFS/GPU_kernel.cu:12,2397,2403. */
const double kFourPi = 12.5663706144;
/* Diagonal self-potential factor of HFS/GPU_kernel.cu:1990-1992. */
const double kDiagPsi = 0.250580605913965;

inline size_t gidx(int i, int j, int k, int d) { return ((size_t)k * d + j) * d + i; }

}  // namespace

extern "C" int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* HFS/BiotSavartSolverImp.cpp:379-409 (setDomain).  The min/max use an
 * else-if, which is equivalent to independent min and max because min <= max
 * holds from the first sample on. */
extern "C" void orc_set_domain(const float *pos4, uint32_t N, double *origin3, double *length) {
    const F4 *pos = as_f4(pos4);
    double maxx, minx, maxy, miny, maxz, minz;
    maxx = minx = pos[0].x;
    maxy = miny = pos[0].y;
    maxz = minz = pos[0].z;
    for (uint32_t i = 1; i < N; i++) {
        if (pos[i].x < minx) minx = pos[i].x; else if (pos[i].x > maxx) maxx = pos[i].x;
        if (pos[i].y < miny) miny = pos[i].y; else if (pos[i].y > maxy) maxy = pos[i].y;
        if (pos[i].z < minz) minz = pos[i].z; else if (pos[i].z > maxz) maxz = pos[i].z;
    }
    double L = 3 * std::max(std::max(maxx - minx, maxy - miny), maxz - minz);
    double cx = minx + 0.5 * (maxx - minx);
    double cy = miny + 0.5 * (maxy - miny);
    double cz = minz + 0.5 * (maxz - minz);
    origin3[0] = cx - 0.5 * L;
    origin3[1] = cy - 0.5 * L;
    origin3[2] = cz - 0.5 * L;
    *length = L;
}

/* PH/particle_hash_kernel.cu:32-70 (calcGridPos, calcGridHash, calcHashD).
 * Cell coordinate = floor((p - origin_f) / h_f) in FP32 with IEEE division;
 * the int % uint wrap turns negatives into large unsigned values. */
extern "C" void orc_calc_hash(const float *pos4, uint32_t N, uint32_t n, float h_f,
                              const float *origin_f3, uint32_t *key, uint32_t *idx) {
    const F4 *pos = as_f4(pos4);
    const float ox = origin_f3[0], oy = origin_f3[1], oz = origin_f3[2];
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < (int64_t)N; t++) {
        volatile float px = pos[t].x, py = pos[t].y, pz = pos[t].z;
        float fx = (px - ox) / h_f;
        float fy = (py - oy) / h_f;
        float fz = (pz - oz) / h_f;
        int gx = (int)std::floor(fx);
        int gy = (int)std::floor(fy);
        int gz = (int)std::floor(fz);
        uint32_t ux = (uint32_t)gx % n, uy = (uint32_t)gy % n, uz = (uint32_t)gz % n;
        key[t] = umul24(umul24(uz, n), n) + umul24(uy, n) + ux;
        idx[t] = (uint32_t)t;
    }
}

/* PH/SpaceHashFunctional.cu:97-102: thrust::sort_by_key, a stable radix sort.
 * A stable sort on the key reproduces its order. */
extern "C" void orc_sort_by_key(uint32_t *key, uint32_t *idx, uint32_t N) {
    std::vector<uint32_t> perm(N);
    std::iota(perm.begin(), perm.end(), 0u);
    std::stable_sort(perm.begin(), perm.end(),
                     [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
    std::vector<uint32_t> k2(N), i2(N);
    for (uint32_t t = 0; t < N; t++) { k2[t] = key[perm[t]]; i2[t] = idx[perm[t]]; }
    std::memcpy(key, k2.data(), sizeof(uint32_t) * N);
    std::memcpy(idx, i2.data(), sizeof(uint32_t) * N);
}

/* PH/SpaceHashFunctional.cu:71-94 + PH/particle_hash_kernel.cu:74-126.
 * Empty cells: start = 0xFFFFFFFF (the memset of :82).  The reference leaves
 * cellEnd of empty cells stale; this restatement writes 0xFFFFFFFF there too. */
extern "C" void orc_find_cell_start(const uint32_t *skey, uint32_t N, uint32_t ncells,
                                    uint32_t *start, uint32_t *end) {
    std::fill(start, start + ncells, 0xFFFFFFFFu);
    std::fill(end, end + ncells, 0xFFFFFFFFu);
    for (uint32_t t = 0; t < N; t++) {
        uint32_t h = skey[t];
        if (t == 0 || h != skey[t - 1]) {
            if (h < ncells) start[h] = t;
            if (t > 0 && skey[t - 1] < ncells) end[skey[t - 1]] = t;
        }
        if (t == N - 1 && h < ncells) end[h] = t + 1;
    }
}

/* HFS/GPU_kernel.cu:218-294 (ParticleToMesh_kernel) with the NGP box weight
 * shape_function_mass (HFS/GPU_kernel.cu:31-50).  The reference gathers, per
 * grid cell, over the 5^3 hash cells around it in (kk, jj, ii) lexicographic
 * order and then in sorted particle order; that is the global sorted order
 * restricted to the window, so scattering each sorted particle to the cells
 * where its weight is 1 accumulates in exactly the reference's order. */
extern "C" void orc_p2m(const uint32_t *start, const uint32_t *end, const float *spos4,
                        const double *smass, double cell_h, uint32_t n, uint32_t N,
                        const double *origin3, double *grid) {
    const F4 *pos = as_f4(spos4);
    const double invh = 1.0 / cell_h;
    const int d = (int)n;
    std::vector<double> sum((size_t)d * d * d, 0.0);
    /* Walk hash cells in key order (the reference's window order). */
    for (int kk = 0; kk < d; kk++)
        for (int jj = 0; jj < d; jj++)
            for (int ii = 0; ii < d; ii++) {
                size_t c = gidx(ii, jj, kk, d);
                if (start[c] == 0xFFFFFFFFu) continue;
                for (uint32_t p = start[c]; p < end[c]; p++) {
                    if (p >= N) continue;
                    float px = (float)((double)pos[p].x - origin3[0]);
                    float py = (float)((double)pos[p].y - origin3[1]);
                    float pz = (float)((double)pos[p].z - origin3[2]);
                    /* grid cells whose window holds hash cell (ii,jj,kk) */
                    for (int k = std::max(0, kk - 2); k <= std::min(d - 1, kk + 2); k++) {
                        double r3 = (double)pz * invh - (double)(float)((double)k + 0.5);
                        if (!(r3 < 0.5 && r3 >= -0.5)) continue;
                        for (int j = std::max(0, jj - 2); j <= std::min(d - 1, jj + 2); j++) {
                            double r2 = (double)py * invh - (double)(float)((double)j + 0.5);
                            if (!(r2 < 0.5 && r2 >= -0.5)) continue;
                            for (int i = std::max(0, ii - 2); i <= std::min(d - 1, ii + 2); i++) {
                                double r1 = (double)px * invh - (double)(float)((double)i + 0.5);
                                if (!(r1 < 0.5 && r1 >= -0.5)) continue;
                                sum[gidx(i, j, k, d)] += 1.0 * smass[p];
                            }
                        }
                    }
                }
            }
    const size_t C = (size_t)d * d * d;
    for (size_t c = 0; c < C; c++) grid[c] = invh * invh * invh * sum[c];
}

/* ------------------------------------------------------------------------
 * Multigrid: MG/MultiGrid.h:114-139 (levels), MG/MultiGrid.cpp:128-250
 * (V-cycle, FMG), MG/Multigrid.cu:46-55,202-330 and
 * MG/MultiGrid_kernel.cu:422-934 (kernels).  Operator: sum of the six
 * neighbours minus 6x, neighbours outside the box read as 0.
 * ---------------------------------------------------------------------- */
namespace {

struct Level { int d; std::vector<double> x, b, r; };

inline double nbr_sum(const double *x, int i, int j, int k, int d) {
    size_t c = gidx(i, j, k, d);
    double lv = (i > 0) ? x[c - 1] : 0.0;
    double rv = (i < d - 1) ? x[c + 1] : 0.0;
    double uv = (j < d - 1) ? x[c + d] : 0.0;
    double dv = (j > 0) ? x[c - d] : 0.0;
    double fv = (k > 0) ? x[c - (size_t)d * d] : 0.0;
    double bv = (k < d - 1) ? x[c + (size_t)d * d] : 0.0;
    double r = lv + rv;
    r += uv + dv;
    r += fv + bv;
    return r;
}

/* MG/Multigrid.cu:202-239, MG/MultiGrid_kernel.cu:722-820: per iteration the
 * "red" launch updates cells with (i+j+k) odd, then the "black" launch the
 * even cells; x <- (1-w) x + w (sum_nbr - b) / 6. */
void rbsor(double *x, const double *b, int d, int iters) {
    const double invdiag = 1.0 / 6.0;
    for (int it = 0; it < iters; it++) {
        for (int color = 1; color >= 0; color--) {
#pragma omp parallel for schedule(static) collapse(2)
            for (int k = 0; k < d; k++)
                for (int j = 0; j < d; j++) {
                    int i0 = ((j + k + color) & 1);
                    for (int i = i0; i < d; i += 2) {
                        size_t c = gidx(i, j, k, d);
                        double r = nbr_sum(x, i, j, k, d);
                        r -= b[c];
                        x[c] = kOneMinusOmega * x[c] + kOmega * r * invdiag;
                    }
                }
        }
    }
}

/* MG/MultiGrid_kernel.cu:821-871: r = b - (sum_nbr - 6 x). */
void residual(const double *x, const double *b, double *res, int d) {
#pragma omp parallel for schedule(static) collapse(2)
    for (int k = 0; k < d; k++)
        for (int j = 0; j < d; j++)
            for (int i = 0; i < d; i++) {
                size_t c = gidx(i, j, k, d);
                double r = nbr_sum(x, i, j, k, d);
                r -= 6 * x[c];
                res[c] = b[c] - r;
            }
}

/* MG/MultiGrid_kernel.cu:873-910: coarse = 0.5 * sum of the 8 children. */
void restrict_(double *coarse, const double *fine, int dc) {
    const int df = 2 * dc;
#pragma omp parallel for schedule(static) collapse(2)
    for (int k = 0; k < dc; k++)
        for (int j = 0; j < dc; j++)
            for (int i = 0; i < dc; i++) {
                size_t f = gidx(2 * i, 2 * j, 2 * k, df);
                size_t fy = f + df, fz = f + (size_t)df * df, fyz = fz + df;
                double r = 0;
                r += fine[f];
                r += fine[f + 1];
                r += fine[fy];
                r += fine[fy + 1];
                r += fine[fz];
                r += fine[fz + 1];
                r += fine[fyz];
                r += fine[fyz + 1];
                r = r * 0.5;
                coarse[gidx(i, j, k, dc)] = r;
            }
}

/* MG/MultiGrid_kernel.cu:912-934: fine += coarse[i/2, j/2, k/2]. */
void prolong(double *fine, const double *coarse, int df) {
    const int dc = df / 2;
#pragma omp parallel for schedule(static) collapse(2)
    for (int k = 0; k < df; k++)
        for (int j = 0; j < df; j++)
            for (int i = 0; i < df; i++)
                fine[gidx(i, j, k, df)] += coarse[gidx(i / 2, j / 2, k / 2, dc)];
}

/* MG/MultiGrid_kernel.cu:422-498 (exact_solve_period3D_jacobi_kerneld): 100
 * iterations of x <- (sum_nbr - b) / 6.  The reference's live phase updates x
 * in place from 512 concurrent threads, so its order is not defined; mode 0
 * runs the update in cell order (in-place Gauss-Seidel), mode 1 as Jacobi. */
void coarse_solve(double *x, const double *b, int d, int coarse_mode) {
    const size_t C = (size_t)d * d * d;
    std::vector<double> xn(x, x + C);
    std::vector<double> tmp(C);
    for (int t = 0; t < 100; t++) {
        if (coarse_mode == 1) {
            for (size_t c = 0; c < C; c++) {
                int i = (int)(c % d), j = (int)((c / d) % d), k = (int)(c / ((size_t)d * d));
                double r = nbr_sum(xn.data(), i, j, k, d);
                r -= b[c];
                tmp[c] = r / 6;
            }
            xn.swap(tmp);
        } else {
            for (size_t c = 0; c < C; c++) {
                int i = (int)(c % d), j = (int)((c / d) % d), k = (int)(c / ((size_t)d * d));
                double r = nbr_sum(xn.data(), i, j, k, d);
                r -= b[c];
                xn[c] = r / 6;
            }
        }
    }
    std::memcpy(x, xn.data(), sizeof(double) * C);
}

struct MG {
    std::vector<Level> lv;
    int coarse_mode = 0;
    explicit MG(int n, int cm) : coarse_mode(cm) {
        int x = n, L = 0;
        while ((long long)x * x * x > 512) { L++; x = x / 2; if (x == 0) x = 1; }
        int levels = L + 1;
        lv.resize(levels);
        int d = n;
        for (int l = 0; l < levels; l++) {
            lv[l].d = d;
            size_t C = (size_t)d * d * d;
            lv[l].x.assign(C, 0.0); lv[l].b.assign(C, 0.0); lv[l].r.assign(C, 0.0);
            d = (d / 2 == 0) ? 1 : d / 2;
        }
    }
    int levels() const { return (int)lv.size(); }
    void zero_from(int l0) {
        for (int l = l0; l < levels(); l++) {
            std::fill(lv[l].x.begin(), lv[l].x.end(), 0.0);
            std::fill(lv[l].b.begin(), lv[l].b.end(), 0.0);
            std::fill(lv[l].r.begin(), lv[l].r.end(), 0.0);
        }
    }
    /* MG/MultiGrid.cpp:128-201, with level `level` holding x and b. */
    void vcycle(int level) {
        const int Lm = levels();
        zero_from(level + 1);
        std::fill(lv[level].r.begin(), lv[level].r.end(), 0.0);
        for (int i = level; i < Lm - 1; ++i) {
            rbsor(lv[i].x.data(), lv[i].b.data(), lv[i].d, 4);
            residual(lv[i].x.data(), lv[i].b.data(), lv[i].r.data(), lv[i].d);
            restrict_(lv[i + 1].b.data(), lv[i].r.data(), lv[i + 1].d);
        }
        coarse_solve(lv[Lm - 1].x.data(), lv[Lm - 1].b.data(), lv[Lm - 1].d, coarse_mode);
        for (int i = Lm - 2; i >= level; --i) {
            prolong(lv[i].x.data(), lv[i + 1].x.data(), lv[i].d);
            rbsor(lv[i].x.data(), lv[i].b.data(), lv[i].d, 4);
        }
        zero_from(level + 1);
    }
    /* MG/MultiGrid.cpp:202-250. */
    void fmg() {
        const int Lm = levels();
        zero_from(1);
        std::fill(lv[0].r.begin(), lv[0].r.end(), 0.0);
        for (int i = 0; i < Lm - 1; ++i) {
            residual(lv[i].x.data(), lv[i].b.data(), lv[i].r.data(), lv[i].d);
            restrict_(lv[i + 1].b.data(), lv[i].r.data(), lv[i + 1].d);
        }
        coarse_solve(lv[Lm - 1].x.data(), lv[Lm - 1].b.data(), lv[Lm - 1].d, coarse_mode);
        for (int i = Lm - 2; i >= 0; --i) {
            prolong(lv[i].x.data(), lv[i + 1].x.data(), lv[i].d);
            vcycle(i);
        }
        vcycle(0);
    }
};

double norm2(const double *v, size_t C) {
    double s = 0;
    for (size_t c = 0; c < C; c++) s += v[c] * v[c];
    return std::sqrt(s);
}

}  // namespace

extern "C" int orc_mg_levels(uint32_t n) { return MG((int)n, 0).levels(); }

extern "C" void orc_apply_laplacian(const double *x, double *y, uint32_t n) {
    const int d = (int)n;
#pragma omp parallel for schedule(static) collapse(2)
    for (int k = 0; k < d; k++)
        for (int j = 0; j < d; j++)
            for (int i = 0; i < d; i++) {
                size_t c = gidx(i, j, k, d);
                y[c] = nbr_sum(x, i, j, k, d) - 6 * x[c];
            }
}

extern "C" double orc_residual_norm(const double *x, const double *b, uint32_t n) {
    const size_t C = (size_t)n * n * n;
    std::vector<double> r(C);
    residual(x, b, r.data(), (int)n);
    return norm2(r.data(), C);
}

/* One V-cycle at the finest level starting from x (MG/MultiGrid.cpp:128-201). */
extern "C" void orc_mg_vcycle(double *x, const double *b, uint32_t n, int coarse_mode) {
    MG mg((int)n, coarse_mode);
    const size_t C = (size_t)n * n * n;
    std::memcpy(mg.lv[0].x.data(), x, sizeof(double) * C);
    std::memcpy(mg.lv[0].b.data(), b, sizeof(double) * C);
    mg.vcycle(0);
    std::memcpy(x, mg.lv[0].x.data(), sizeof(double) * C);
}

/* HFS/BiotSavartSolverImp.cpp:603-620: psi = 0, then m_FullMultiGrid.  In
 * mode 1 further V-cycles run until the relative residual meets tol. */
/* MultiGridSolver3DPeriod_double::m_FullMultiGrid called `repeats` times
 * from the x given (MG/MultiGrid.cpp:202-250: its first residual is b - A x). */
extern "C" void orc_mg_fmg(double *x, const double *b, uint32_t n, int repeats, int coarse_mode) {
    MG mg((int)n, coarse_mode);
    const size_t C = (size_t)n * n * n;
    std::memcpy(mg.lv[0].x.data(), x, sizeof(double) * C);
    std::memcpy(mg.lv[0].b.data(), b, sizeof(double) * C);
    for (int r = 0; r < repeats; r++) mg.fmg();
    std::memcpy(x, mg.lv[0].x.data(), sizeof(double) * C);
}

extern "C" void orc_mg_solve(double *x, const double *b, uint32_t n, int mg_mode,
                             int coarse_mode, double tol, int max_cycles,
                             int32_t *cycles_out, double *relres_out) {
    MG mg((int)n, coarse_mode);
    const size_t C = (size_t)n * n * n;
    std::fill(mg.lv[0].x.begin(), mg.lv[0].x.end(), 0.0);
    std::memcpy(mg.lv[0].b.data(), b, sizeof(double) * C);
    mg.fmg();
    int cycles = 1;
    double bn = norm2(b, C);
    std::vector<double> r(C);
    residual(mg.lv[0].x.data(), b, r.data(), (int)n);
    double rel = bn > 0 ? norm2(r.data(), C) / bn : 0.0;
    if (mg_mode == 1) {
        while (rel > tol && cycles < max_cycles) {
            mg.vcycle(0);
            cycles++;
            residual(mg.lv[0].x.data(), b, r.data(), (int)n);
            rel = bn > 0 ? norm2(r.data(), C) / bn : 0.0;
        }
    }
    std::memcpy(x, mg.lv[0].x.data(), sizeof(double) * C);
    if (cycles_out) *cycles_out = cycles;
    if (relres_out) *relres_out = rel;
}

/* HFS/GPU_kernel.cu:1750-1805 (compute_curl_kernel) with the clamped
 * sampling of sample3D (HFS/GPU_kernel.cu:23-30). */
extern "C" void orc_curl(const double *psi3, double *u3, uint32_t n, double h) {
    const int d = (int)n;
    const size_t C = (size_t)d * d * d;
    const double *Fx = psi3, *Fy = psi3 + C, *Fz = psi3 + 2 * C;
    double *u = u3, *v = u3 + C, *w = u3 + 2 * C;
    const double inv_h = 1.0 / h;
    auto S = [&](const double *f, int x, int y, int z) {
        int i = std::min(std::max(0, x), d - 1);
        int j = std::min(std::max(0, y), d - 1);
        int k = std::min(std::max(0, z), d - 1);
        return f[gidx(i, j, k, d)];
    };
#pragma omp parallel for schedule(static) collapse(2)
    for (int k = 0; k < d; k++)
        for (int j = 0; j < d; j++)
            for (int i = 0; i < d; i++) {
                size_t c = gidx(i, j, k, d);
                double Fz_up = S(Fz, i, j + 1, k), Fz_down = S(Fz, i, j - 1, k);
                double Fz_left = S(Fz, i - 1, j, k), Fz_right = S(Fz, i + 1, j, k);
                double Fy_front = S(Fy, i, j, k - 1), Fy_back = S(Fy, i, j, k + 1);
                double Fy_left = S(Fy, i - 1, j, k), Fy_right = S(Fy, i + 1, j, k);
                double Fx_front = S(Fx, i, j, k - 1), Fx_back = S(Fx, i, j, k + 1);
                double Fx_up = S(Fx, i, j + 1, k), Fx_down = S(Fx, i, j - 1, k);
                u[c] = 0.5 * inv_h * (Fz_up - Fz_down + Fy_front - Fy_back);
                v[c] = 0.5 * inv_h * (Fx_back - Fx_front + Fz_left - Fz_right);
                w[c] = 0.5 * inv_h * (Fy_right - Fy_left + Fx_down - Fx_up);
            }
}

/* HFS/GPU_kernel.cu:11-17 (cpu_compute_r) and 2646-2677: central-difference
 * gradient (step h) of 1/(4 pi |X - X'|) with X at the centre slot (the only
 * slot Step1 reads, :2546-2549) and X' the cell-centre offset.  A coincident
 * pair reads 1/1e24.  table[(off_z+K)(2K+1)^2 + (off_y+K)(2K+1) + off_x+K][3];
 * the centre entry is left 0 (the reference never reads it). */
extern "C" void orc_farfield_table(int K, double h, double *table) {
    auto inv_r = [](double ax, double ay, double az, double bx, double by, double bz) {
        double r_sqr = (ax - bx) * (ax - bx) + (ay - by) * (ay - by) + (az - bz) * (az - bz);
        double r = (r_sqr > 1e-12) ? kFourPi * std::sqrt(r_sqr) : 1e+24;
        return 1.0 / r;
    };
    const int W = 2 * K + 1;
    for (int kk = -K; kk <= K; kk++)
        for (int jj = -K; jj <= K; jj++)
            for (int ii = -K; ii <= K; ii++) {
                double *t = table + 3 * ((size_t)((kk + K) * W + (jj + K)) * W + (ii + K));
                if (ii == 0 && jj == 0 && kk == 0) { t[0] = t[1] = t[2] = 0; continue; }
                double Xpx = ((double)ii + 0.5) * h, Xpy = ((double)jj + 0.5) * h, Xpz = ((double)kk + 0.5) * h;
                double Xx = 0.5 * h, Xy = 0.5 * h, Xz = 0.5 * h;
                t[0] = 0.5 * (inv_r(Xx + h, Xy, Xz, Xpx, Xpy, Xpz) - inv_r(Xx - h, Xy, Xz, Xpx, Xpy, Xpz)) / h;
                t[1] = 0.5 * (inv_r(Xx, Xy + h, Xz, Xpx, Xpy, Xpz) - inv_r(Xx, Xy - h, Xz, Xpx, Xpy, Xpz)) / h;
                t[2] = 0.5 * (inv_r(Xx, Xy, Xz + h, Xpx, Xpy, Xpz) - inv_r(Xx, Xy, Xz - h, Xpx, Xpy, Xpz)) / h;
            }
}

/* HFS/GPU_kernel.cu:2634-2734 (BiotSavartComputeFarField):
 *   Step1 (:2487-2564): far = U - sum_{c' != c, |c'-c|<=K, in box}
 *                              D[c'-c] x (omega(c') h^3)
 *   then psi_d = 0.250580605913965 * omega * h^2 (:1976-2001), its clamped
 *   curl, and far -= curl(psi_d) (:2566-2630; the jjj*dimy index equals
 *   jjj*dimx on the cubic grids used here). */
extern "C" void orc_farfield(const double *vort3, const double *u3, double *far3,
                             uint32_t n, int K, double h) {
    const int d = (int)n;
    const size_t C = (size_t)d * d * d;
    const int W = 2 * K + 1;
    std::vector<double> table((size_t)W * W * W * 3);
    orc_farfield_table(K, h, table.data());
    const double vh3 = h * h * h;
#pragma omp parallel for schedule(static) collapse(2)
    for (int k = 0; k < d; k++)
        for (int j = 0; j < d; j++)
            for (int i = 0; i < d; i++) {
                size_t c = gidx(i, j, k, d);
                double mx = 0, my = 0, mz = 0;
                for (int kk = k - K; kk <= k + K; kk++)
                    for (int jj = j - K; jj <= j + K; jj++)
                        for (int ii = i - K; ii <= i + K; ii++) {
                            double ox = 0, oy = 0, oz = 0, dx = 0, dy = 0, dz = 0;
                            if (kk >= 0 && kk < d && jj >= 0 && jj < d && ii >= 0 && ii < d) {
                                size_t s = gidx(ii, jj, kk, d);
                                ox = vort3[s] * vh3; oy = vort3[C + s] * vh3; oz = vort3[2 * C + s] * vh3;
                                if (!(kk == k && jj == j && ii == i)) {
                                    const double *t = table.data() + 3 * ((size_t)((kk - k + K) * W + (jj - j + K)) * W + (ii - i + K));
                                    dx = t[0]; dy = t[1]; dz = t[2];
                                }
                            }
                            mx += dy * oz - dz * oy;
                            my += dz * ox - dx * oz;
                            mz += dx * oy - dy * ox;
                        }
                far3[c] = u3[c] - mx;
                far3[C + c] = u3[C + c] - my;
                far3[2 * C + c] = u3[2 * C + c] - mz;
            }
    std::vector<double> psid(3 * C), ud(3 * C);
    const double h2 = h * h;
    for (size_t c = 0; c < 3 * C; c++) psid[c] = kDiagPsi * vort3[c] * h2;
    orc_curl(psid.data(), ud.data(), n, h);
    for (size_t c = 0; c < 3 * C; c++) far3[c] -= ud[c];
}

/* HFS/GPU_kernel.cu:2886-2976 (BiotSavartInterpolate_far_field_kernel2) with
 * the hat weight poly_shape (HFS/GPU_kernel.cu:51-84).  Points whose own cell
 * lies outside the grid are left untouched (the caller has zeroed out3). */
extern "C" void orc_interp(const float *eval4, uint32_t M, const double *far3, uint32_t n,
                           double cell_h, const double *origin3, double *out3) {
    const F4 *pos = as_f4(eval4);
    const int d = (int)n;
    const size_t C = (size_t)d * d * d;
    const double invh = 1.0 / cell_h;
    auto poly = [](double r) { double rr = std::fabs(r); return rr < 1 ? 1 - rr : 0.0; };
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < (int64_t)M; t++) {
        float px = (float)((double)pos[t].x - origin3[0]);
        float py = (float)((double)pos[t].y - origin3[1]);
        float pz = (float)((double)pos[t].z - origin3[2]);
        int i = (int)std::floor((double)px * invh);
        int j = (int)std::floor((double)py * invh);
        int k = (int)std::floor((double)pz * invh);
        if (!(i >= 0 && i < d && j >= 0 && j < d && k >= 0 && k < d)) continue;
        double sx = 0, sy = 0, sz = 0;
        double qx = (double)px * invh, qy = (double)py * invh, qz = (double)pz * invh;
        for (int kk = k - 2; kk <= k + 2; kk++)
            for (int jj = j - 2; jj <= j + 2; jj++)
                for (int ii = i - 2; ii <= i + 2; ii++) {
                    if (!(kk >= 0 && kk < d && jj >= 0 && jj < d && ii >= 0 && ii < d)) continue;
                    size_t g = gidx(ii, jj, kk, d);
                    double gx = (double)(float)((double)ii + 0.5);
                    double gy = (double)(float)((double)jj + 0.5);
                    double gz = (double)(float)((double)kk + 0.5);
                    double wgt = poly(gx - qx) * poly(gy - qy) * poly(gz - qz);
                    sx += far3[g] * wgt;
                    sy += far3[C + g] * wgt;
                    sz += far3[2 * C + g] * wgt;
                }
        out3[t] = sx;
        out3[M + t] = sy;
        out3[2 * (size_t)M + t] = sz;
    }
}

/* HFS/GPU_kernel.cu:2262-2485 (BiotSavartPPCorrScaleMN_kernel).  For every
 * evaluation point, over hash cells [i-K-1, i+K+1]^3 and vortices inside the
 * axis box |dx|,|dy|,|dz| < (K+0.5) h (float differences of float relative
 * positions):  u += (alpha x (x_a - y_p)) * c(r) with
 *   c = (1 - exp(-(r/a)^3)) / (4 pi r^3)        for r/a >= 0.01,
 *   c = (1 - (r/a)^3 / 2) / (4 pi a^3)           otherwise (the 1/6 and 1/24
 *                                                 terms are integer 0, :2401),
 * c = 0 if r < 1e-12 or, for segments, if |x_b - y_p| < 1e-12.  Adds into u3
 * (which holds the interpolated far field).  Returns the number of vortex
 * candidates that passed the axis box. */
extern "C" uint64_t orc_pp(const uint32_t *start, const uint32_t *end,
                           const float *eval_a4, const float *eval_b4, int is_segment,
                           const float *svort4, const double *salpha3, double *u3,
                           uint32_t n, double cell_h, int K, uint32_t M, uint32_t N,
                           const double *origin3, double a) {
    const F4 *ea = as_f4(eval_a4), *eb = as_f4(eval_b4), *vp = as_f4(svort4);
    const double *vx = salpha3, *vy = salpha3 + N, *vz = salpha3 + 2 * (size_t)N;
    const int d = (int)n;
    const double invh = 1.0 / cell_h;
    const double correct_radius = ((double)K + 0.5) / invh;
    uint64_t pairs = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : pairs)
    for (int64_t t = 0; t < (int64_t)M; t++) {
        float pax = (float)((double)ea[t].x - origin3[0]);
        float pay = (float)((double)ea[t].y - origin3[1]);
        float paz = (float)((double)ea[t].z - origin3[2]);
        float pbx = 0, pby = 0, pbz = 0;
        if (is_segment == 1) {
            pbx = (float)((double)eb[t].x - origin3[0]);
            pby = (float)((double)eb[t].y - origin3[1]);
            pbz = (float)((double)eb[t].z - origin3[2]);
        }
        int i = (int)std::floor((double)pax * invh);
        int j = (int)std::floor((double)pay * invh);
        int k = (int)std::floor((double)paz * invh);
        double ux = 0, uy = 0, uz = 0;
        for (int kk = k - K - 1; kk <= k + K + 1; kk++)
            for (int jj = j - K - 1; jj <= j + K + 1; jj++)
                for (int ii = i - K - 1; ii <= i + K + 1; ii++) {
                    if (!(kk >= 0 && kk < d && jj >= 0 && jj < d && ii >= 0 && ii < d)) continue;
                    size_t c = gidx(ii, jj, kk, d);
                    if (start[c] == 0xFFFFFFFFu) continue;
                    for (uint32_t p = start[c]; p < end[c]; p++) {
                        if (p >= N) continue;
                        float qx = (float)((double)vp[p].x - origin3[0]);
                        float qy = (float)((double)vp[p].y - origin3[1]);
                        float qz = (float)((double)vp[p].z - origin3[2]);
                        if (!((double)std::fabs(qx - pax) < correct_radius &&
                              (double)std::fabs(qy - pay) < correct_radius &&
                              (double)std::fabs(qz - paz) < correct_radius))
                            continue;
                        pairs++;
                        double ox = vx[p], oy = vy[p], oz = vz[p];
                        double dax = (double)(float)(pax - qx), day = (double)(float)(pay - qy),
                               daz = (double)(float)(paz - qz);
                        double r1 = std::sqrt(dax * dax + day * day + daz * daz);
                        double coeff;
                        double r_inva = r1 / a;
                        if (r_inva >= 0.01) {
                            coeff = (1 - std::exp(-r_inva * r_inva * r_inva)) / (kFourPi * r1 * r1 * r1);
                        } else {
                            double r3a3 = r_inva * r_inva * r_inva;
                            coeff = 1 / (kFourPi * a * a * a) * (1 - 0.5 * r3a3);
                        }
                        if (r1 < 1e-12) coeff = 0;
                        if (is_segment == 1) {
                            double dbx = (double)(float)(pbx - qx), dby = (double)(float)(pby - qy),
                                   dbz = (double)(float)(pbz - qz);
                            double r2 = std::sqrt(dbx * dbx + dby * dby + dbz * dbz);
                            if (r2 < 1e-12) coeff = 0;
                        }
                        double cx = oy * daz - oz * day;
                        double cy = oz * dax - ox * daz;
                        double cz = ox * day - oy * dax;
                        ux += cx * coeff;
                        uy += cy * coeff;
                        uz += cz * coeff;
                    }
                }
        u3[t] += ux;
        u3[M + t] += uy;
        u3[2 * (size_t)M + t] += uz;
    }
    return pairs;
}

/* HFS/BiotSavartSolverImp.cpp:756-816 (computeFarFieldBuffer) followed by
 * :410-516 (evaluateVelocity), non-VIC branch.  Evaluation points are not
 * reordered: each point's result is independent of the evaluation order. */
extern "C" int orc_pppm(const orc_params *prm, uint32_t N, const float *vort_pos4,
                        const double *ax, const double *ay, const double *az,
                        uint32_t M, const float *eval_a4, const float *eval_b4,
                        int is_segment, double *u, double *v, double *w, orc_dump *dump) {
    if (!prm || N == 0 || prm->n < 2) return 1;
    const uint32_t n = prm->n;
    const size_t C = (size_t)n * n * n;
    const F4 *vp = as_f4(vort_pos4);

    double origin[3], L;
    if (prm->domain_mode == 1) {
        origin[0] = prm->fixed_origin[0]; origin[1] = prm->fixed_origin[1];
        origin[2] = prm->fixed_origin[2]; L = prm->fixed_length;
    } else {
        orc_set_domain(vort_pos4, N, origin, &L);
    }
    /* setSpatialHashGrid(n, L/n as float, origin as float3), PH/SpaceHashClass.h:46-54 */
    const float h_f = (float)(L / (double)n);
    const float of[3] = {(float)origin[0], (float)origin[1], (float)origin[2]};
    const double cell_h = (double)h_f;

    std::vector<uint32_t> key(N), idx(N), start(C), end(C);
    orc_calc_hash(vort_pos4, N, n, h_f, of, key.data(), idx.data());
    orc_sort_by_key(key.data(), idx.data(), N);
    orc_find_cell_start(key.data(), N, (uint32_t)C, start.data(), end.data());

    std::vector<F4> spos(N);
    std::vector<double> salpha(3 * (size_t)N);
    for (uint32_t t = 0; t < N; t++) {
        spos[t] = vp[idx[t]];
        salpha[t] = ax[idx[t]];
        salpha[N + t] = ay[idx[t]];
        salpha[2 * (size_t)N + t] = az[idx[t]];
    }

    std::vector<double> gvort(3 * C), rhs(3 * C), psi(3 * C), gu(3 * C), far(3 * C);
    const double h2f = (double)(h_f * h_f); /* getCellSize().x squared in float, :557 */
    for (int c = 0; c < 3; c++) {
        orc_p2m(start.data(), end.data(), reinterpret_cast<const float *>(spos.data()),
                salpha.data() + c * (size_t)N, cell_h, n, N, origin, gvort.data() + c * C);
        for (size_t q = 0; q < C; q++) rhs[c * C + q] = gvort[c * C + q] * h2f * -1.0;
    }
    for (int c = 0; c < 3; c++) {
        int32_t cyc = 0; double rr = 0;
        orc_mg_solve(psi.data() + c * C, rhs.data() + c * C, n, prm->mg_mode, prm->coarse_mode,
                     prm->mg_tol, prm->mg_max_cycles, &cyc, &rr);
        if (dump && dump->mg_cycles) dump->mg_cycles[c] = cyc;
        if (dump && dump->mg_relres) dump->mg_relres[c] = rr;
    }
    orc_curl(psi.data(), gu.data(), n, cell_h);
    if (prm->K >= 0)
        orc_farfield(gvort.data(), gu.data(), far.data(), n, prm->K, cell_h);
    else
        far = gu; /* BiotSavartComputeFarField is a no-op for K < 0 (:2640) */

    std::vector<double> U(3 * (size_t)M, 0.0);
    orc_interp(eval_a4, M, far.data(), n, cell_h, origin, U.data());
    if (dump && dump->u_far_only) std::memcpy(dump->u_far_only, U.data(), sizeof(double) * 3 * M);
    uint64_t pairs = 0;
    if (prm->K >= 0)
        pairs = orc_pp(start.data(), end.data(), eval_a4, eval_b4, is_segment,
                       reinterpret_cast<const float *>(spos.data()), salpha.data(), U.data(), n,
                       cell_h, prm->K, M, N, origin, prm->a);
    for (uint32_t t = 0; t < M; t++) {
        u[t] = U[t];
        v[t] = U[M + t];
        w[t] = U[2 * (size_t)M + t];
    }
    if (dump) {
        if (dump->origin) std::memcpy(dump->origin, origin, sizeof(origin));
        if (dump->length) *dump->length = L;
        if (dump->h_f) *dump->h_f = h_f;
        if (dump->vort_key) std::memcpy(dump->vort_key, key.data(), sizeof(uint32_t) * N);
        if (dump->vort_idx) std::memcpy(dump->vort_idx, idx.data(), sizeof(uint32_t) * N);
        if (dump->cell_start) std::memcpy(dump->cell_start, start.data(), sizeof(uint32_t) * C);
        if (dump->cell_end) std::memcpy(dump->cell_end, end.data(), sizeof(uint32_t) * C);
        if (dump->grid_vort) std::memcpy(dump->grid_vort, gvort.data(), sizeof(double) * 3 * C);
        if (dump->psi) std::memcpy(dump->psi, psi.data(), sizeof(double) * 3 * C);
        if (dump->grid_u) std::memcpy(dump->grid_u, gu.data(), sizeof(double) * 3 * C);
        if (dump->far_u) std::memcpy(dump->far_u, far.data(), sizeof(double) * 3 * C);
        if (dump->pairs) *dump->pairs = pairs;
    }
    return 0;
}

/* BiotSavartSolver::sortVort (HFS/BiotSavartSolverImp.cpp:733-755) on the
 * centres, then ParticleGaussianSmooth (HFS/GPU_kernel.cu:3327-3438): for each
 * centre t, with (i, j, k) = floor(float(x_t - origin) / h), the weighted mean
 * of the strengths d over all vortices hashed into the 5^3 cells around
 * (i, j, k) inside the grid, weights exp(-|x_p - x_t|^2 / (2 nu^2)); a weight
 * sum below 1e-12 is replaced by 1e24. */
extern "C" void orc_gaussian_smooth(const orc_params *prm, uint32_t N, const float *cent4_in, const double *dx_,
                                    const double *dy_, const double *dz_, double nu, double *ox, double *oy,
                                    double *oz) {
    const F4 *cent = reinterpret_cast<const F4 *>(cent4_in);
    const float *cent4 = cent4_in;
    double origin[3], L;
    if (prm->domain_mode == 1) {
        origin[0] = prm->fixed_origin[0]; origin[1] = prm->fixed_origin[1];
        origin[2] = prm->fixed_origin[2]; L = prm->fixed_length;
    } else {
        orc_set_domain(cent4, N, origin, &L);
    }
    const uint32_t n = prm->n;
    const size_t C = (size_t)n * n * n;
    const float h_f = (float)(L / (double)n);
    const float of[3] = {(float)origin[0], (float)origin[1], (float)origin[2]};
    const double invh = 1.0 / (double)h_f;
    std::vector<uint32_t> key(N), idx(N), start(C), end(C);
    orc_calc_hash(cent4, N, n, h_f, of, key.data(), idx.data());
    orc_sort_by_key(key.data(), idx.data(), N);
    orc_find_cell_start(key.data(), N, (uint32_t)C, start.data(), end.data());
    const int d = (int)n;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t t = 0; t < (int64_t)N; t++) {
        const float ax = (float)((double)cent[t].x - origin[0]);
        const float ay = (float)((double)cent[t].y - origin[1]);
        const float az = (float)((double)cent[t].z - origin[2]);
        // a cell more than two outside the grid sees no in-grid cell; clamping
        // keeps the int conversion defined for centres far outside a fixed domain
        auto cell = [&](float r) {
            const double q = std::floor((double)r * invh);
            return !(q >= -3.0) ? -3 : (q > (double)(d + 2) ? d + 2 : (int)q);
        };
        const int i = cell(ax), j = cell(ay), k = cell(az);
        double wx = 0, wy = 0, wz = 0, tw = 0;
        for (int kk = k - 2; kk <= k + 2; kk++)
            for (int jj = j - 2; jj <= j + 2; jj++)
                for (int ii = i - 2; ii <= i + 2; ii++) {
                    if (!(kk >= 0 && kk < d && jj >= 0 && jj < d && ii >= 0 && ii < d)) continue;
                    const size_t c = gidx(ii, jj, kk, d);
                    if (start[c] == 0xFFFFFFFFu) continue;
                    for (uint32_t p = start[c]; p < end[c]; p++) {
                        const uint32_t q = idx[p];
                        const float bx = (float)((double)cent[q].x - origin[0]);
                        const float by = (float)((double)cent[q].y - origin[1]);
                        const float bz = (float)((double)cent[q].z - origin[2]);
                        const double dx = (double)(float)(bx - ax), dy = (double)(float)(by - ay),
                                     dz = (double)(float)(bz - az);
                        const double dsq = dx * dx + dy * dy + dz * dz;
                        const double w = std::exp(-dsq / (2 * nu * nu));
                        tw += w;
                        wx += w * dx_[q];
                        wy += w * dy_[q];
                        wz += w * dz_[q];
                    }
                }
        if (tw < 1e-12) tw = 1e+24;
        ox[t] = wx / tw;
        oy[t] = wy / tw;
        oz[t] = wz / tw;
    }
}

/* HFS/VortexSimulationSystemImp.cpp:90-125 and 127-143, 277-336, 466-525;
 * HFS/GPU_kernel.cu:3118-3254 (move, ComputeVortex, ComputePosb, ComputePosa),
 * 3327-3438 (ParticleGaussianSmooth), 3440-3459 (VectorAdd). */
extern "C" int orc_vortex_step(const orc_params *prm, uint32_t N, float *cent4, double *vx, double *vy,
                               double *vz, double dt, double h_seg, double nu, float *enda4_out,
                               float *endb4_out, uint32_t P, float *passive4, double *pu, double *pv,
                               double *pw) {
    if (!prm || N == 0) return 1;
    F4 *cent = reinterpret_cast<F4 *>(cent4);
    std::vector<F4> enda(N), endb(N);
    std::vector<double> kappa(N);
    // convertVortToSeg: ComputePosb(posa = cent, posc = enda, posb = endb)
    for (uint32_t i = 0; i < N; i++) {
        const double sx = vx[i], sy = vy[i], sz = vz[i];
        const double l = std::sqrt(sx * sx + sy * sy + sz * sz);
        enda[i] = cent[i];
        endb[i] = cent[i];
        if (l < h_seg) {
            kappa[i] = 1;
            endb[i].x = (float)(cent[i].x + 0.5 * sx);
            endb[i].y = (float)(cent[i].y + 0.5 * sy);
            endb[i].z = (float)(cent[i].z + 0.5 * sz);
            enda[i].x = (float)(cent[i].x - 0.5 * sx);
            enda[i].y = (float)(cent[i].y - 0.5 * sy);
            enda[i].z = (float)(cent[i].z - 0.5 * sz);
        } else {
            kappa[i] = l / h_seg;
            endb[i].x = (float)(cent[i].x + 0.5 * sx / l * h_seg);
            endb[i].y = (float)(cent[i].y + 0.5 * sy / l * h_seg);
            endb[i].z = (float)(cent[i].z + 0.5 * sz / l * h_seg);
            enda[i].x = (float)(cent[i].x - 0.5 * sx / l * h_seg);
            enda[i].y = (float)(cent[i].y - 0.5 * sy / l * h_seg);
            enda[i].z = (float)(cent[i].z - 0.5 * sz / l * h_seg);
        }
    }
    // computeURotation: velocities at both ends, segment mode against the centre
    std::vector<double> ub(3 * (size_t)N), ua(3 * (size_t)N);
    orc_pppm(prm, N, cent4, vx, vy, vz, N, reinterpret_cast<const float *>(endb.data()), cent4, 1, ub.data(),
             ub.data() + N, ub.data() + 2 * (size_t)N, nullptr);
    orc_pppm(prm, N, cent4, vx, vy, vz, N, reinterpret_cast<const float *>(enda.data()), cent4, 1, ua.data(),
             ua.data() + N, ua.data() + 2 * (size_t)N, nullptr);
    // computeURotation, tracers and heat (evaluateBiotSavart, VSSImp.cpp:1195-1244):
    // plain evaluation (is_segment 0) with the same far field, then move_particle
    if (P > 0) {
        orc_pppm(prm, N, cent4, vx, vy, vz, P, passive4, passive4, 0, pu, pv, pw, nullptr);
        F4 *q = reinterpret_cast<F4 *>(passive4);
        for (uint32_t i = 0; i < P; i++) {
            const double x = (double)q[i].x + pu[i] * dt;
            const double y = (double)q[i].y + pv[i] * dt;
            const double z = (double)q[i].z + pw[i] * dt;
            q[i].x = (float)x; q[i].y = (float)y; q[i].z = (float)z; q[i].w = 0.f;
        }
    }
    // applyFlow: move_particle on both ends (w = 0), then ComputePosa
    auto move = [&](std::vector<F4> &p, const std::vector<double> &u) {
        for (uint32_t i = 0; i < N; i++) {
            const double x = (double)p[i].x + u[i] * dt;
            const double y = (double)p[i].y + u[N + i] * dt;
            const double z = (double)p[i].z + u[2 * (size_t)N + i] * dt;
            p[i].x = (float)x; p[i].y = (float)y; p[i].z = (float)z; p[i].w = 0.f;
        }
    };
    move(enda, ua);
    move(endb, ub);
    for (uint32_t i = 0; i < N; i++) {
        cent[i].x = (float)(0.5 * (double)(endb[i].x + enda[i].x));
        cent[i].y = (float)(0.5 * (double)(endb[i].y + enda[i].y));
        cent[i].z = (float)(0.5 * (double)(endb[i].z + enda[i].z));
    }
    // convertSegToVort: dvort = kappa * (endb - enda) - vort; computeStretching:
    // dvort = 1 * vort + 1 * dvort
    std::vector<double> dv(3 * (size_t)N);
    for (uint32_t i = 0; i < N; i++) {
        const double s[3] = {(double)(float)(endb[i].x - enda[i].x), (double)(float)(endb[i].y - enda[i].y),
                             (double)(float)(endb[i].z - enda[i].z)};
        const double v[3] = {vx[i], vy[i], vz[i]};
        for (int c = 0; c < 3; c++) {
            const double d = kappa[i] * s[c] - v[c];
            dv[c * (size_t)N + i] = 1 * v[c] + 1 * d;
        }
    }
    // computeStretching: hash of the new centres + ParticleGaussianSmooth
    std::vector<double> out(3 * (size_t)N);
    orc_gaussian_smooth(prm, N, cent4, dv.data(), dv.data() + N, dv.data() + 2 * (size_t)N, nu, out.data(),
                        out.data() + N, out.data() + 2 * (size_t)N);
    // vort = 0 * vort + 1 * dvort
    for (uint32_t i = 0; i < N; i++) {
        vx[i] = 0 * vx[i] + 1 * out[i];
        vy[i] = 0 * vy[i] + 1 * out[N + i];
        vz[i] = 0 * vz[i] + 1 * out[2 * (size_t)N + i];
    }
    if (enda4_out) std::memcpy(enda4_out, enda.data(), sizeof(F4) * N);
    if (endb4_out) std::memcpy(endb4_out, endb.data(), sizeof(F4) * N);
    return 0;
}

/* FP64 O(N*M) sum with the same smoothing kernel as the near field,
 * c(r) = (1 - exp(-(r/a)^3)) / (4 pi r^3), on the float input positions
 * promoted to double; r = 0 and (for segments) |x_b - y_p| = 0 excluded. */
extern "C" void orc_direct_sum(uint32_t N, const float *vort_pos4, const double *ax,
                               const double *ay, const double *az, uint32_t M,
                               const float *eval_a4, const float *eval_b4, int is_segment,
                               double a, double *u, double *v, double *w) {
    const F4 *vp = as_f4(vort_pos4), *ea = as_f4(eval_a4), *eb = as_f4(eval_b4);
    const double inva = 1.0 / a;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t t = 0; t < (int64_t)M; t++) {
        const double xa = ea[t].x, ya = ea[t].y, za = ea[t].z;
        double xb = 0, yb = 0, zb = 0;
        if (is_segment == 1) { xb = eb[t].x; yb = eb[t].y; zb = eb[t].z; }
        double sx = 0, sy = 0, sz = 0;
        for (uint32_t p = 0; p < N; p++) {
            double dx = xa - (double)vp[p].x, dy = ya - (double)vp[p].y, dz = za - (double)vp[p].z;
            double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 == 0.0) continue;
            if (is_segment == 1) {
                double ex = xb - (double)vp[p].x, ey = yb - (double)vp[p].y, ez = zb - (double)vp[p].z;
                if (ex == 0.0 && ey == 0.0 && ez == 0.0) continue;
            }
            double r = std::sqrt(r2);
            double s = r * inva;
            double s3 = s * s * s;
            double c = (s3 > 1e-8) ? -std::expm1(-s3) / (kFourPi * r2 * r)
                                   : (1.0 - 0.5 * s3) * inva * inva * inva / kFourPi;
            double ox = ax[p], oy = ay[p], oz = az[p];
            sx += (oy * dz - oz * dy) * c;
            sy += (oz * dx - ox * dz) * c;
            sz += (ox * dy - oy * dx) * c;
        }
        u[t] = sx; v[t] = sy; w[t] = sz;
    }
}

/* VortexSimulationSystem::setDensityDomain (HFS/VortexSimulationSystemImp.cpp:
 * 336-366): 1.2 x the largest bounding-box edge, centred on the box. */
extern "C" void orc_density_domain(const float *pos4, uint32_t N, double *origin3, double *length) {
    const F4 *pos = as_f4(pos4);
    double maxx, minx, maxy, miny, maxz, minz;
    maxx = minx = pos[0].x;
    maxy = miny = pos[0].y;
    maxz = minz = pos[0].z;
    for (uint32_t i = 1; i < N; i++) {
        if (pos[i].x < minx) minx = pos[i].x; else if (pos[i].x > maxx) maxx = pos[i].x;
        if (pos[i].y < miny) miny = pos[i].y; else if (pos[i].y > maxy) maxy = pos[i].y;
        if (pos[i].z < minz) minz = pos[i].z; else if (pos[i].z > maxz) maxz = pos[i].z;
    }
    const double L = 1.2 * std::max(std::max(maxx - minx, maxy - miny), maxz - minz);
    origin3[0] = (minx + 0.5 * (maxx - minx)) - 0.5 * L;
    origin3[1] = (miny + 0.5 * (maxy - miny)) - 0.5 * L;
    origin3[2] = (minz + 0.5 * (maxz - minz)) - 0.5 * L;
    *length = L;
}

/* HFS/GPU_kernel.cu:79-110 interpolate_weights2 / poly_shape2: (1 - r)^4 of the
 * squared distance r in cells, zero for r >= 1. */
static double weight_quartic(double gx, double gy, double gz, double px, double py, double pz) {
    const double dx = gx - px, dy = gy - py, dz = gz - pz;
    const double r = dx * dx + dy * dy + dz * dz;
    const double rr = std::fabs(r);
    const double r1 = 1 - rr;
    const double r2 = r1 * r1;
    const double r4 = r2 * r2;
    return rr < 1 ? r4 : 0.0;
}

/* HFS/GPU_kernel.cu:52-90 interpolate_weights / poly_shape: trilinear hat. */
static double hat(double r) {
    const double rr = std::fabs(r);
    return rr < 1 ? 1 - rr : 0.0;
}

/* VortexSimulationSystem::addBaroclinicForce (HFS/VortexSimulationSystemImp.cpp:
 * 369-465): density grid of edge min(floor(L / 0.2) + 1, 200) over the heat
 * particles' 1.2 x box; the heat particles hashed on it; AssignDensity
 * (HFS/GPU_kernel.cu:3655-3740) = quartic-weighted mean of the particles' heat
 * over the 5^3 hash cells around each grid cell, an empty hash cell adding its
 * centre's weight with zero heat; GradDensity (3742-3797) = periodic central
 * differences; ParticleGetBaroclinic (3800-3898) = the gradient interpolated
 * (trilinear hat over 5^3 cells) at each vortex, crossed with (0, 10, 0), times
 * 5 dt * 0.1, added to the strength.  Returns the grid edge (0 = nothing done:
 * no heat particles or a zero-size box).  rho / grad (may be NULL) receive the
 * grids when dim^3 <= cap. */
extern "C" uint32_t orc_baroclinic(uint32_t H, const float *heat4, const float *life, uint32_t N,
                                   const float *cent4, double *vx, double *vy, double *vz, double dt,
                                   double *origin_out, double *h_out, float *rho_out, float *grad_out,
                                   size_t cap) {
    if (H == 0) return 0;
    double origin[3], L;
    orc_density_domain(heat4, H, origin, &L);
    if (!(L > 0.0)) return 0;
    double h = 0.2;
    uint32_t dim = (uint32_t)(std::floor(L / h) + 1);
    dim = std::min(std::max((uint32_t)0, dim), (uint32_t)200);
    h = L / (double)dim;
    const int d = (int)dim;
    const size_t C = (size_t)dim * dim * dim;
    const float h_f = (float)(L / (double)dim);
    const float of[3] = {(float)origin[0], (float)origin[1], (float)origin[2]};
    std::vector<uint32_t> key(H), idx(H), start(C), end(C);
    orc_calc_hash(heat4, H, dim, h_f, of, key.data(), idx.data());
    orc_sort_by_key(key.data(), idx.data(), H);
    orc_find_cell_start(key.data(), H, (uint32_t)C, start.data(), end.data());
    const F4 *hp = as_f4(heat4);
    // AssignDensity
    std::vector<float> rho(C);
    const double invh = 1.0 / h;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t c = 0; c < (int64_t)C; c++) {
        const int i = (int)(c % d), j = (int)((c / d) % d), k = (int)(c / ((int64_t)d * d));
        const double gx = i + 0.5, gy = j + 0.5, gz = k + 0.5;
        double sum = 0, tw = 0;
        for (int kk = k - 2; kk <= k + 2; kk++)
            for (int jj = j - 2; jj <= j + 2; jj++)
                for (int ii = i - 2; ii <= i + 2; ii++) {
                    if (!(kk >= 0 && kk < d && jj >= 0 && jj < d && ii >= 0 && ii < d)) continue;
                    const size_t r = gidx(ii, jj, kk, d);
                    if (start[r] != 0xFFFFFFFFu) {
                        for (uint32_t p = start[r]; p < end[r]; p++) {
                            const uint32_t q = idx[p];
                            const float px = (float)((double)hp[q].x - origin[0]);
                            const float py = (float)((double)hp[q].y - origin[1]);
                            const float pz = (float)((double)hp[q].z - origin[2]);
                            const double w = weight_quartic(gx, gy, gz, px * invh, py * invh, pz * invh);
                            sum += w * (double)life[q];
                            tw += w;
                        }
                    } else {
                        // empty hash cell: its centre's weight, zero heat
                        tw += weight_quartic(gx, gy, gz, ii + 0.5, jj + 0.5, kk + 0.5);
                    }
                }
        if (tw < 1e-12) tw = 1e+24;
        rho[c] = (float)(sum / tw);
    }
    // GradDensity (periodic)
    std::vector<float> grad(3 * C);
    for (int k = 0; k < d; k++)
        for (int j = 0; j < d; j++)
            for (int i = 0; i < d; i++) {
                const size_t c = gidx(i, j, k, d);
                const double t = rho[gidx(i, (j + 1) % d, k, d)], dn = rho[gidx(i, (j + d - 1) % d, k, d)];
                const double l = rho[gidx((i + d - 1) % d, j, k, d)], r = rho[gidx((i + 1) % d, j, k, d)];
                const double f = rho[gidx(i, j, (k + d - 1) % d, d)], b = rho[gidx(i, j, (k + 1) % d, d)];
                grad[3 * c + 0] = (float)((r - l) * 0.5 * invh);
                grad[3 * c + 1] = (float)((t - dn) * 0.5 * invh);
                grad[3 * c + 2] = (float)((b - f) * 0.5 * invh);
            }
    // ParticleGetBaroclinic
    const double inv_hf = 1.0 / (double)h_f;
    const double dt_beta = dt * 5.0;
    const F4 *cp = as_f4(cent4);
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < (int64_t)N; t++) {
        const float px = (float)((double)cp[t].x - origin[0]);
        const float py = (float)((double)cp[t].y - origin[1]);
        const float pz = (float)((double)cp[t].z - origin[2]);
        auto cell = [&](float r) {
            const double q = std::floor(r * inv_hf);
            return !(q >= -3.0) ? -3 : (q > (double)(d + 2) ? d + 2 : (int)q);
        };
        const int i = cell(px), j = cell(py), k = cell(pz);
        double sx = 0, sy = 0, sz = 0;
        for (int kk = k - 2; kk <= k + 2; kk++)
            for (int jj = j - 2; jj <= j + 2; jj++)
                for (int ii = i - 2; ii <= i + 2; ii++) {
                    if (!(kk >= 0 && kk < d && jj >= 0 && jj < d && ii >= 0 && ii < d)) continue;
                    const size_t c = gidx(ii, jj, kk, d);
                    const double w = hat((ii + 0.5) - px * inv_hf) * hat((jj + 0.5) - py * inv_hf) *
                                     hat((kk + 0.5) - pz * inv_hf);
                    sx += grad[3 * c + 0] * w;
                    sy += grad[3 * c + 1] * w;
                    sz += grad[3 * c + 2] * w;
                }
        const double v[3] = {0, 10, 0};
        const double bx = sy * v[2] - sz * v[1], by = sz * v[0] - sx * v[2], bz = sx * v[1] - sy * v[0];
        vx[t] += dt_beta * 0.1 * bx;
        vy[t] += dt_beta * 0.1 * by;
        vz[t] += dt_beta * 0.1 * bz;
    }
    if (origin_out) { origin_out[0] = origin[0]; origin_out[1] = origin[1]; origin_out[2] = origin[2]; }
    if (h_out) *h_out = h;
    if (rho_out && C <= cap) std::memcpy(rho_out, rho.data(), sizeof(float) * C);
    if (grad_out && C <= cap) std::memcpy(grad_out, grad.data(), sizeof(float) * 3 * C);
    return dim;
}

/* ------------------------------------------------------------------------
 * Scalar PPPM: PotentialFieldSolver (HFS/PotentialFieldSolver.cpp:45-739),
 * kernels HFS/GPU_kernel.cu:524-1748 and 2977-3115.
 * ------------------------------------------------------------------------ */
namespace {

/* HFS/GPU_kernel.cu:204-211 compute_r: 4 pi |r1 - r2|, or 1e12 when coincident. */
double compute_r_dev(double ax, double ay, double az, double bx, double by, double bz) {
    const double r_sqr = (ax - bx) * (ax - bx) + (ay - by) * (ay - by) + (az - bz) * (az - bz);
    return r_sqr > 1e-12 ? kFourPi * std::sqrt(r_sqr) : 1e+12;
}

/* HFS/GPU_kernel.cu:546-601 compute_gradient_kernel: periodic central
 * differences, direction * (right - left) * 0.5 * invh per axis. */
void periodic_gradient(const double *phi, double *g3, int d, double invh, double direction) {
    const size_t C = (size_t)d * d * d;
    for (int k = 0; k < d; k++)
        for (int j = 0; j < d; j++)
            for (int i = 0; i < d; i++) {
                const size_t c = gidx(i, j, k, d);
                const double t = phi[gidx(i, (j + 1) % d, k, d)], dn = phi[gidx(i, (j + d - 1) % d, k, d)];
                const double l = phi[gidx((i + d - 1) % d, j, k, d)], r = phi[gidx((i + 1) % d, j, k, d)];
                const double f = phi[gidx(i, j, (k + d - 1) % d, d)], b = phi[gidx(i, j, (k + 1) % d, d)];
                g3[c] = direction * (r - l) * 0.5 * invh;
                g3[C + c] = direction * (t - dn) * 0.5 * invh;
                g3[2 * C + c] = direction * (b - f) * 0.5 * invh;
            }
}

/* Trilinear hat weights over the 5^3 cells around the point's cell
 * (HFS/GPU_kernel.cu:1520-1676); no write when the point's cell is outside
 * the grid (the caller's value stays 0). */
template <typename Get>
bool interp5(float px, float py, float pz, double invh, int d, Get get) {
    const int i = (int)std::floor((double)px * invh), j = (int)std::floor((double)py * invh),
              k = (int)std::floor((double)pz * invh);
    if (!(i >= 0 && i < d && j >= 0 && j < d && k >= 0 && k < d)) return false;
    for (int kk = k - 2; kk <= k + 2; kk++)
        for (int jj = j - 2; jj <= j + 2; jj++)
            for (int ii = i - 2; ii <= i + 2; ii++) {
                if (!(kk >= 0 && kk < d && jj >= 0 && jj < d && ii >= 0 && ii < d)) continue;
                const double gx = (double)(float)((double)ii + 0.5), gy = (double)(float)((double)jj + 0.5),
                             gz = (double)(float)((double)kk + 0.5);
                auto hat = [](double r) { const double rr = std::fabs(r); return rr < 1 ? 1 - rr : 0.0; };
                const double w = hat(gx - (double)px * invh) * hat(gy - (double)py * invh) * hat(gz - (double)pz * invh);
                get(gidx(ii, jj, kk, d), w);
            }
    return true;
}

}  // namespace

/* PotentialFieldSolver::setDomain (:343-373): 2 x the bounding box. */
extern "C" void orc_potential_domain(const float *pos4, uint32_t N, double *origin3, double *length) {
    const F4 *pos = as_f4(pos4);
    double maxx, minx, maxy, miny, maxz, minz;
    maxx = minx = pos[0].x;
    maxy = miny = pos[0].y;
    maxz = minz = pos[0].z;
    for (uint32_t i = 1; i < N; i++) {
        if (pos[i].x < minx) minx = pos[i].x; else if (pos[i].x > maxx) maxx = pos[i].x;
        if (pos[i].y < miny) miny = pos[i].y; else if (pos[i].y > maxy) maxy = pos[i].y;
        if (pos[i].z < minz) minz = pos[i].z; else if (pos[i].z > maxz) maxz = pos[i].z;
    }
    const double dl = 2.0 * std::max(std::max(maxx - minx, maxy - miny), maxz - minz);
    origin3[0] = (minx + 0.5 * (maxx - minx)) - 0.5 * dl;
    origin3[1] = (miny + 0.5 * (maxy - miny)) - 0.5 * dl;
    origin3[2] = (minz + 0.5 * (maxz - minz)) - 0.5 * dl;
    *length = dl;
}

/* computeFarFieldBuffer (:695-707) + evaluateGradient (:441-526), or with
 * scalar != 0 computeFarFieldPotentialBuffer (:726-737) +
 * evaluateScalarPotential (:708-739).  Masses at pos4 (N), evaluation points
 * eval4 (M); out receives the gradient (3 x M, caller order) or the potential
 * (M).  dump (optional) receives origin[3], L, density[C], rhs[C] (after the
 * Dirichlet data), phi[C] (after the three full-multigrid calls), and for
 * the gradient far[3C]. */
extern "C" int orc_potential(uint32_t n, int K, int scalar, uint32_t N, const float *pos4, const double *mass,
                             uint32_t M, const float *eval4, double *out, double *dump_origin, double *dump_density,
                             double *dump_rhs, double *dump_phi, double *dump_far, double *dump_monopole) {
    if (N == 0 || n < 2) return 1;
    const int d = (int)n;
    const size_t C = (size_t)d * d * d;
    double origin[3], L;
    orc_potential_domain(pos4, N, origin, &L);
    // m_ParticleToMesh (:527-609): hash, reorder, P2M, RHS, monopole, Dirichlet data
    const float h_f = (float)(L / (double)n);
    const float of[3] = {(float)origin[0], (float)origin[1], (float)origin[2]};
    const double cell_h = (double)h_f;
    std::vector<uint32_t> key(N), idx(N), start(C), end(C);
    orc_calc_hash(pos4, N, n, h_f, of, key.data(), idx.data());
    orc_sort_by_key(key.data(), idx.data(), N);
    orc_find_cell_start(key.data(), N, (uint32_t)C, start.data(), end.data());
    const F4 *pos = as_f4(pos4);
    std::vector<F4> spos(N);
    std::vector<double> smass(N);
    for (uint32_t s = 0; s < N; s++) { spos[s] = pos[idx[s]]; smass[s] = mass[idx[s]]; }
    std::vector<double> density(C), rhs(C);
    orc_p2m(start.data(), end.data(), reinterpret_cast<const float *>(spos.data()), smass.data(), cell_h, n, N,
            origin, density.data());
    const double h2 = (double)(h_f * h_f);
    for (size_t c = 0; c < C; c++) rhs[c] = density[c] * h2 * -1.0;
    double total_weight = 0, total_mass = 0;
    for (uint32_t s = 0; s < N; s++) { total_weight += std::fabs(smass[s]); total_mass += smass[s]; }
    double cx = 0, cy = 0, cz = 0;
    for (uint32_t s = 0; s < N; s++) {
        cx += spos[s].x * std::fabs(smass[s]);
        cy += spos[s].y * std::fabs(smass[s]);
        cz += spos[s].z * std::fabs(smass[s]);
    }
    cx = cx / total_weight; cy = cy / total_weight; cz = cz / total_weight;
    // applyDirichlet (HFS/GPU_kernel.cu:2977-3115): ghost values of the
    // monopole moved to the right-hand side of the boundary cells
    for (int k = 0; k < d; k++)
        for (int j = 0; j < d; j++)
            for (int i = 0; i < d; i++) {
                const size_t c = gidx(i, j, k, d);
                auto ghost = [&](double gi, double gj, double gk) {
                    const double wx = gi * cell_h + origin[0], wy = gj * cell_h + origin[1], wz = gk * cell_h + origin[2];
                    rhs[c] -= total_mass / compute_r_dev(wx, wy, wz, cx, cy, cz);
                };
                if (i == 0) ghost((double)i - 1.0 + 0.5, (double)j + 0.5, (double)k + 0.5);
                if (i == d - 1) ghost((double)i + 1.0 + 0.5, (double)j + 0.5, (double)k + 0.5);
                if (j == 0) ghost((double)i + 0.5, (double)j - 1.0 + 0.5, (double)k + 0.5);
                if (j == d - 1) ghost((double)i + 0.5, (double)j + 1.0 + 0.5, (double)k + 0.5);
                if (k == 0) ghost((double)i + 0.5, (double)j + 0.5, (double)k - 1.0 + 0.5);
                if (k == d - 1) ghost((double)i + 0.5, (double)j + 0.5, (double)k + 1.0 + 0.5);
            }
    // m_SolvePoisson (:610-621): phi = 0, three full-multigrid calls
    std::vector<double> phi(C, 0.0);
    {
        MG mg(d, 1);
        std::memcpy(mg.lv[0].b.data(), rhs.data(), sizeof(double) * C);
        for (int it = 0; it < 3; it++) mg.fmg();
        std::memcpy(phi.data(), mg.lv[0].x.data(), sizeof(double) * C);
    }
    if (dump_origin) { dump_origin[0] = origin[0]; dump_origin[1] = origin[1]; dump_origin[2] = origin[2]; dump_origin[3] = L; }
    if (dump_density) std::memcpy(dump_density, density.data(), sizeof(double) * C);
    if (dump_rhs) std::memcpy(dump_rhs, rhs.data(), sizeof(double) * C);
    if (dump_phi) std::memcpy(dump_phi, phi.data(), sizeof(double) * C);
    if (dump_monopole) { dump_monopole[0] = cx; dump_monopole[1] = cy; dump_monopole[2] = cz; dump_monopole[3] = total_mass; }
    const double invh = 1.0 / cell_h;
    const F4 *ev = as_f4(eval4);
    const double G = 1.0;
    if (!scalar) {
        // m_ComputeGradient + PotentialComputeFarField (HFS/GPU_kernel.cu:988-1197)
        std::vector<double> grad(3 * C), far(3 * C);
        periodic_gradient(phi.data(), grad.data(), d, invh, 1.0);
        const size_t W3 = K >= 0 ? (size_t)(2 * K + 1) * (2 * K + 1) * (2 * K + 1) : 1;
        std::vector<double> table(3 * W3);
        if (K >= 0) orc_farfield_table(K, cell_h, table.data());
        const int W = 2 * K + 1;
        for (int k = 0; k < d; k++)
            for (int j = 0; j < d; j++)
                for (int i = 0; i < d; i++) {
                    const size_t c = gidx(i, j, k, d);
                    double fm[3] = {0, 0, 0};
                    if (K >= 0)
                        for (int kk = k - K; kk <= k + K; kk++)
                            for (int jj = j - K; jj <= j + K; jj++)
                                for (int ii = i - K; ii <= i + K; ii++) {
                                    double m = 0, dx[3] = {0, 0, 0};
                                    if (kk >= 0 && kk < d && jj >= 0 && jj < d && ii >= 0 && ii < d) {
                                        m = G * density[gidx(ii, jj, kk, d)] * (cell_h * cell_h * cell_h);
                                        if (!(kk == k && jj == j && ii == i)) {
                                            const double *t = &table[3 * ((size_t)((kk - k + K) * W + (jj - j + K)) * W + (ii - i + K))];
                                            dx[0] = t[0]; dx[1] = t[1]; dx[2] = t[2];
                                        }
                                    }
                                    for (int q = 0; q < 3; q++) fm[q] += dx[q] * m;
                                }
                    for (int q = 0; q < 3; q++) far[q * C + c] = grad[q * C + c] - fm[q];
                }
        if (K >= 0) {
            std::vector<double> phid(C), gd(3 * C);
            for (size_t c = 0; c < C; c++) phid[c] = 0.250580605913965 * density[c] * (cell_h * cell_h) * G;
            periodic_gradient(phid.data(), gd.data(), d, invh, 1.0);
            for (size_t q = 0; q < 3 * C; q++) far[q] -= gd[q];
        } else {
            far = grad;
        }
        if (dump_far) std::memcpy(dump_far, far.data(), sizeof(double) * 3 * C);
        // evaluateGradient: interpolation + Potential_PPCorrMN (a = 0.05) + outside points
        const double cr = ((double)K + 0.5) / invh;
        const float bbmin[3] = {of[0], of[1], of[2]};
        const float bbmax[3] = {(float)(of[0] + L), (float)(of[1] + L), (float)(of[2] + L)};
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t t = 0; t < (int64_t)M; t++) {
            const float px = (float)((double)ev[t].x - origin[0]), py = (float)((double)ev[t].y - origin[1]),
                        pz = (float)((double)ev[t].z - origin[2]);
            double g[3] = {0, 0, 0};
            interp5(px, py, pz, invh, d, [&](size_t c, double w) {
                g[0] += far[c] * w; g[1] += far[C + c] * w; g[2] += far[2 * C + c] * w;
            });
            if (K >= 0) {
                const int i = (int)std::floor((double)px * invh), j = (int)std::floor((double)py * invh),
                          k = (int)std::floor((double)pz * invh);
                const double a = 0.05;
                double f[3] = {0, 0, 0};
                for (int kk = k - K - 1; kk <= k + K + 1; kk++)
                    for (int jj = j - K - 1; jj <= j + K + 1; jj++)
                        for (int ii = i - K - 1; ii <= i + K + 1; ii++) {
                            if (!(kk >= 0 && kk < d && jj >= 0 && jj < d && ii >= 0 && ii < d)) continue;
                            const size_t c = gidx(ii, jj, kk, d);
                            if (start[c] == 0xFFFFFFFFu) continue;
                            for (uint32_t p = start[c]; p < end[c]; p++) {
                                const float qx = (float)((double)spos[p].x - origin[0]);
                                const float qy = (float)((double)spos[p].y - origin[1]);
                                const float qz = (float)((double)spos[p].z - origin[2]);
                                if (!(std::fabs((double)(float)(qx - px)) < cr && std::fabs((double)(float)(qy - py)) < cr &&
                                      std::fabs((double)(float)(qz - pz)) < cr))
                                    continue;
                                const double dx = (float)(qx - px), dy = (float)(qy - py), dz = (float)(qz - pz);
                                const double r1 = std::sqrt(dx * dx + dy * dy + dz * dz);
                                double r3;
                                if (r1 > a) r3 = kFourPi * r1 * r1 * r1;
                                else r3 = (r1 < 1e-12) ? 1e+14 : kFourPi * a * a * a;
                                f[0] += G * dx / r3 * smass[p];
                                f[1] += G * dy / r3 * smass[p];
                                f[2] += G * dz / r3 * smass[p];
                            }
                        }
                for (int q = 0; q < 3; q++) g[q] += f[q];
            }
            // Potentialparticle_outside_kernel (HFS/GPU_kernel.cu:1678-1716): zero outside the grid box
            const double ex = ev[t].x, ey = ev[t].y, ez = ev[t].z;
            if (ex < bbmin[0] || ex > bbmax[0] || ey < bbmin[1] || ey > bbmax[1] || ez < bbmin[2] || ez > bbmax[2])
                g[0] = g[1] = g[2] = 0;
            out[t] = g[0]; out[M + t] = g[1]; out[2 * (size_t)M + t] = g[2];
        }
    } else {
        // PotentialComputeScalarFarField (HFS/GPU_kernel.cu:1200-1298)
        std::vector<double> sphi(phi);
        if (K >= 0)
            for (int k = 0; k < d; k++)
                for (int j = 0; j < d; j++)
                    for (int i = 0; i < d; i++) {
                        double s = 0;
                        for (int kk = k - K; kk <= k + K; kk++)
                            for (int jj = j - K; jj <= j + K; jj++)
                                for (int ii = i - K; ii <= i + K; ii++) {
                                    if (!(kk >= 0 && kk < d && jj >= 0 && jj < d && ii >= 0 && ii < d)) continue;
                                    const double m = G * density[gidx(ii, jj, kk, d)] * (cell_h * cell_h);
                                    double w;
                                    if (i == ii && j == jj && k == kk) w = 0.25;
                                    else {
                                        const double x = (double)ii - (double)i, y = (double)jj - (double)j,
                                                     z = (double)kk - (double)k;
                                        w = 1.0 / (kFourPi * std::sqrt(x * x + y * y + z * z));
                                    }
                                    s += w * m;
                                }
                        sphi[gidx(i, j, k, d)] = phi[gidx(i, j, k, d)] - s;
                    }
        if (dump_far) std::memcpy(dump_far, sphi.data(), sizeof(double) * C);
        const double cr = ((double)K + 0.5) / invh;
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t t = 0; t < (int64_t)M; t++) {
            const float px = (float)((double)ev[t].x - origin[0]), py = (float)((double)ev[t].y - origin[1]),
                        pz = (float)((double)ev[t].z - origin[2]);
            double v = 0;
            interp5(px, py, pz, invh, d, [&](size_t c, double w) { v += sphi[c] * w; });
            if (K >= 0) {
                const int i = (int)std::floor((double)px * invh), j = (int)std::floor((double)py * invh),
                          k = (int)std::floor((double)pz * invh);
                const double qx0 = (double)px * invh, qy0 = (double)py * invh, qz0 = (double)pz * invh;
                const int ilo = qx0 > i + 0.5 ? i - K : i - K - 1, ihi = qx0 > i + 0.5 ? i + K + 1 : i + K;
                const int jlo = qy0 > j + 0.5 ? j - K : j - K - 1, jhi = qy0 > j + 0.5 ? j + K + 1 : j + K;
                const int klo = qz0 > k + 0.5 ? k - K : k - K - 1, khi = qz0 > k + 0.5 ? k + K + 1 : k + K;
                const double a = 0.125;
                double s = 0;
                for (int kk = klo; kk <= khi; kk++)
                    for (int jj = jlo; jj <= jhi; jj++)
                        for (int ii = ilo; ii <= ihi; ii++) {
                            if (!(kk >= 0 && kk < d && jj >= 0 && jj < d && ii >= 0 && ii < d)) continue;
                            const size_t c = gidx(ii, jj, kk, d);
                            if (start[c] == 0xFFFFFFFFu) continue;
                            for (uint32_t p = start[c]; p < end[c]; p++) {
                                const float qx = (float)((double)spos[p].x - origin[0]);
                                const float qy = (float)((double)spos[p].y - origin[1]);
                                const float qz = (float)((double)spos[p].z - origin[2]);
                                if (!(std::fabs((double)(float)(qx - px)) < cr && std::fabs((double)(float)(qy - py)) < cr &&
                                      std::fabs((double)(float)(qz - pz)) < cr))
                                    continue;
                                const double dx = (float)(qx - px), dy = (float)(qy - py), dz = (float)(qz - pz);
                                const double r1 = std::sqrt(dx * dx + dy * dy + dz * dz);
                                double r2;
                                if (r1 > a) r2 = kFourPi * r1;
                                else r2 = (r1 < 1e-12) ? 1e+14 : kFourPi * a;
                                s += G / r2 * smass[p];
                            }
                        }
                v += s;
            }
            out[t] = v;
        }
    }
    return 0;
}
