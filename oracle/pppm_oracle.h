/*
 * CPU oracle for the PPPM vortex-particle velocity evaluation.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain C++17 / OpenMP / FP64 restatement
 * of the reference's BiotSavartSolver::computeFarFieldBuffer +
 * evaluateVelocity path (hybridFastSummation, multigrid, particle_hash).  It is
 * the checker the CUDA path is compared against and the timed CPU baseline.
 * Nothing in the product links it: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py load it.
 *
 * Parity status: PINNED against the reference's own GPU kernels for every
 * stage.  The reference ships no golden vectors and its whole solver cannot be
 * built as shipped (its multigrid's host wrappers and array class include GL
 * headers, and its kernels use the texture-reference API that CUDA 12
 * removed).  Its hash kernels (particle_hash_kernel.cu), its P2M, curl,
 * far-field, interpolation, near-field, segment, move, smoothing, density,
 * baroclinic and PotentialFieldSolver kernels (GPU_kernel.cu) and its FP64
 * multigrid kernels (MultiGrid_kernel.cu, with ref_gpu/texref_compat.h standing
 * in for the texture references) do build from their sources for sm_100a
 * (`make -C oracle refgpu`, ref_gpu/).  The GPU tests run them beside this
 * restatement, stage by stage (tests/test_gpu_ref_kernels.py: keys, order and
 * cell tables bit-exact; grids, velocities and strengths to FP64 round-off).
 * The multigrid's coarsest solve races in the reference (512 threads update x
 * in place with no order), so its psi varies from run to run; this
 * restatement takes the Jacobi reading, one order the race allows, which lies
 * within 1.1e-5 of the reference's psi (velocities within 6.1e-7).  The
 * multigrid is also anchored by known-answer tests (tests/golden/,
 * tests/test_oracle_*.py): the discrete zero-ghost Laplacian's sine
 * eigenmodes, the level rule, and an independent numpy restatement at small
 * sizes; so are the FP32 cell assignment on crafted face / +-1 ulp particles,
 * the closed-form smoothed Biot-Savart kernel for one and two blobs, and the
 * finite-difference Green's-gradient table.
 *
 * Every function cites the reference file:line it restates.  Paths are
 * relative to the reference project root; HFS = hybridFastSummation/
 * hybridFastSummation, MG = multigrid/multigrid, PH = particle_hash/
 * particle_hash.
 */
#ifndef PPPM_ORACLE_H
#define PPPM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Solver options.  mg_mode 0 = the reference schedule (full multigrid followed
 * by one V(4,4) cycle, MG/MultiGrid.cpp:202-250); 1 = converged (further
 * V-cycles until ||b-Ax||_2 <= mg_tol * ||b||_2).  coarse_mode selects the
 * deterministic stand-in for the reference's racy in-place coarsest solve
 * (MG/MultiGrid_kernel.cu:422-498): 0 = in-place sweeps in cell order
 * (Gauss-Seidel), 1 = Jacobi (every read before any write). */
typedef struct {
    uint32_t n;            /* cubic grid edge (gridx == gridy == gridz)        */
    int32_t  K;            /* near-field range in cells                        */
    double   a;            /* smoothing radius (absolute length)               */
    int32_t  domain_mode;  /* 0 = 3x vortex bbox (reference), 1 = fixed        */
    double   fixed_origin[3];
    double   fixed_length;
    int32_t  mg_mode;
    int32_t  coarse_mode;
    double   mg_tol;
    int32_t  mg_max_cycles;
} orc_params;

/* Optional intermediate outputs of orc_pppm (any pointer may be NULL). */
typedef struct {
    double   *origin;      /* [3]                                              */
    double   *length;      /* [1]                                              */
    float    *h_f;         /* [1] cell size as the hash stores it (float)      */
    uint32_t *vort_key;    /* [N] sorted cell keys                             */
    uint32_t *vort_idx;    /* [N] sorted original indices                      */
    uint32_t *cell_start;  /* [n^3]                                            */
    uint32_t *cell_end;    /* [n^3]                                            */
    double   *grid_vort;   /* [3][n^3] P2M result (sum alpha / h^3)            */
    double   *psi;         /* [3][n^3] vector potential                        */
    double   *grid_u;      /* [3][n^3] curl(psi)                               */
    double   *far_u;       /* [3][n^3] far-field velocity                      */
    double   *u_far_only;  /* [3][M] interpolated far field (caller order)     */
    uint64_t *pairs;       /* [1] near-field pairs inside the axis box         */
    int32_t  *mg_cycles;   /* [3] V-cycles run after FMG per component         */
    double   *mg_relres;   /* [3] final ||b-Ax||/||b|| per component           */
} orc_dump;

/* --- individual stages ------------------------------------------------- */
void orc_set_domain(const float *pos4, uint32_t N, double *origin3, double *length);
void orc_calc_hash(const float *pos4, uint32_t N, uint32_t n, float h_f,
                   const float *origin_f3, uint32_t *key, uint32_t *idx);
void orc_sort_by_key(uint32_t *key, uint32_t *idx, uint32_t N);
void orc_find_cell_start(const uint32_t *skey, uint32_t N, uint32_t ncells,
                         uint32_t *start, uint32_t *end);
void orc_p2m(const uint32_t *start, const uint32_t *end, const float *spos4,
             const double *smass, double cell_h, uint32_t n, uint32_t N,
             const double *origin3, double *grid);
int  orc_mg_levels(uint32_t n);
void orc_mg_solve(double *x, const double *b, uint32_t n, int mg_mode,
                  int coarse_mode, double tol, int max_cycles,
                  int32_t *cycles_out, double *relres_out);
void orc_mg_vcycle(double *x, const double *b, uint32_t n, int coarse_mode);
void orc_mg_fmg(double *x, const double *b, uint32_t n, int repeats, int coarse_mode);
double orc_residual_norm(const double *x, const double *b, uint32_t n);
void orc_apply_laplacian(const double *x, double *y, uint32_t n);
void orc_curl(const double *psi3, double *u3, uint32_t n, double h);
void orc_farfield_table(int K, double h, double *table);
void orc_farfield(const double *vort3, const double *u3, double *far3,
                  uint32_t n, int K, double h);
void orc_interp(const float *eval4, uint32_t M, const double *far3, uint32_t n,
                double cell_h, const double *origin3, double *out3);
uint64_t orc_pp(const uint32_t *start, const uint32_t *end,
                const float *eval_a4, const float *eval_b4, int is_segment,
                const float *svort4, const double *salpha3, double *u3,
                uint32_t n, double cell_h, int K, uint32_t M, uint32_t N,
                const double *origin3, double a);

/* --- whole path: computeFarFieldBuffer + evaluateVelocity --------------- */
int orc_pppm(const orc_params *p, uint32_t N, const float *vort_pos4,
             const double *ax, const double *ay, const double *az,
             uint32_t M, const float *eval_a4, const float *eval_b4,
             int is_segment, double *u, double *v, double *w, orc_dump *dump);

/* --- one vortex-segment time step (no boundary, heat or emitters) --------
 * HFS/VortexSimulationSystemImp.cpp:90-125 solveTimeStep: convertVortToSeg
 * (ComputePosb, HFS/GPU_kernel.cu:3184-3229, segment length cap h_seg),
 * computeURotation (velocity at both segment ends, other end = centre),
 * applyFlow (move_particle both ends, ComputePosa), convertSegToVort
 * (ComputeVortex), computeStretching (VectorAdd, hash of the new centres,
 * ParticleGaussianSmooth with width nu over the 5^3 hash cells,
 * HFS/GPU_kernel.cu:3327-3438).  cent4 and vort (x,y,z arrays) are updated
 * in place; enda4 / endb4 (optional, N float4) receive the moved ends.
 * P passive points (tracers, heat particles; may be 0) are evaluated with the
 * same far field (is_segment 0) and moved: pu/pv/pw receive their velocity. */
void orc_gaussian_smooth(const orc_params *p, uint32_t N, const float *cent4, const double *dx, const double *dy,
                         const double *dz, double nu, double *ox, double *oy, double *oz);
int orc_vortex_step(const orc_params *p, uint32_t N, float *cent4, double *vx, double *vy, double *vz,
                    double dt, double h_seg, double nu, float *enda4, float *endb4, uint32_t P,
                    float *passive4, double *pu, double *pv, double *pw);

/* --- buoyancy: heat particles -> density grid -> baroclinic vorticity ----
 * HFS/VortexSimulationSystemImp.cpp:336-465, HFS/GPU_kernel.cu:3655-3898.
 * Returns the density grid edge (0: nothing done). */
void orc_density_domain(const float *pos4, uint32_t N, double *origin3, double *length);
uint32_t orc_baroclinic(uint32_t H, const float *heat4, const float *life, uint32_t N,
                        const float *cent4, double *vx, double *vy, double *vz, double dt,
                        double *origin_out, double *h_out, float *rho_out, float *grad_out,
                        size_t cap);

/* --- FP64 O(N*M) smoothed Biot-Savart sum (accuracy ground truth) ------- */
void orc_direct_sum(uint32_t N, const float *vort_pos4, const double *ax,
                    const double *ay, const double *az, uint32_t M,
                    const float *eval_a4, const float *eval_b4, int is_segment,
                    double a, double *u, double *v, double *w);

/* --- scalar PPPM: PotentialFieldSolver (HFS/PotentialFieldSolver.cpp) --- */
void orc_potential_domain(const float *pos4, uint32_t N, double *origin3, double *length);
int orc_potential(uint32_t n, int K, int scalar, uint32_t N, const float *pos4, const double *mass, uint32_t M,
                  const float *eval4, double *out, double *dump_origin4, double *dump_density, double *dump_rhs,
                  double *dump_phi, double *dump_far, double *dump_monopole4);

int orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
