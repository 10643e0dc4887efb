/*
 * pppm.h — C ABI of the B200 (sm_100a) PPPM vortex-particle velocity
 * evaluation.
 *
 * It replaces the reference's hot path, BiotSavartSolver::computeFarFieldBuffer
 * followed by BiotSavartSolver::evaluateVelocity, together with the spatial
 * hash and the multigrid solver underneath it.  Reference files are cited by
 * their path inside the reference project (HFS = hybridFastSummation/
 * hybridFastSummation, MG = multigrid/multigrid, PH = particle_hash/
 * particle_hash).
 *
 * Conventions
 *   - Every function returns a pppm_status; pppm_last_error() describes the
 *     last failure on the calling thread.  (The reference returns bool true
 *     and exits the process on CUDA errors through helper_cuda.)
 *   - Pointers named *_dev are CUDA device pointers; *_host are host pointers.
 *     Positions are float4 records (x, y, z, w; w ignored), four floats each.
 *     Strengths and velocities are double arrays, one per component, as the
 *     reference's GpuArrayd buffers.
 *   - All work is enqueued on the scene's stream (cudaStream_t passed as
 *     void*; NULL = the legacy default stream).  Calls on different scenes are
 *     independent; one scene must not be used from two threads at once.
 *   - Grids are cubic, n^3 cells, x-fastest ((k*n + j)*n + i), as the
 *     reference's hash and multigrid assume.
 */
#ifndef PPPM_H
#define PPPM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pppm_status {
    PPPM_OK = 0,
    PPPM_ERR_INVALID = 1,   /* bad argument (NULL, size, capacity, mode)     */
    PPPM_ERR_CUDA = 2,      /* CUDA runtime error                            */
    PPPM_ERR_OOM = 3,       /* device allocation failed                      */
    PPPM_ERR_STATE = 4,     /* call out of order (e.g. eval before far field) */
    PPPM_ERR_DOMAIN = 5     /* degenerate domain (zero or non-finite extent) */
} pppm_status;

/* Domain selection.  BBOX3X is the reference's rule: edge L = 3 * largest
 * extent of the vortex bounding box, centred on the box
 * (HFS/BiotSavartSolverImp.cpp:379-409).  FIXED uses fixed_origin and
 * fixed_length. */
enum { PPPM_DOMAIN_BBOX3X = 0, PPPM_DOMAIN_FIXED = 1 };

/* Poisson solve.  REFERENCE runs the reference schedule — full multigrid then
 * one V(4,4) cycle, red-black SOR with omega = 1.43f, zero ghost values, 100
 * Jacobi sweeps on the coarsest level (MG/MultiGrid.cpp:128-250) — in FP32,
 * with the final V-cycle applied as an FP64 defect correction (FP64
 * residual, FP64 accumulation of psi).  CONVERGED repeats FP64
 * defect-correction V-cycles until ||b - A psi|| <= mg_tol * ||b||. */
enum { PPPM_MG_REFERENCE = 0, PPPM_MG_CONVERGED = 1 };

typedef struct pppm_params {
    uint32_t n;              /* grid edge (gdx == gdy == gdz), 4..512            */
    int32_t K;               /* near-field range in cells (m_K), -1..4; <0 = off */
    double a;                /* smoothing radius, absolute (0.08 in the reference,
                                HFS/GPU_kernel.cu:2306)                           */
    int32_t domain_mode;     /* PPPM_DOMAIN_*                                     */
    double fixed_origin[3];
    double fixed_length;
    int32_t mg_mode;         /* PPPM_MG_*                                         */
    double mg_tol;           /* relative residual target for CONVERGED            */
    int32_t mg_max_cycles;   /* cap on defect-correction cycles                   */
    double a_cells;          /* > 0: smoothing radius in cells, a = a_cells * h with
                                h the cell size of each build's domain (overrides a);
                                0: a is absolute, as in the reference              */
} pppm_params;

typedef struct pppm_scene pppm_scene;

/* Grids exposed for inspection (device pointers owned by the scene). */
enum {
    PPPM_GRID_VORT = 0,      /* float [3][n^3]: P2M result sum(alpha)/h^3        */
    PPPM_GRID_PSI = 1,       /* double [3][n^3]: vector potential                */
    PPPM_GRID_FAR = 2        /* float [3][n^3]: far-field velocity               */
};

const char *pppm_last_error(void);
const char *pppm_version(void);

/* Defaults = the reference's constants: K = 1, a = 0.08, BBOX3X,
 * PPPM_MG_REFERENCE, mg_tol 1e-10, 50 cycles, a_cells = 0; n must still be
 * set. */
pppm_status pppm_params_default(pppm_params *p);
/* The most accurate setting measured against the FP64 direct sum with the
 * same smoothing kernel (no reference counterpart: the reference hard-codes
 * a = 0.08, HFS/GPU_kernel.cu:2306): BBOX3X, smoothing radius one cell
 * (a_cells = 1), near field K = 3, multigrid converged to mg_tol = 1e-6 in
 * FP64 defect-correction cycles.  n must still be set. */
pppm_status pppm_params_accurate(pppm_params *p);

/* BiotSavartSolver::initializeSolver (HFS/BiotSavartSolverImp.cpp:44-229):
 * allocates every buffer for up to cap_vort vortices and cap_eval evaluation
 * points; later calls allocate only if a count exceeds its capacity. */
pppm_status pppm_scene_create(const pppm_params *p, uint32_t cap_vort, uint32_t cap_eval,
                              void *stream, pppm_scene **out);
/* BiotSavartSolver::shutdown (HFS/BiotSavartSolverImp.cpp:230-264). */
pppm_status pppm_scene_destroy(pppm_scene *s);
pppm_status pppm_scene_set_stream(pppm_scene *s, void *stream);
pppm_status pppm_scene_get_params(const pppm_scene *s, pppm_params *p);

/* BiotSavartSolver::setVortParameter (HFS/BiotSavartSolverImp.cpp:318-377):
 * copies N float4 positions and three double strength arrays (device). */
pppm_status pppm_set_vortices(pppm_scene *s, uint32_t N, const float *pos4_dev,
                              const double *ax_dev, const double *ay_dev, const double *az_dev);

/* BiotSavartSolver::computeFarFieldBuffer (HFS/BiotSavartSolverImp.cpp:756-816):
 * bounding box, hash + sort + cell tables + reorder, P2M, Poisson solve of the
 * three potential components, curl, far-field correction. */
pppm_status pppm_build_far_field(pppm_scene *s);

/* BiotSavartSolver::setEvalParameter + evaluateVelocity
 * (HFS/BiotSavartSolverImp.cpp:266-316, 410-516): far field interpolated at
 * eval_a plus the near-field smoothed Biot-Savart correction; with
 * is_segment = 1, vortices coinciding with eval_b (the segment's other end)
 * are excluded.  Writes velocities in the caller's order.  eval_b may be NULL
 * when is_segment = 0. */
pppm_status pppm_eval(pppm_scene *s, uint32_t M, const float *eval_a4_dev,
                      const float *eval_b4_dev, int is_segment,
                      double *u_dev, double *v_dev, double *w_dev);

/* Same evaluation with float output, interleaved (M x 3). */
pppm_status pppm_eval_f32(pppm_scene *s, uint32_t M, const float *eval_a4_dev,
                          const float *eval_b4_dev, int is_segment, float *uvw_dev);

/* End-to-end on host buffers: copies the inputs to the device, runs
 * set_vortices + build_far_field + eval, copies velocities back, and
 * synchronises the stream.  eval_a4_host = NULL evaluates at the vortex
 * positions with is_segment = 1 against themselves (each vortex excludes
 * itself), the way the reference drives a velocity evaluation of its own
 * particles. */
pppm_status pppm_solve_host(pppm_scene *s, uint32_t N, const float *pos4_host,
                            const double *ax_host, const double *ay_host, const double *az_host,
                            uint32_t M, const float *eval_a4_host, const float *eval_b4_host,
                            int is_segment, double *u_host, double *v_host, double *w_host);

/* One time step of the vortex positions (device, in place) by their own
 * velocity, strengths fixed.  Euler: the reference's particle move
 * (HFS/VortexSimulationSystemImp.cpp:277-314, move_particle at
 * HFS/GPU_kernel.cu:3118-3140): p <- float(double(p) + u dt), w = 0, with u the
 * full evaluation at the vortices.  RK2 (midpoint): u1 = U(x),
 * x_mid = x + dt/2 u1, u2 = U(x_mid), x <- x + dt u2 (two far-field builds and
 * two evaluations).  The scene's far field afterwards is the last one built. */
pppm_status pppm_advect_euler(pppm_scene *s, uint32_t N, float *pos4_dev, const double *ax_dev,
                              const double *ay_dev, const double *az_dev, double dt);
pppm_status pppm_advect_rk2(pppm_scene *s, uint32_t N, float *pos4_dev, const double *ax_dev,
                            const double *ay_dev, const double *az_dev, double dt);

/* One vortex-segment time step, VortexSimulationSystem::solveTimeStep
 * (HFS/VortexSimulationSystemImp.cpp:90-125) for a system without solid
 * boundary or shedding (call pppm_baroclinic first for the buoyancy source):
 *   convertVortToSeg  (:127-140, ComputePosb HFS/GPU_kernel.cu:3184-3229):
 *       s = alpha capped to length h_seg, endb = c + s/2, enda = c - s/2,
 *       kappa = max(|alpha| / h_seg, 1)
 *   computeURotation  (:142-228): far field of the blobs, velocity at endb and
 *       at enda, each a segment against the centre; with P > 0 also at the
 *       passive points passive4 (tracers, heat particles; evaluateBiotSavart
 *       :1195-1244), which receive their velocity in pu/pv/pw and move by it
 *       (p <- float(p + u dt), w = 0)
 *   applyFlow         (:277-314): both ends move (p <- float(p + u dt)), the
 *       centre becomes their midpoint
 *   convertSegToVort  (:315-331): dalpha = kappa (endb - enda) - alpha
 *   computeStretching (:466-525): alpha + dalpha is hashed at the new centres
 *       and smoothed with exp(-d^2 / (2 nu^2)) over the 5^3 hash cells around
 *       each centre (ParticleGaussianSmooth, HFS/GPU_kernel.cu:3327-3438).
 * cent4 (centres, w kept) and ax/ay/az (strengths) are updated in place on the
 * device.  enda4 / endb4 (N float4 each, may be NULL) receive the moved ends.
 * The reference passes h_seg = d_h (0.1 in its setups) and nu = 0.1.  Afterwards
 * the scene holds the hash of the new centres (cell tables, sorted index) but
 * no far field: call pppm_set_vortices before pppm_build_far_field. */
pppm_status pppm_vortex_step(pppm_scene *s, uint32_t N, float *cent4_dev, double *ax_dev, double *ay_dev,
                             double *az_dev, double dt, double h_seg, double nu, float *enda4_dev,
                             float *endb4_dev, uint32_t P, float *passive4_dev, double *pu_dev,
                             double *pv_dev, double *pw_dev);

/* Buoyancy source, VortexSimulationSystem::addBaroclinicForce
 * (HFS/VortexSimulationSystemImp.cpp:369-465): H heat particles (positions,
 * heat value per particle, cpu_heat_life in the reference) are deposited on a
 * density grid of edge min(floor(L / 0.2) + 1, 200) over 1.2 x their bounding
 * box (setDensityDomain :336-366; AssignDensity HFS/GPU_kernel.cu:3655-3740),
 * differentiated (GradDensity :3742-3797, periodic), and the gradient
 * interpolated at each of the N vortices adds 5 dt * 0.1 * (grad rho x (0,10,0))
 * to its strength (ParticleGetBaroclinic :3800-3898).  The reference applies
 * nothing for N > 262,144 (its launch has block and grid swapped); here every
 * vortex gets the force.  One stream synchronisation (the grid size depends on
 * the bounding box).  H == 0 or a zero-size box: no change. */
pppm_status pppm_baroclinic(pppm_scene *s, uint32_t H, const float *heat4_dev, const float *heat_dev,
                            uint32_t N, const float *cent4_dev, double *ax_dev, double *ay_dev,
                            double *az_dev, double dt);
/* The last density grid pppm_baroclinic built: edge, origin, cell size, and
 * device pointers to rho [dim^3] and grad rho [3][dim^3] (float, x-fastest). */
pppm_status pppm_get_density(pppm_scene *s, uint32_t *dim, double origin[3], double *h,
                             const float **rho_dev, const float **grad_dev);

/* Accessors matching BiotSavartSolver::getOrigin / getCellh
 * (HFS/BiotSavartSolver.h:34-35); synchronises the stream.  PPPM_ERR_DOMAIN
 * (origin and length still filled) when the last far field had a zero or
 * non-finite domain edge (one vortex, or all coincident); pppm_eval then
 * returned zero velocities. */
pppm_status pppm_get_domain(pppm_scene *s, double origin[3], double *length, double *cell_h);
/* Smoothing radius a of the last far field (a, or a_cells times its cell
 * size); synchronises the stream. */
pppm_status pppm_get_smoothing(pppm_scene *s, double *a);
/* getVortStartTable / getVortEndTable (HFS/BiotSavartSolver.h:28-29): device
 * pointers to n^3 uint32 tables (empty cells hold 0xFFFFFFFF in both). */
pppm_status pppm_get_cell_tables(pppm_scene *s, const uint32_t **start_dev,
                                 const uint32_t **end_dev);
/* Sorted order of the vortices (ParticleManager's gridParticleIndex and
 * gridParticleHash, PH/SpaceHashClass.h:87-89): device pointers, N entries. */
pppm_status pppm_get_sorted_index(pppm_scene *s, const uint32_t **key_dev,
                                  const uint32_t **idx_dev);
/* getSortPos / getSortVort (HFS/BiotSavartSolver.h:25,27): gathers the
 * vortex positions and double strengths into sorted order. */
pppm_status pppm_get_sorted_vortices(pppm_scene *s, float *pos4_dev, double *ax_dev,
                                     double *ay_dev, double *az_dev);
pppm_status pppm_get_grid(pppm_scene *s, int which, const void **ptr_dev);
/* Near-field pairs inside the axis box at the last eval with pair counting
 * on, multigrid cycles and final relative residual of the last solve. */
pppm_status pppm_get_stats(pppm_scene *s, uint64_t *pairs, int32_t *mg_cycles,
                           double *mg_relres);
/* Re-runs the last eval with pair counting on (diagnostics; not timed). */
pppm_status pppm_count_pairs(pppm_scene *s, uint32_t M, const float *eval_a4_dev,
                             uint64_t *pairs);

/* Per-stage timing with CUDA events on the scene stream (off by default, on
 * from creation when the environment variable PPPM_PROFILE is set to anything
 * but "" or "0"; no reference counterpart — the reference prints no timings).
 * Stages: 0 domain, 1 vort_sort, 2 cells_reorder, 3 p2m, 4 multigrid,
 * 5 farfield, 6 eval_sort, 7 eval, 8 segments, 9 seg_to_blob, 10 rehash,
 * 11 gaussian_smooth.  pppm_get_stage_times synchronises the stream and
 * writes the last recorded duration of each stage in ms (-1 = not run). */
pppm_status pppm_scene_set_profiling(pppm_scene *s, int on);
const char *pppm_stage_name(int stage);
pppm_status pppm_get_stage_times(pppm_scene *s, double *ms, int cap, int *count);
/* Number of kernels this library has launched in the process so far. */
uint64_t pppm_kernel_launches(void);
/* The multigrid smoother's autotuner (no reference counterpart).  By default
 * every level runs the plain red-black half sweeps.  With PPPM_MG_TB=auto in
 * the environment when a scene or multigrid object is created, each level of
 * edge >= 256 runs either the plain half sweeps or one of the temporally
 * blocked variants (T half sweeps per pass, TX x TY tiles, TMA plane
 * staging), whichever measured fastest for that edge and component count on
 * this device; PPPM_MG_TB=<index> forces one variant.  Every choice gives the
 * same values bit for bit.  Writes a text table of the autotuner's
 * measurements, one line per edge, into buf (NUL-terminated, truncated to
 * cap; empty when it has not run); *written receives its length. */
pppm_status pppm_tuning_report(char *buf, size_t cap, size_t *written);

/* ---- several independent scenes in one call -----------------------------
 * No reference counterpart (the reference drives one solver from one host
 * thread).  Each item is one scene's set_vortices + build_far_field + eval
 * (M = 0 skips the eval).  The builds and the evaluation points' sorts run on
 * a set of streams the call borrows (longest predicted build first, each onto
 * the least loaded stream), ordered after the caller's earlier work on
 * `stream`; then all items' evaluations run as one launch on `stream` over a
 * work list of (scene, block of 128 points), the scenes with the most
 * particles per cell first (one launch per group of items that differ in
 * smoothing series or segment mode).  `stream` has all the batch's work when
 * the call returns.  A scene may appear once per batch.  Each scene's result
 * is bit for bit the one it gets alone.  Concurrent calls from several
 * threads borrow different stream sets and overlap on the device. */
typedef struct pppm_batch_item {
    pppm_scene *scene;
    uint32_t N;
    const float *pos4_dev;
    const double *ax_dev, *ay_dev, *az_dev;
    uint32_t M;
    const float *eval_a4_dev;
    const float *eval_b4_dev;
    int is_segment;
    double *u_dev, *v_dev, *w_dev;
} pppm_batch_item;
pppm_status pppm_batch_run(pppm_batch_item *items, uint32_t count, void *stream);

/* ---- request loop over resident scenes ----------------------------------
 * No reference counterpart.  Scenes are registered with host particles; a
 * request asks for the velocity at a scene's particles (EVAL) or for `steps`
 * RK2 steps of them (ADVANCE, dt).  `slots` worker threads, one CUDA stream
 * each, serve requests as they arrive (continuous batching: new requests
 * start as soon as a slot frees and overlap on the GPU).  A scene's device
 * footprint is admitted against hbm_budget_bytes; idle resident scenes are
 * evicted least recently used first, their positions saved to the host.
 * Requests of one scene run in submission order.  Times are seconds on a
 * monotonic host clock. */
typedef struct pppm_server pppm_server;
typedef struct pppm_server_config {
    uint64_t hbm_budget_bytes;
    uint32_t slots;
} pppm_server_config;
enum { PPPM_REQ_EVAL = 0, PPPM_REQ_ADVANCE = 1 };
typedef struct pppm_request_info {
    int32_t status;      /* pppm_status of the request */
    double submit_s;
    double start_s;
    double end_s;
} pppm_request_info;
pppm_status pppm_server_create(const pppm_server_config *cfg, pppm_server **out);
pppm_status pppm_server_destroy(pppm_server *srv);
pppm_status pppm_server_add_scene(pppm_server *srv, const pppm_params *p, uint32_t N, const float *pos4_host,
                                  const double *ax_host, const double *ay_host, const double *az_host,
                                  uint64_t *scene_id);
pppm_status pppm_server_submit(pppm_server *srv, uint64_t scene_id, int kind, uint32_t steps, double dt,
                               uint64_t *ticket);
/* Waits for a request; vel_host (3*N doubles, may be NULL) receives an EVAL
 * result as [3][N].  Each ticket can be waited for once. */
pppm_status pppm_server_wait(pppm_server *srv, uint64_t ticket, double timeout_s, pppm_request_info *info,
                             double *vel_host);
/* Current positions of a scene (after its queued requests have finished). */
pppm_status pppm_server_read_positions(pppm_server *srv, uint64_t scene_id, float *pos4_host);
pppm_status pppm_server_stats(pppm_server *srv, uint64_t *resident_bytes, uint64_t *completed);

/* ---- frame files ----------------------------------------------------------
 * The demo driver's output (HFS/newTest.cpp:23-36): <dir>/Particle_data%04d.bin,
 * N raw float4 records (x, y, z, 1.0f).  pos4 may be a host or device array
 * (on_device).  pppm_read_frame with pos4_host = NULL returns the record count. */
pppm_status pppm_frame_path(const char *dir, int frame, char *out, size_t cap);
pppm_status pppm_write_frame(const char *dir, int frame, uint32_t N, const float *pos4, int on_device);
pppm_status pppm_read_frame(const char *path, float *pos4_host, uint32_t cap, uint32_t *N);

/* SGI image file as Particle_renderer/.../write_sgi.cpp:6-67 writes it
 * (host pixels, i-fastest, `channels` 1 or 3 interleaved per pixel; 8-bit, or
 * 16-bit with high_precision). */
pppm_status pppm_write_sgi(const char *path, uint32_t ni, uint32_t nj, int channels, const float *pix_host,
                           int high_precision);

/* --- headless splatting renderer (Particle_renderer/particle_renderer/
 * particle_renderer/shadow.cpp, render.cpp) ------------------------------
 * Positions are float4 records (w ignored); per-particle density / opacity
 * factors and colours are float arrays on the device.  Work runs on the
 * renderer's stream; each call reads sizes back to the host once or twice. */
typedef struct pppm_renderer pppm_renderer;
pppm_status pppm_renderer_create(void *stream, pppm_renderer **out);
pppm_status pppm_renderer_destroy(pppm_renderer *r);
/* compute_shadows (shadow.cpp:56-145): the particles, nearest to the light
 * first, darken a perspective shadow map seen from the light by
 * exp(-opacity * dens * (1 - d^2/r^2)^2) per pixel; illum_dev[i] receives the map
 * at particle i's pixel before its own disc.  Map edge = int(quality * R /
 * radius) for the bounding-sphere radius R.  PPPM_ERR_DOMAIN when the light is
 * inside 1.25 R (the reference returns false there). */
pppm_status pppm_render_shadows(pppm_renderer *r, uint32_t n, const float *pos4_dev, const float *dens_dev,
                                float radius, float opacity, const float light[3], float quality,
                                float *illum_dev, uint32_t *npix);
/* The last shadow map (npix x npix floats, i-fastest, device). */
pppm_status pppm_render_shadow_map(pppm_renderer *r, const float **map_dev, uint32_t *npix);
/* render_smoke (render.cpp:61-125): back-to-front over-compositing of
 * (1 - illum) base_rgb + illum lit_rgb discs into a width x height RGB image
 * (image_dev[3 * (i + width * j) + c]) that starts as the background; camera
 * at `camera` looking at `target`, perspective factor `perspective`. */
pppm_status pppm_render_smoke(pppm_renderer *r, uint32_t n, const float *pos4_dev, const float *illum_dev,
                              const float *base_rgb_dev, const float *lit_rgb_dev, float radius, float opacity,
                              const float *den_dev, const float background[3], const float camera[3],
                              const float target[3], float perspective, uint32_t width, uint32_t height,
                              float *image_dev);

/* ---- multigrid surface: gf::MultiGridSolver3DPeriod_double
 * (MG/MultiGrid.h:188-209, MG/MultiGrid.cpp:128-250) ---------------------- */
typedef struct pppm_mg pppm_mg;
/* m_InitialSystem(n, n, n). */
pppm_status pppm_mg_create(uint32_t n, void *stream, pppm_mg **out);
pppm_status pppm_mg_destroy(pppm_mg *mg);
/* m_FullMultiGrid(x, b, tol, residual) on FP64 device arrays of n^3: solves
 * sum_nbr(x) - 6x = b with zero ghost values, starting from the x given (the
 * reference's first residual is b - A x): x <- x + FMG(0, b - A x).
 * mode = PPPM_MG_REFERENCE runs the reference schedule (tol ignored, as in the
 * reference); CONVERGED adds defect-correction cycles until the residual is
 * below tol relative to ||b - A x_initial||, which *relres (may be NULL)
 * receives. */
pppm_status pppm_mg_full_multigrid(pppm_mg *mg, double *x_dev, const double *b_dev,
                                   int mode, double tol, int max_cycles, double *relres);
/* m_Vcycle(x, b, tol, residual, level) (MG/MultiGrid.cpp:128-201): one V(4,4)
 * cycle from `level` down to the coarsest level and back, on that level's FP64
 * arrays x and b of d_level^3 entries (level 0 = the n^3 grid).  Applied as a
 * defect correction: r = b - A x in FP64, an FP32 cycle on A e = r from
 * e = 0, x += e in FP64 — the reference's cycle in exact arithmetic.  The
 * reference ignores tol and leaves residual unset; so does the C++ mirror. */
pppm_status pppm_mg_vcycle(pppm_mg *mg, double *x_dev, const double *b_dev, int level);
/* Level count of the hierarchy (halve while a level has more than 512 cells,
 * MG/MultiGrid.h:114-127) and the edge of each level (up to cap entries). */
pppm_status pppm_mg_levels(const pppm_mg *mg, int *levels, uint32_t *edges, int cap);

/* ---- scalar PPPM: PotentialFieldSolver (HFS/PotentialFieldSolver.h:10-91,
 * HFS/PotentialFieldSolver.cpp:45-739) ------------------------------------
 * Masses on a 2 x bounding-box grid of edge n, the monopole as Dirichlet
 * data, three full-multigrid calls, and evaluation of the single-layer
 * potential or its gradient with a near-field particle correction over K
 * cells.  Grids and sums are FP64 as in the reference. */
typedef struct pppm_potential pppm_potential;
/* initializeSolver(n, n, n, K, M, N). */
pppm_status pppm_potential_create(uint32_t n, int K, uint32_t cap_mass, uint32_t cap_eval, void *stream,
                                  pppm_potential **out);
pppm_status pppm_potential_destroy(pppm_potential *p);
/* setMassParameter (:344-392): N float4 positions and N double masses (device). */
pppm_status pppm_potential_set_masses(pppm_potential *p, uint32_t N, const float *pos4_dev,
                                      const double *mass_dev);
/* computeFarFieldBuffer (scalar = 0, :695-707) or
 * computeFarFieldPotentialBuffer (scalar = 1, :726-737).  One stream
 * synchronisation (the grid spacing comes from the bounding box). */
pppm_status pppm_potential_build(pppm_potential *p, int scalar);
/* evaluateGradient (:441-526): gradient at M points (device), caller order;
 * zero at points outside the grid box.  Needs the gradient buffer. */
pppm_status pppm_potential_eval_gradient(pppm_potential *p, uint32_t M, const float *eval4_dev,
                                         double *gx_dev, double *gy_dev, double *gz_dev);
/* The same with the gradient interleaved per point (x, y, z), the layout of
 * the reference's GpuArrayd3 m_particle_gradPhi. */
pppm_status pppm_potential_eval_gradient3(pppm_potential *p, uint32_t M, const float *eval4_dev,
                                          double *grad3_dev);
/* evaluateScalarPotential (:708-739): potential at M points.  Needs the
 * scalar buffer. */
pppm_status pppm_potential_eval_scalar(pppm_potential *p, uint32_t M, const float *eval4_dev, double *phi_dev);
/* computeDphiDn (:621-626, HFS/GPU_kernel.cu:1719-1740):
 * out = -0.5 mass / area + n . grad per panel. */
pppm_status pppm_potential_dphidn(pppm_potential *p, uint32_t M, const double *nx_dev, const double *ny_dev,
                                  const double *nz_dev, const double *gx_dev, const double *gy_dev,
                                  const double *gz_dev, const double *mass_dev, const double *area_dev,
                                  double *out_dev);
/* Inspection: origin and edge L of the last build, device pointers to the
 * density, right-hand side (with the Dirichlet data), potential and
 * far-field buffer ([3][n^3] gradient or [n^3] scalar), and the monopole
 * (centre x, y, z, total mass) copied to the host. */
pppm_status pppm_potential_grids(pppm_potential *p, double origin_length[4], const double **density_dev,
                                 const double **rhs_dev, const double **phi_dev, const double **far_dev,
                                 double monopole_host[4]);

/* ---- spatial hash surface: ParticleManager (PH/SpaceHashClass.h:10-84) and
 * the extern "C" calcHash / sortParticles / FindCellStart / reorder / deorder
 * of PH/SpaceHashHeader.cuh:12-47 ------------------------------------------ */
typedef struct pppm_hasher pppm_hasher;
/* initSpatialHash(numParticles, n, n, n). */
pppm_status pppm_hasher_create(uint32_t cap_particles, uint32_t n, void *stream,
                               pppm_hasher **out);
pppm_status pppm_hasher_destroy(pppm_hasher *h);
/* setSpatialHashGrid(n, h, origin) + doSpatialHash(pos, N): cell key
 * floor((p - origin)/h) in FP32 per axis, wrapped mod n, stable sort of
 * (key, index), cell start/end tables. */
pppm_status pppm_hasher_run(pppm_hasher *h, uint32_t N, const float *pos4_dev, float cell_h,
                            const float origin[3]);
pppm_status pppm_hasher_tables(pppm_hasher *h, const uint32_t **key_dev, const uint32_t **idx_dev,
                               const uint32_t **start_dev, const uint32_t **end_dev);
/* reorderData / deorderData (PH/SpaceHashClassImp.cpp:24-34): gather
 * out[i] = in[idx[i]] or scatter out[idx[i]] = in[i] of `stride` elements of
 * 4 bytes (precision 1) or 8 bytes (precision 2) each. */
pppm_status pppm_hasher_reorder(pppm_hasher *h, uint32_t N, const void *in_dev, void *out_dev,
                                uint32_t stride, uint32_t precision);
pppm_status pppm_hasher_deorder(pppm_hasher *h, uint32_t N, const void *in_dev, void *out_dev,
                                uint32_t stride, uint32_t precision);

/* ---- spatial hash that allocates nothing ---------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory on this path: a simulation loop with a fixed per-frame budget, where
 * cudaMalloc / cudaFree would synchronise the device and stall the frame; a
 * host whose device allocator has a fixed size and must not grow; or a
 * process in which another framework's pool already owns the device heap.
 * It gives the same result as pppm_hasher_run into caller-provided device
 * arrays, with the sort's scratch in a fixed device array of
 * PPPM_NOALLOC_SCRATCH_BYTES that every GPU loading the library keeps until
 * the process exits.
 *   - pos4_dev: N float4 records (x, y, z, w; 16-byte stride, w ignored).
 *   - sorted_key_dev, sorted_idx_dev: N entries each (cell keys in sorted
 *     order, original indices in the same order).
 *   - cell_start_dev, cell_end_dev: n^3 entries each; every entry is written
 *     (0xFFFFFFFF for empty cells, filled first, then the occupied cells, in
 *     stream order), so they need no initialisation.
 *   - N must not exceed PPPM_NOALLOC_MAX_PARTICLES (else PPPM_ERR_INVALID,
 *     before any device work).
 *   - The first call on a device looks up the array's device address and
 *     keeps it for the process; make that first call before any stream
 *     capture on that device.  After cudaDeviceReset on that device the kept
 *     address is stale: do not call this entry point again in that process.
 *   - All calls share the array: calls whose work overlaps on the GPU (other
 *     streams, other threads) race and corrupt each other's results.
 *   - No cudaMalloc, cudaFree or allocating library routine is called. */
#define PPPM_NOALLOC_MAX_PARTICLES 1048576u
#define PPPM_NOALLOC_SCRATCH_BYTES 8651776u
pppm_status pppm_spatial_hash_noalloc(uint32_t N, const float *pos4_dev, uint32_t n, float cell_h,
                                      const float origin[3], uint32_t *sorted_key_dev,
                                      uint32_t *sorted_idx_dev, uint32_t *cell_start_dev,
                                      uint32_t *cell_end_dev, void *stream);

/* ---- FP64 O(N*M) direct sum with the near field's smoothing kernel ------
 * (accuracy ground truth; no reference counterpart) */
pppm_status pppm_direct_sum_fp64(uint32_t N, const float *vort_pos4_dev, const double *ax_dev,
                                 const double *ay_dev, const double *az_dev, uint32_t M,
                                 const float *eval_a4_dev, const float *eval_b4_dev, int is_segment,
                                 double a, double *u_dev, double *v_dev, double *w_dev,
                                 void *stream);

/* Test hook, no counterpart in the reference: after `after` more device or
 * pinned-host allocations by the library succeed, the next one fails as if
 * the device were out of memory (the call that made it returns PPPM_ERR_OOM);
 * later allocations succeed again.  after < 0 disarms it.  Lets a test walk
 * every allocation of a call sequence and check that each failure is reported
 * and leaves nothing allocated, with no real memory pressure. */
pppm_status pppm_debug_fail_allocation(int64_t after);

#ifdef __cplusplus
}
#endif
#endif
