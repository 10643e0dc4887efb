// Internal declarations shared by the sm_100a kernels and the C ABI.
//
// Data layout in HBM (one scene, grid edge n, C = n^3 cells, N vortices,
// M evaluation points):
//   * grids are x-fastest, index (k*n + j)*n + i, components stored as three
//     consecutive planes [3][C] (structure of arrays);
//   * sorted vortex records are two float4 streams: {rel.x, rel.y, rel.z,
//     ngp cell id as bits} and {alpha.x, alpha.y, alpha.z, 0}, where rel is the
//     position relative to the domain origin rounded to float exactly as the
//     reference rounds it, and the ngp cell is floor(rel * (1/h)) in FP64;
//   * multigrid levels are FP32 [3][C_l] planes; the corrected potential psi is
//     FP64 [3][C].
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "../../include/pppm.h"

namespace pppm {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr int kMaxLevels = 12;
constexpr int kMaxK = 4;  // near-field range limit (table (2K+1)^3 in shared memory)
constexpr uint32_t kRsTileHost = 4096;  // radix-sort keys per block (kRsThreads * kRsItems)

// Literal constants of the reference kernels.
constexpr double kFourPi = 12.5663706144;          // HFS/GPU_kernel.cu:12,2397,2403
constexpr double kDiagPsi = 0.250580605913965;     // HFS/GPU_kernel.cu:1990-1992

// Per-scene parameters derived on the device from the vortex bounding box
// (HFS/BiotSavartSolverImp.cpp:379-409, PH/SpaceHashClass.h:46-54), so that no
// host round trip is needed between the bounding box and the hash.
struct DevParams {
    double origin[3];   // domain origin (double, as the solver keeps it)
    double length;      // domain edge L
    double cell_h;      // (double)h_f: the solver reads the float cell size back
    double invh;        // 1.0 / cell_h
    float origin_f[3];  // float origin the hash uses
    float h_f;          // float cell size the hash uses
    float h2f;          // h_f*h_f rounded to float (ComputeRHS argument, :557)
    float invh3_f;      // (float)(invh^3)
    float cr_f;         // largest float strictly below (K+0.5)/invh
    float vh3_f;        // (float)(h^3) for the mesh correction
    float kdiag_f;      // (float)(0.5 * invh * 0.250580605913965 * h^2)
    double a;           // smoothing radius of this build (prm.a, or prm.a_cells * cell_h)
    float inv_a3_f;     // 1/a^3
    float inv4pia3_f;   // 1/(4 pi a^3)
    int32_t need_exp;   // some pair inside the box can reach (r/a)^3 >= 0.25
    int32_t need_exp2;  // ... and (r/a)^3 >= 2
    double prune_cells; // bound, in cells, on |hash cell coordinate - FP64 NGP coordinate|
                        // plus the float rounding of the box test (near-field cell pruning)
    uint32_t n;
    int32_t K;
    int32_t status;     // 0 ok, else PPPM_ERR_* raised on the device
};

struct Level {
    uint32_t d;       // edge
    uint32_t cells;   // d^3
    float *x;         // [comps][cells]
    float *b;         // [comps][cells]
    float *x2 = nullptr;  // [comps][cells] second copy of x for the blocked smoother (its levels only)
};

// Temporally blocked smoother (mg_tb.cu): T half sweeps per pass over a level.
constexpr uint32_t kTbErrTimeout = 0x7B000001u;  // an mbarrier wait ran out
int tb_variant_count();
void tb_variant_shape(int variant, int *T, int *TX, int *TY, int *G4 = nullptr);  // G4: groups of 4 cells
cudaError_t tb_make_map(CUtensorMap *map, float *base, int d, int comps, int variant);
cudaError_t tb_prepare(int variant, int *blocks_per_sm);
cudaError_t tb_smooth(int variant, const CUtensorMap &map_x, const CUtensorMap &map_b, const float *b_dev, int load_x,
                      const float *xc, float *x_out, int d, int comps, int zchunk, uint32_t *err, cudaStream_t st);

// Tensor maps of one level for the blocked smoother.
struct TbMaps {
    CUtensorMap x, x2, b;
};

// Everything one multigrid solve touches; comps independent right-hand sides.
struct MGPlan {
    int levels = 0;
    Level lv[kMaxLevels];
    // blocked smoother per level: its variant (-1 = plain half sweeps), tensor
    // maps and z-chunk length (levels with edge >= tb_min_edge, x2 allocated),
    // and the device error flag
    int tb_var[kMaxLevels] = {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1};
    uint32_t tb_min_edge = 256;  // smaller levels measured faster with the plain half sweeps
    bool tb_fuse_prolong = false;  // prolongation inside the first post-smoothing pass
    TbMaps tb_maps[kMaxLevels];
    int tb_zchunk[kMaxLevels] = {};
    uint32_t *err = nullptr;
    int comps = 3;
    cudaStream_t st = nullptr;
    double *psi = nullptr;          // [comps][C0] FP64 solution
    const double *b64 = nullptr;    // FP64 right-hand side, or
    const float *vort = nullptr;    // b = -(vort * h2f) from the P2M grid
    const DevParams *P = nullptr;
    double *norms = nullptr;        // [2] device scratch
    const double *coarse_op = nullptr;  // [cells][cells] FP64 map b -> x of the coarsest solve, or null
};

// Every device and pinned-host allocation of the library goes through these
// two, so that a test can make one of them fail on purpose
// (pppm_debug_fail_allocation) without a real out-of-memory condition.
cudaError_t device_malloc(void **p, size_t bytes);
cudaError_t host_malloc(void **p, size_t bytes);

cudaError_t build_coarse_operator(int d, double *op, cudaStream_t st);
cudaError_t mg_capture_graph(const MGPlan &m, cudaGraphExec_t *exec, unsigned *kernel_nodes);

// Density grid and heat-particle hash of the buoyancy source (buoyancy.cu),
// allocated on first use.
struct Buoyancy;
void free_buoyancy(Buoyancy *b);

}  // namespace pppm

// Scene: every buffer is sized at creation (or on growth in
// pppm_set_vortices / pppm_eval), so the per-call path allocates nothing.
struct pppm_scene {
    pppm_params prm;
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t n = 0, C = 0;
    int levels = 0;
    pppm::Level lv[pppm::kMaxLevels];

    uint32_t capN = 0, capM = 0;
    uint32_t N = 0, M = 0;
    bool vort_set = false, far_ready = false;

    pppm::DevParams *dparams = nullptr;   // device
    float *bbox_partial = nullptr;        // [6][bbox_blocks]
    int bbox_blocks = 0;

    // vortex side
    float4 *vpos = nullptr;               // caller order copy [capN]
    double *valpha = nullptr;             // caller order copy [3][capN]
    uint32_t *vkey[2] = {nullptr, nullptr};
    uint32_t *vidx[2] = {nullptr, nullptr};
    uint32_t *vsorted_key = nullptr, *vsorted_idx = nullptr;  // near-field order, point into vkey/vidx
    uint32_t *rkey[2] = {nullptr, nullptr};                   // reference order, built on request
    uint32_t *ridx[2] = {nullptr, nullptr};
    uint32_t *ref_sorted_key = nullptr, *ref_sorted_idx = nullptr;
    bool ref_valid = false;
    float4 *vrec = nullptr;               // sorted {rel, ngp}
    float4 *valf = nullptr;               // sorted {alpha, 0}
    uint32_t *cell_start = nullptr, *cell_end = nullptr, *mflag = nullptr;
    uint32_t *sub_start = nullptr, *sub_end = nullptr;   // [8 n^3] runs of (cell, octant)
    uint32_t epoch = 0;

    // radix-sort histogram scratch
    uint32_t *hist = nullptr;
    size_t hist_cap = 0;

    // grid side
    float *vort = nullptr;                // [3][C]
    float *mg_pool = nullptr;             // all levels' x and b
    double *psi = nullptr;                // [3][C]
    float *far = nullptr;                 // [3][C]
    double *norms = nullptr;              // [2] residual / rhs squared norms
    double *coarse_op = nullptr;          // coarsest-level operator (levels >= 2)
    cudaGraphExec_t mg_graph = nullptr;   // reference-schedule solve, captured once
    unsigned mg_graph_kernels = 0;
    float *mg_x2_pool = nullptr;          // second x copies of the blocked-smoother levels
    uint32_t *mg_err = nullptr;           // device error flag of the blocked smoother
    pppm::MGPlan mg_tb;                   // its variant, tensor maps and z-chunks (lv[].x2 in lv)

    // evaluation side
    uint32_t *ekey[2] = {nullptr, nullptr};
    uint32_t *eidx[2] = {nullptr, nullptr};
    uint32_t *esorted_idx = nullptr;
    float4 *stage_ea = nullptr, *stage_eb = nullptr;  // pppm_solve_host staging [capM]
    double *stage_out = nullptr;                       // [3][capM]
    float4 *adv_mid = nullptr;                         // RK2 midpoint positions [capN]
    double *ts_kappa = nullptr;                        // segment stretch factor [capN]
    pppm::Buoyancy *buoy = nullptr;                    // heat -> density grid, on first use

    // per-stage CUDA-event timing (pppm_scene_set_profiling)
    bool profiling = false;
    cudaEvent_t ev_begin[16] = {}, ev_end[16] = {};
    bool ev_used[16] = {};

    // statistics
    unsigned long long *pair_count = nullptr;
    int mg_cycles_last = 0;
    double mg_relres_last = 0.0;
};

namespace pppm {

// Stages timed by the profiling events, in pipeline order.
enum Stage {
    kStageDomain = 0,      // bounding box + device parameters
    kStageVortSort = 1,    // vortex keys + radix sort
    kStageCells = 2,       // cell tables + reorder
    kStageP2M = 3,
    kStageMG = 4,
    kStageFar = 5,         // curl + far-field correction
    kStageEvalSort = 6,    // evaluation-point keys + radix sort
    kStageEval = 7,        // interpolation + near field + deorder
    kStageSegments = 8,    // vortex step: blobs -> segments
    kStageSegToBlob = 9,   // vortex step: move ends, midpoint, strength update
    kStageRehash = 10,     // vortex step: domain + hash of the moved centres
    kStageSmooth = 11,     // vortex step: Gaussian smoothing of the strengths
    kNumStages = 12
};
const char *stage_name(int i);

// Library-wide lock held around CUDA graph capture and around every call that
// can synchronise the whole device (cudaMalloc, cudaFree, scene creation and
// destruction), so that no capture in one thread is ever invalidated by an
// implicit device synchronisation in another thread.
std::recursive_mutex &device_lock();
cudaError_t prepare_multigrid_graph(pppm_scene *s);

// Process-wide count of kernel launches issued by this library.
void note_launch();
unsigned long long launch_count();
void prof_begin(pppm_scene *s, int stage);
void prof_end(pppm_scene *s, int stage);

// Kernel launchers (each enqueues on s->stream and returns the launch status).
cudaError_t launch_bbox_and_params(pppm_scene *s);
cudaError_t launch_hash_sort(pppm_scene *s, const float4 *pos, uint32_t N, uint32_t *key[2],
                             uint32_t *idx[2], uint32_t **sorted_key, uint32_t **sorted_idx);
cudaError_t launch_cells_reorder(pppm_scene *s);
cudaError_t launch_reference_order(pppm_scene *s);
cudaError_t launch_p2m(pppm_scene *s);
cudaError_t run_multigrid(pppm_scene *s);
cudaError_t launch_farfield(pppm_scene *s);
cudaError_t launch_eval(pppm_scene *s, const float4 *eval_a, const float4 *eval_b, int is_segment,
                        uint32_t M, double *u, double *v, double *w, float *uf, int count_pairs);

// Everything the evaluation of one scene's points reads and writes.
struct EvalArgs {
    const uint32_t *eidx;          // sorted original indices of the points
    uint32_t M;
    const float4 *eval_a, *eval_b;
    const float *far;
    const uint32_t *start, *end, *sub_start, *sub_end;
    const float4 *vrec, *valf;
    const DevParams *P;
    int n, K;
    double *u, *v, *w;
    float *uf;
    unsigned long long *pair_count;
};
// What items of one batched evaluation launch must share: the smoothing
// series (bytes), its folding and the segment mode.
struct EvalMode {
    bool fold = false, seg = false;
    unsigned char series[192] = {};
    bool same(const EvalMode &o) const {
        if (fold != o.fold || seg != o.seg) return false;
        for (int i = 0; i < 192; i++)
            if (series[i] != o.series[i]) return false;
        return true;
    }
};
cudaError_t eval_batch_prepare(pppm_scene *s, const float4 *eval_a, const float4 *eval_b, int is_segment, uint32_t M,
                               double *u, double *v, double *w, EvalArgs *args, EvalMode *mode);
cudaError_t launch_eval_batch(const EvalMode &mode, const EvalArgs *args_dev, const uint2 *work_dev, uint32_t blocks,
                              cudaStream_t st);
cudaError_t launch_gather_sorted(pppm_scene *s, float4 *pos_out, double *alpha_out);
cudaError_t launch_move(pppm_scene *s, const float4 *base, const double *u, size_t stride, double dt, uint32_t N,
                        float4 *out);

// Reference hash (keys, stable sort, start/end tables) on an explicit grid.
cudaError_t launch_explicit_hash(cudaStream_t st, const float4 *pos, uint32_t N, float h, const float of[3],
                                 uint32_t n, uint32_t *key[2], uint32_t *idx[2], uint32_t *hist,
                                 uint32_t **skey, uint32_t **sidx, uint32_t *start, uint32_t *end);
cudaError_t launch_segments(pppm_scene *s, double h_seg, uint32_t N, float4 *ends, float4 *other, double *kappa);
cudaError_t launch_segment_to_blob(pppm_scene *s, const float4 *ends, const double *u, size_t ustride,
                                   const double *kappa, double dt, uint32_t N, float4 *cent, float4 *enda_out,
                                   float4 *endb_out);
cudaError_t launch_gaussian_smooth(pppm_scene *s, double nu, uint32_t N, double *ox, double *oy, double *oz);
cudaError_t launch_move3(pppm_scene *s, float4 *pos, const double *u, const double *v, const double *w, double dt,
                         uint32_t N);

cudaError_t mg_solve(const MGPlan &m, int mode, double tol, int max_cycles, int *cycles_out,
                     double *relres_out);
cudaError_t mg_vcycle_update(const MGPlan &m, double *x64);
// Second x copy per level for the blocked smoother: bytes to allocate (all of
// a plan's levels that qualify), then tensor maps and z-chunks over them.
size_t mg_tb_extra_floats(const MGPlan &m);
cudaError_t mg_tb_setup(MGPlan &m, float *pool, int forced);
size_t mg_tune_report(char *buf, size_t cap);

cudaError_t radix_sort_pairs(cudaStream_t st, uint32_t N, uint32_t bits, uint32_t *key[2], uint32_t *idx[2],
                             uint32_t *hist, uint32_t **sorted_key, uint32_t **sorted_idx);

int mg_level_count(uint32_t n);
// Blocked-smoother choice for new multigrid objects: -1 (the plain half
// sweeps) unless PPPM_MG_TB in the environment names a variant index, or
// "auto" (-2: the autotuner picks per level).
int mg_tb_default_variant();
bool mg_shape_ok(uint32_t n);
uint32_t key_bits(uint32_t n);
size_t radix_hist_entries(uint32_t N);

}  // namespace pppm

#define PPPM_CUDA_TRY(expr)                            \
    do {                                               \
        cudaError_t _e = (expr);                       \
        if (_e != cudaSuccess) return _e;              \
    } while (0)
