// C ABI of the PPPM path: scene lifecycle, the BiotSavartSolver entry points,
// the standalone multigrid object, and the FP64 direct sum.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "pppm_internal.cuh"

namespace pppm {

namespace {
// Allocations still to succeed before one is made to fail (-1: none armed).
std::atomic<long long> g_alloc_fail_after{-1};

bool fail_this_allocation() {
    long long c = g_alloc_fail_after.load();
    while (c >= 0) {
        if (g_alloc_fail_after.compare_exchange_weak(c, c - 1)) return c == 0;
    }
    return false;
}
}  // namespace

cudaError_t device_malloc(void **p, size_t bytes) {
    if (fail_this_allocation()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMalloc(p, bytes);
}

cudaError_t host_malloc(void **p, size_t bytes) {
    if (fail_this_allocation()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMallocHost(p, bytes);
}

}  // namespace pppm

extern "C" pppm_status pppm_debug_fail_allocation(int64_t after) {
    pppm::g_alloc_fail_after.store(after < 0 ? -1 : (long long)after);
    return PPPM_OK;
}

namespace {

thread_local char g_err[512] = "";

bool valid_params(const pppm_params *p, char *why, size_t cap) {
    if (!p) { snprintf(why, cap, "params is NULL"); return false; }
    if (p->n < 4 || p->n > 512) { snprintf(why, cap, "grid edge n=%u outside [4, 512]", p->n); return false; }
    if (!pppm::mg_shape_ok(p->n)) {
        snprintf(why, cap, "grid edge n=%u: a multigrid level above the coarsest has an odd edge", p->n);
        return false;
    }
    if (p->K < -1 || p->K > pppm::kMaxK) { snprintf(why, cap, "K=%d outside [-1, %d]", p->K, pppm::kMaxK); return false; }
    if (!(p->a_cells >= 0.0) || !std::isfinite(p->a_cells)) {
        snprintf(why, cap, "a_cells=%g must be finite and >= 0", p->a_cells);
        return false;
    }
    if (p->a_cells == 0.0 && (!(p->a > 0.0) || !std::isfinite(p->a))) {
        snprintf(why, cap, "smoothing radius a=%g must be > 0", p->a);
        return false;
    }
    if (p->domain_mode != PPPM_DOMAIN_BBOX3X && p->domain_mode != PPPM_DOMAIN_FIXED) {
        snprintf(why, cap, "unknown domain_mode %d", p->domain_mode);
        return false;
    }
    if (p->domain_mode == PPPM_DOMAIN_FIXED && !(p->fixed_length > 0.0 && std::isfinite(p->fixed_length))) {
        snprintf(why, cap, "fixed_length must be > 0");
        return false;
    }
    if (p->mg_mode != PPPM_MG_REFERENCE && p->mg_mode != PPPM_MG_CONVERGED) {
        snprintf(why, cap, "unknown mg_mode %d", p->mg_mode);
        return false;
    }
    if (p->mg_mode == PPPM_MG_CONVERGED && (p->mg_max_cycles < 1 || !(p->mg_tol > 0.0))) {
        snprintf(why, cap, "CONVERGED needs mg_tol > 0 and mg_max_cycles >= 1");
        return false;
    }
    return true;
}

pppm_status cuda_fail(const char *where, cudaError_t e) {
    snprintf(g_err, sizeof(g_err), "%s: %s", where, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? PPPM_ERR_OOM : PPPM_ERR_CUDA;
}

template <typename T>
cudaError_t dalloc(T **p, size_t count) {
    return ::pppm::device_malloc((void **)p, sizeof(T) * (count ? count : 1));
}

void free_vortex_side(pppm_scene *s) {
    cudaFree(s->vpos); s->vpos = nullptr;
    cudaFree(s->valpha); s->valpha = nullptr;
    for (int q = 0; q < 2; q++) { cudaFree(s->vkey[q]); cudaFree(s->vidx[q]); s->vkey[q] = s->vidx[q] = nullptr; }
    for (int q = 0; q < 2; q++) { cudaFree(s->rkey[q]); cudaFree(s->ridx[q]); s->rkey[q] = s->ridx[q] = nullptr; }
    s->ref_valid = false;
    cudaFree(s->vrec); s->vrec = nullptr;
    cudaFree(s->valf); s->valf = nullptr;
    cudaFree(s->adv_mid); s->adv_mid = nullptr;
    cudaFree(s->ts_kappa); s->ts_kappa = nullptr;
    cudaFree(s->bbox_partial); s->bbox_partial = nullptr;
}

void free_eval_side(pppm_scene *s) {
    for (int q = 0; q < 2; q++) { cudaFree(s->ekey[q]); cudaFree(s->eidx[q]); s->ekey[q] = s->eidx[q] = nullptr; }
    cudaFree(s->stage_ea); s->stage_ea = nullptr;
    cudaFree(s->stage_eb); s->stage_eb = nullptr;
    cudaFree(s->stage_out); s->stage_out = nullptr;
}

cudaError_t alloc_hist(pppm_scene *s) {
    std::lock_guard<std::recursive_mutex> lk(pppm::device_lock());
    const size_t need = pppm::radix_hist_entries(s->capN > s->capM ? s->capN : s->capM);
    if (need <= s->hist_cap) return cudaSuccess;
    cudaFree(s->hist);
    s->hist = nullptr;
    s->hist_cap = 0;
    PPPM_CUDA_TRY(dalloc(&s->hist, need));
    s->hist_cap = need;
    return cudaSuccess;
}

cudaError_t alloc_vortex_buffers(pppm_scene *s, uint32_t cap) {
    PPPM_CUDA_TRY(dalloc(&s->vpos, cap));
    PPPM_CUDA_TRY(dalloc(&s->valpha, 3 * (size_t)cap));
    for (int q = 0; q < 2; q++) {
        PPPM_CUDA_TRY(dalloc(&s->vkey[q], cap));
        PPPM_CUDA_TRY(dalloc(&s->vidx[q], cap));
        PPPM_CUDA_TRY(dalloc(&s->rkey[q], cap));
        PPPM_CUDA_TRY(dalloc(&s->ridx[q], cap));
    }
    PPPM_CUDA_TRY(dalloc(&s->vrec, cap));
    PPPM_CUDA_TRY(dalloc(&s->valf, cap));
    PPPM_CUDA_TRY(dalloc(&s->adv_mid, cap));
    PPPM_CUDA_TRY(dalloc(&s->ts_kappa, cap));
    s->bbox_blocks = 148 * 2;
    PPPM_CUDA_TRY(dalloc(&s->bbox_partial, 6 * (size_t)s->bbox_blocks));
    return cudaSuccess;
}

// A failed growth leaves the side empty with capacity 0, so that the next call
// that needs it allocates again instead of using a freed buffer.
cudaError_t alloc_vortex_side(pppm_scene *s, uint32_t cap) {
    std::lock_guard<std::recursive_mutex> lk(pppm::device_lock());
    free_vortex_side(s);
    s->capN = 0;
    s->vort_set = false;   // the vortices went with the old buffers
    s->far_ready = false;
    cudaError_t e = alloc_vortex_buffers(s, cap);
    if (e == cudaSuccess) {
        s->capN = cap;
        e = alloc_hist(s);
    }
    if (e != cudaSuccess) {
        free_vortex_side(s);
        s->capN = 0;
    }
    return e;
}

cudaError_t alloc_eval_buffers(pppm_scene *s, uint32_t cap) {
    for (int q = 0; q < 2; q++) {
        PPPM_CUDA_TRY(dalloc(&s->ekey[q], cap));
        PPPM_CUDA_TRY(dalloc(&s->eidx[q], cap));
    }
    PPPM_CUDA_TRY(dalloc(&s->stage_ea, cap));
    PPPM_CUDA_TRY(dalloc(&s->stage_eb, cap));
    PPPM_CUDA_TRY(dalloc(&s->stage_out, 3 * (size_t)cap));
    return cudaSuccess;
}

cudaError_t alloc_eval_side(pppm_scene *s, uint32_t cap) {
    std::lock_guard<std::recursive_mutex> lk(pppm::device_lock());
    free_eval_side(s);
    s->capM = 0;
    cudaError_t e = alloc_eval_buffers(s, cap);
    if (e == cudaSuccess) {
        s->capM = cap;
        e = alloc_hist(s);
    }
    if (e != cudaSuccess) {
        free_eval_side(s);
        s->capM = 0;
    }
    return e;
}

cudaError_t alloc_grid_side(pppm_scene *s) {
    const uint32_t n = s->n;
    s->C = n * n * n;
    s->levels = pppm::mg_level_count(n);
    size_t pool = 0;
    uint32_t d = n;
    for (int l = 0; l < s->levels; l++) {
        s->lv[l].d = d;
        s->lv[l].cells = d * d * d;
        pool += 2 * 3 * (size_t)s->lv[l].cells;
        d = (d / 2 == 0) ? 1 : d / 2;
    }
    PPPM_CUDA_TRY(dalloc(&s->mg_pool, pool));
    float *p = s->mg_pool;
    for (int l = 0; l < s->levels; l++) {
        s->lv[l].x = p; p += 3 * (size_t)s->lv[l].cells;
        s->lv[l].b = p; p += 3 * (size_t)s->lv[l].cells;
    }
    {
        // second x copies and tensor maps of the blocked-smoother levels
        pppm::MGPlan m;
        m.levels = s->levels;
        for (int l = 0; l < s->levels; l++) m.lv[l] = s->lv[l];
        m.comps = 3;
        const int variant = pppm::mg_tb_default_variant();
        const size_t extra = variant != -1 ? pppm::mg_tb_extra_floats(m) : 0;
        if (extra) {
            PPPM_CUDA_TRY(dalloc(&s->mg_x2_pool, extra));
            PPPM_CUDA_TRY(dalloc(&s->mg_err, 1));
            PPPM_CUDA_TRY(cudaMemset(s->mg_err, 0, sizeof(uint32_t)));
            m.err = s->mg_err;
            PPPM_CUDA_TRY(pppm::mg_tb_setup(m, s->mg_x2_pool, variant));
            for (int l = 0; l < s->levels; l++) s->lv[l].x2 = m.lv[l].x2;
        }
        s->mg_tb = m;
    }
    PPPM_CUDA_TRY(dalloc(&s->vort, 3 * (size_t)s->C));
    PPPM_CUDA_TRY(dalloc(&s->psi, 3 * (size_t)s->C));
    PPPM_CUDA_TRY(dalloc(&s->far, 3 * (size_t)s->C));
    PPPM_CUDA_TRY(dalloc(&s->cell_start, s->C));
    PPPM_CUDA_TRY(dalloc(&s->cell_end, s->C));
    PPPM_CUDA_TRY(dalloc(&s->mflag, s->C));
    PPPM_CUDA_TRY(dalloc(&s->sub_start, 8 * (size_t)s->C));
    PPPM_CUDA_TRY(dalloc(&s->sub_end, 8 * (size_t)s->C));
    PPPM_CUDA_TRY(cudaMemset(s->mflag, 0, sizeof(uint32_t) * s->C));
    PPPM_CUDA_TRY(dalloc(&s->dparams, 1));
    PPPM_CUDA_TRY(dalloc(&s->norms, 2));
    PPPM_CUDA_TRY(dalloc(&s->pair_count, 1));
    if (s->levels >= 2) {
        const int dc = (int)s->lv[s->levels - 1].d;
        const size_t cc = (size_t)dc * dc * dc;
        PPPM_CUDA_TRY(dalloc(&s->coarse_op, cc * cc));
    }
    // initialise on a private stream (no device-wide synchronisation)
    cudaStream_t st = nullptr;
    PPPM_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    cudaError_t e = cudaMemsetAsync(s->mflag, 0, sizeof(uint32_t) * s->C, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->dparams, 0, sizeof(pppm::DevParams), st);
    if (e == cudaSuccess && s->coarse_op)
        e = pppm::build_coarse_operator((int)s->lv[s->levels - 1].d, s->coarse_op, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    return e;
}

void destroy_scene(pppm_scene *s) {
    if (!s) return;
    std::lock_guard<std::recursive_mutex> lk(pppm::device_lock());
    for (int i = 0; i < 16; i++) {
        if (s->ev_begin[i]) cudaEventDestroy(s->ev_begin[i]);
        if (s->ev_end[i]) cudaEventDestroy(s->ev_end[i]);
    }
    free_vortex_side(s);
    free_eval_side(s);
    cudaFree(s->hist);
    cudaFree(s->mg_pool);
    cudaFree(s->mg_x2_pool);
    cudaFree(s->mg_err);
    cudaFree(s->vort);
    cudaFree(s->psi);
    cudaFree(s->far);
    cudaFree(s->cell_start);
    cudaFree(s->cell_end);
    cudaFree(s->mflag);
    cudaFree(s->sub_start);
    cudaFree(s->sub_end);
    cudaFree(s->dparams);
    cudaFree(s->norms);
    cudaFree(s->pair_count);
    cudaFree(s->coarse_op);
    if (s->mg_graph) cudaGraphExecDestroy(s->mg_graph);
    pppm::free_buoyancy(s->buoy);
    delete s;
}

// Evaluation with either double SoA or float interleaved output.
pppm_status eval_common(pppm_scene *s, uint32_t M, const float *ea, const float *eb, int is_segment, double *u,
                        double *v, double *w, float *uf, int count_pairs) {
    if (!s) { snprintf(g_err, sizeof(g_err), "pppm_eval: scene is NULL"); return PPPM_ERR_INVALID; }
    if (!s->far_ready) {
        snprintf(g_err, sizeof(g_err), "pppm_eval: call pppm_build_far_field after pppm_set_vortices first");
        return PPPM_ERR_STATE;
    }
    if (M == 0) return PPPM_OK;
    if (!ea || (is_segment == 1 && !eb) || (!uf && (!u || !v || !w))) {
        snprintf(g_err, sizeof(g_err), "pppm_eval: NULL pointer argument");
        return PPPM_ERR_INVALID;
    }
    if (M > s->capM) {
        cudaError_t e = alloc_eval_side(s, M);
        if (e != cudaSuccess) return cuda_fail("pppm_eval (grow eval buffers)", e);
    }
    s->M = M;
    cudaError_t e = pppm::launch_eval(s, reinterpret_cast<const float4 *>(ea), reinterpret_cast<const float4 *>(eb),
                                      is_segment, M, u, v, w, uf, count_pairs);
    if (e != cudaSuccess) return cuda_fail("pppm_eval", e);
    return PPPM_OK;
}

}  // namespace

// The first half of an evaluation for the batched path (pppm_batch_run):
// the checks and buffer growth of pppm_eval, then the points' sort; the
// evaluation itself runs later in one launch with the batch's other scenes.
pppm_status pppm_eval_batch_prepare(pppm_scene *s, uint32_t M, const float *ea, const float *eb, int is_segment,
                                    double *u, double *v, double *w, pppm::EvalArgs *args, pppm::EvalMode *mode) {
    if (!s) { snprintf(g_err, sizeof(g_err), "pppm_eval: scene is NULL"); return PPPM_ERR_INVALID; }
    if (!s->far_ready) {
        snprintf(g_err, sizeof(g_err), "pppm_eval: call pppm_build_far_field after pppm_set_vortices first");
        return PPPM_ERR_STATE;
    }
    if (M == 0) return PPPM_OK;
    if (!ea || (is_segment == 1 && !eb) || !u || !v || !w) {
        snprintf(g_err, sizeof(g_err), "pppm_eval: NULL pointer argument");
        return PPPM_ERR_INVALID;
    }
    if (M > s->capM) {
        cudaError_t e = alloc_eval_side(s, M);
        if (e != cudaSuccess) return cuda_fail("pppm_eval (grow eval buffers)", e);
    }
    s->M = M;
    cudaError_t e = pppm::eval_batch_prepare(s, reinterpret_cast<const float4 *>(ea), reinterpret_cast<const float4 *>(eb),
                                             is_segment, M, u, v, w, args, mode);
    if (e != cudaSuccess) return cuda_fail("pppm_eval", e);
    return PPPM_OK;
}

extern "C" __attribute__((visibility("hidden"))) void pppm_set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

extern "C" const char *pppm_last_error(void) { return g_err; }

extern "C" const char *pppm_version(void) { return "pppm-b200 0.1 (sm_100a)"; }

extern "C" pppm_status pppm_params_default(pppm_params *p) {
    if (!p) return PPPM_ERR_INVALID;
    memset(p, 0, sizeof(*p));
    p->n = 0;
    p->K = 1;
    p->a = 0.08;
    p->domain_mode = PPPM_DOMAIN_BBOX3X;
    p->fixed_length = 1.0;
    p->mg_mode = PPPM_MG_REFERENCE;
    p->mg_tol = 1e-10;
    p->mg_max_cycles = 50;
    return PPPM_OK;
}

extern "C" pppm_status pppm_tuning_report(char *buf, size_t cap, size_t *written) {
    if (!buf || cap == 0) {
        snprintf(g_err, sizeof(g_err), "pppm_tuning_report: empty buffer");
        return PPPM_ERR_INVALID;
    }
    const size_t w = pppm::mg_tune_report(buf, cap);
    buf[w < cap ? w : cap - 1] = 0;
    if (written) *written = w < cap ? w : cap - 1;
    return PPPM_OK;
}

extern "C" pppm_status pppm_params_accurate(pppm_params *p) {
    if (!p) return PPPM_ERR_INVALID;
    pppm_params_default(p);
    p->a_cells = 1.0;
    p->K = 3;
    p->mg_mode = PPPM_MG_CONVERGED;
    p->mg_tol = 1e-6;
    p->mg_max_cycles = 50;
    return PPPM_OK;
}

extern "C" pppm_status pppm_scene_create(const pppm_params *p, uint32_t cap_vort, uint32_t cap_eval, void *stream,
                                         pppm_scene **out) {
    if (!out) { snprintf(g_err, sizeof(g_err), "pppm_scene_create: out is NULL"); return PPPM_ERR_INVALID; }
    *out = nullptr;
    char why[256];
    if (!valid_params(p, why, sizeof(why))) {
        snprintf(g_err, sizeof(g_err), "pppm_scene_create: %s", why);
        return PPPM_ERR_INVALID;
    }
    std::lock_guard<std::recursive_mutex> lk(pppm::device_lock());
    pppm_scene *s = new pppm_scene();
    s->prm = *p;
    s->n = p->n;
    s->stream = (cudaStream_t)stream;
    {
        // PPPM_PROFILE set to anything but "" or "0": stage timing from creation on
        const char *env = std::getenv("PPPM_PROFILE");
        s->profiling = env && env[0] && std::strcmp(env, "0") != 0;
    }
    cudaGetDevice(&s->device);
    cudaError_t e = alloc_grid_side(s);
    if (e == cudaSuccess) e = alloc_vortex_side(s, cap_vort ? cap_vort : 1);
    if (e == cudaSuccess) e = alloc_eval_side(s, cap_eval ? cap_eval : 1);
    if (e == cudaSuccess) e = pppm::prepare_multigrid_graph(s);
    if (e != cudaSuccess) {
        pppm_status st = cuda_fail("pppm_scene_create", e);
        destroy_scene(s);
        return st;
    }
    *out = s;
    return PPPM_OK;
}

extern "C" pppm_status pppm_scene_destroy(pppm_scene *s) {
    if (!s) return PPPM_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    destroy_scene(s);
    return PPPM_OK;
}

extern "C" pppm_status pppm_scene_set_stream(pppm_scene *s, void *stream) {
    if (!s) return PPPM_ERR_INVALID;
    s->stream = (cudaStream_t)stream;
    return PPPM_OK;
}

extern "C" pppm_status pppm_scene_get_params(const pppm_scene *s, pppm_params *p) {
    if (!s || !p) return PPPM_ERR_INVALID;
    *p = s->prm;
    return PPPM_OK;
}

extern "C" pppm_status pppm_set_vortices(pppm_scene *s, uint32_t N, const float *pos4, const double *ax,
                                         const double *ay, const double *az) {
    if (!s || N == 0 || !pos4 || !ax || !ay || !az) {
        snprintf(g_err, sizeof(g_err), "pppm_set_vortices: NULL pointer or N == 0");
        return PPPM_ERR_INVALID;
    }
    cudaError_t e = cudaSuccess;
    if (N > s->capN) e = alloc_vortex_side(s, N);
    if (e != cudaSuccess) return cuda_fail("pppm_set_vortices (grow)", e);
    s->N = N;
    const size_t cap = s->capN;
    e = cudaMemcpyAsync(s->vpos, pos4, sizeof(float4) * N, cudaMemcpyDeviceToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->valpha, ax, sizeof(double) * N, cudaMemcpyDeviceToDevice, s->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->valpha + cap, ay, sizeof(double) * N, cudaMemcpyDeviceToDevice, s->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->valpha + 2 * cap, az, sizeof(double) * N, cudaMemcpyDeviceToDevice, s->stream);
    if (e != cudaSuccess) return cuda_fail("pppm_set_vortices", e);
    s->vort_set = true;
    s->far_ready = false;
    return PPPM_OK;
}

extern "C" pppm_status pppm_build_far_field(pppm_scene *s) {
    if (!s) return PPPM_ERR_INVALID;
    if (!s->vort_set) {
        snprintf(g_err, sizeof(g_err), "pppm_build_far_field: call pppm_set_vortices first");
        return PPPM_ERR_STATE;
    }
    using namespace pppm;
    prof_begin(s, kStageDomain);
    cudaError_t e = launch_bbox_and_params(s);
    prof_end(s, kStageDomain);
    prof_begin(s, kStageVortSort);
    if (e == cudaSuccess) e = launch_hash_sort(s, s->vpos, s->N, s->vkey, s->vidx, &s->vsorted_key, &s->vsorted_idx);
    prof_end(s, kStageVortSort);
    prof_begin(s, kStageCells);
    if (e == cudaSuccess) e = launch_cells_reorder(s);
    prof_end(s, kStageCells);
    prof_begin(s, kStageP2M);
    if (e == cudaSuccess) e = launch_p2m(s);
    prof_end(s, kStageP2M);
    prof_begin(s, kStageMG);
    if (e == cudaSuccess) e = run_multigrid(s);
    prof_end(s, kStageMG);
    prof_begin(s, kStageFar);
    if (e == cudaSuccess) e = launch_farfield(s);
    prof_end(s, kStageFar);
    if (e != cudaSuccess) return cuda_fail("pppm_build_far_field", e);
    s->far_ready = true;
    s->ref_valid = false;
    return PPPM_OK;
}

extern "C" pppm_status pppm_eval(pppm_scene *s, uint32_t M, const float *ea, const float *eb, int is_segment,
                                 double *u, double *v, double *w) {
    return eval_common(s, M, ea, eb, is_segment, u, v, w, nullptr, 0);
}

extern "C" pppm_status pppm_eval_f32(pppm_scene *s, uint32_t M, const float *ea, const float *eb, int is_segment,
                                     float *uvw) {
    return eval_common(s, M, ea, eb, is_segment, nullptr, nullptr, nullptr, uvw, 0);
}

extern "C" pppm_status pppm_count_pairs(pppm_scene *s, uint32_t M, const float *ea, uint64_t *pairs) {
    if (!s || !pairs) return PPPM_ERR_INVALID;
    std::lock_guard<std::recursive_mutex> lk(pppm::device_lock());
    float *tmp = nullptr;
    cudaError_t e = ::pppm::device_malloc((void **)&tmp, sizeof(float) * 3 * (size_t)(M ? M : 1));
    if (e != cudaSuccess) return cuda_fail("pppm_count_pairs", e);
    pppm_status st = eval_common(s, M, ea, ea, 0, nullptr, nullptr, nullptr, tmp, 1);
    unsigned long long h = 0;
    if (st == PPPM_OK) {
        e = cudaMemcpyAsync(&h, s->pair_count, sizeof(h), cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) st = cuda_fail("pppm_count_pairs", e);
    }
    cudaFree(tmp);
    *pairs = h;
    return st;
}

extern "C" pppm_status pppm_solve_host(pppm_scene *s, uint32_t N, const float *pos4_h, const double *ax_h,
                                       const double *ay_h, const double *az_h, uint32_t M, const float *ea_h,
                                       const float *eb_h, int is_segment, double *u_h, double *v_h, double *w_h) {
    if (!s || !pos4_h || !ax_h || !ay_h || !az_h || !u_h || !v_h || !w_h || N == 0) {
        snprintf(g_err, sizeof(g_err), "pppm_solve_host: NULL pointer or N == 0");
        return PPPM_ERR_INVALID;
    }
    const bool self = (ea_h == nullptr);
    if (self) { M = N; is_segment = 1; }
    if (!self && is_segment == 1 && !eb_h) {
        snprintf(g_err, sizeof(g_err), "pppm_solve_host: is_segment needs eval_b");
        return PPPM_ERR_INVALID;
    }
    // Staging buffers: the input copy lands directly in the scene's own
    // caller-order arrays; evaluation points and results use temporaries.
    cudaError_t e = cudaSuccess;
    if (N > s->capN) e = alloc_vortex_side(s, N);
    if (e != cudaSuccess) return cuda_fail("pppm_solve_host (grow)", e);
    s->N = N;
    const size_t cap = s->capN;
    cudaStream_t st = s->stream;
    e = cudaMemcpyAsync(s->vpos, pos4_h, sizeof(float4) * N, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->valpha, ax_h, sizeof(double) * N, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->valpha + cap, ay_h, sizeof(double) * N, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->valpha + 2 * cap, az_h, sizeof(double) * N, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail("pppm_solve_host (H2D)", e);
    s->vort_set = true;
    pppm_status rc = pppm_build_far_field(s);
    if (rc != PPPM_OK) return rc;
    if (M > s->capM) {
        e = alloc_eval_side(s, M);
        if (e != cudaSuccess) return cuda_fail("pppm_solve_host (grow eval buffers)", e);
    }
    float4 *ea = s->stage_ea, *eb = s->stage_eb;
    double *out = s->stage_out;
    if (!self) {
        e = cudaMemcpyAsync(ea, ea_h, sizeof(float4) * M, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && is_segment == 1)
            e = cudaMemcpyAsync(eb, eb_h, sizeof(float4) * M, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return cuda_fail("pppm_solve_host (H2D eval)", e);
    }
    const float *pa = self ? reinterpret_cast<const float *>(s->vpos) : reinterpret_cast<const float *>(ea);
    const float *pb = self ? pa : reinterpret_cast<const float *>(eb);
    rc = eval_common(s, M, pa, pb, is_segment, out, out + M, out + 2 * (size_t)M, nullptr, 0);
    if (rc == PPPM_OK) {
        e = cudaMemcpyAsync(u_h, out, sizeof(double) * M, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(v_h, out + M, sizeof(double) * M, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(w_h, out + 2 * (size_t)M, sizeof(double) * M, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = cuda_fail("pppm_solve_host (D2H)", e);
    }
    return rc;
}

// Velocity of the vortices at positions `pos` (self evaluation) into the
// scene's staging buffer; strengths must already be in the scene.
static pppm_status self_velocity(pppm_scene *s, uint32_t N, const float4 *pos) {
    cudaError_t e = cudaMemcpyAsync(s->vpos, pos, sizeof(float4) * N, cudaMemcpyDeviceToDevice, s->stream);
    if (e != cudaSuccess) return cuda_fail("advect (positions)", e);
    s->far_ready = false;
    pppm_status rc = pppm_build_far_field(s);
    if (rc != PPPM_OK) return rc;
    if (N > s->capM) {
        e = alloc_eval_side(s, N);
        if (e != cudaSuccess) return cuda_fail("advect (grow eval buffers)", e);
    }
    const float *p = reinterpret_cast<const float *>(s->vpos);
    return eval_common(s, N, p, p, 1, s->stage_out, s->stage_out + s->capM, s->stage_out + 2 * (size_t)s->capM,
                       nullptr, 0);
}

static pppm_status advect_common(pppm_scene *s, uint32_t N, float *pos4, const double *ax, const double *ay,
                                 const double *az, double dt, bool rk2) {
    if (!s || !pos4 || !ax || !ay || !az || N == 0 || !std::isfinite(dt)) {
        snprintf(g_err, sizeof(g_err), "pppm_advect: invalid argument");
        return PPPM_ERR_INVALID;
    }
    pppm_status rc = pppm_set_vortices(s, N, pos4, ax, ay, az);
    if (rc != PPPM_OK) return rc;
    float4 *x = reinterpret_cast<float4 *>(pos4);
    rc = self_velocity(s, N, x);
    if (rc != PPPM_OK) return rc;
    cudaError_t e;
    if (rk2) {
        e = pppm::launch_move(s, x, s->stage_out, s->capM, 0.5 * dt, N, s->adv_mid);
        if (e != cudaSuccess) return cuda_fail("pppm_advect_rk2 (midpoint)", e);
        rc = self_velocity(s, N, s->adv_mid);
        if (rc != PPPM_OK) return rc;
    }
    e = pppm::launch_move(s, x, s->stage_out, s->capM, dt, N, x);
    if (e != cudaSuccess) return cuda_fail("pppm_advect (move)", e);
    return PPPM_OK;
}

extern "C" pppm_status pppm_advect_euler(pppm_scene *s, uint32_t N, float *pos4, const double *ax, const double *ay,
                                         const double *az, double dt) {
    return advect_common(s, N, pos4, ax, ay, az, dt, false);
}

extern "C" pppm_status pppm_advect_rk2(pppm_scene *s, uint32_t N, float *pos4, const double *ax, const double *ay,
                                       const double *az, double dt) {
    return advect_common(s, N, pos4, ax, ay, az, dt, true);
}

// One vortex-segment time step (HFS/VortexSimulationSystemImp.cpp:90-125 without
// boundary, buoyancy, heat or shedding).  The kernels and the order of the
// reference's sub-steps are described in timestep.cu.
extern "C" pppm_status pppm_vortex_step(pppm_scene *s, uint32_t N, float *cent4, double *ax, double *ay, double *az,
                                        double dt, double h_seg, double nu, float *enda4, float *endb4, uint32_t P,
                                        float *passive4, double *pu, double *pv, double *pw) {
    if (!s || !cent4 || !ax || !ay || !az || N == 0) {
        snprintf(g_err, sizeof(g_err), "pppm_vortex_step: NULL pointer or N == 0");
        return PPPM_ERR_INVALID;
    }
    if (!std::isfinite(dt) || !(h_seg > 0.0) || !std::isfinite(h_seg) || !(nu > 0.0) || !std::isfinite(nu)) {
        snprintf(g_err, sizeof(g_err), "pppm_vortex_step: dt must be finite, h_seg and nu finite and > 0");
        return PPPM_ERR_INVALID;
    }
    if (P > 0 && (!passive4 || !pu || !pv || !pw)) {
        snprintf(g_err, sizeof(g_err), "pppm_vortex_step: passive points need positions and velocity arrays");
        return PPPM_ERR_INVALID;
    }
    if ((uint64_t)N * 2u > 0xFFFFFFFFull) {
        snprintf(g_err, sizeof(g_err), "pppm_vortex_step: N=%u too large (2N evaluation points)", N);
        return PPPM_ERR_INVALID;
    }
    using namespace pppm;
    pppm_status rc = pppm_set_vortices(s, N, cent4, ax, ay, az);
    if (rc != PPPM_OK) return rc;
    const uint32_t M = 2 * N;
    cudaError_t e = cudaSuccess;
    if (std::max(M, P) > s->capM) e = alloc_eval_side(s, std::max(M, P));
    if (e != cudaSuccess) return cuda_fail("pppm_vortex_step (grow eval buffers)", e);
    float4 *ends = s->stage_ea, *other = s->stage_eb;
    double *u = s->stage_out;
    const size_t us = s->capM;
    prof_begin(s, kStageSegments);
    e = launch_segments(s, h_seg, N, ends, other, s->ts_kappa);
    prof_end(s, kStageSegments);
    if (e != cudaSuccess) return cuda_fail("pppm_vortex_step (segments)", e);
    rc = pppm_build_far_field(s);
    if (rc != PPPM_OK) return rc;
    rc = eval_common(s, M, reinterpret_cast<const float *>(ends), reinterpret_cast<const float *>(other), 1, u,
                     u + us, u + 2 * us, nullptr, 0);
    if (rc != PPPM_OK) return rc;
    // tracers and heat particles: plain evaluation with the same far field,
    // then move_particle (evaluateBiotSavart, VSSImp.cpp:1195-1244)
    if (P > 0) {
        rc = eval_common(s, P, passive4, passive4, 0, pu, pv, pw, nullptr, 0);
        if (rc != PPPM_OK) return rc;
        e = launch_move3(s, reinterpret_cast<float4 *>(passive4), pu, pv, pw, dt, P);
        if (e != cudaSuccess) return cuda_fail("pppm_vortex_step (passive move)", e);
    }
    // From here the scene's vortex copy holds the moved centres and the
    // unsmoothed strengths: its far field no longer matches them.
    s->far_ready = false;
    s->vort_set = false;
    s->ref_valid = false;
    prof_begin(s, kStageSegToBlob);
    e = launch_segment_to_blob(s, ends, u, us, s->ts_kappa, dt, N, reinterpret_cast<float4 *>(cent4),
                               reinterpret_cast<float4 *>(enda4), reinterpret_cast<float4 *>(endb4));
    prof_end(s, kStageSegToBlob);
    if (e != cudaSuccess) return cuda_fail("pppm_vortex_step (move)", e);
    prof_begin(s, kStageRehash);
    e = launch_bbox_and_params(s);
    if (e == cudaSuccess) e = launch_hash_sort(s, s->vpos, N, s->vkey, s->vidx, &s->vsorted_key, &s->vsorted_idx);
    if (e == cudaSuccess) e = launch_cells_reorder(s);
    prof_end(s, kStageRehash);
    if (e != cudaSuccess) return cuda_fail("pppm_vortex_step (hash)", e);
    prof_begin(s, kStageSmooth);
    e = launch_gaussian_smooth(s, nu, N, ax, ay, az);
    prof_end(s, kStageSmooth);
    if (e != cudaSuccess) return cuda_fail("pppm_vortex_step (smoothing)", e);
    return PPPM_OK;
}

extern "C" pppm_status pppm_get_domain(pppm_scene *s, double origin[3], double *length, double *cell_h) {
    if (!s) return PPPM_ERR_INVALID;
    if (!s->far_ready) { snprintf(g_err, sizeof(g_err), "pppm_get_domain: no far field built"); return PPPM_ERR_STATE; }
    pppm::DevParams h;
    cudaError_t e = cudaMemcpyAsync(&h, s->dparams, sizeof(h), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return cuda_fail("pppm_get_domain", e);
    if (origin) { origin[0] = h.origin[0]; origin[1] = h.origin[1]; origin[2] = h.origin[2]; }
    if (length) *length = h.length;
    if (cell_h) *cell_h = h.cell_h;
    if (h.status != 0) { snprintf(g_err, sizeof(g_err), "degenerate domain (L = %g)", h.length); return PPPM_ERR_DOMAIN; }
    return PPPM_OK;
}

extern "C" pppm_status pppm_get_smoothing(pppm_scene *s, double *a) {
    if (!s || !a) return PPPM_ERR_INVALID;
    if (!s->far_ready) { snprintf(g_err, sizeof(g_err), "pppm_get_smoothing: no far field built"); return PPPM_ERR_STATE; }
    pppm::DevParams h;
    cudaError_t e = cudaMemcpyAsync(&h, s->dparams, sizeof(h), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return cuda_fail("pppm_get_smoothing", e);
    *a = h.a;
    return PPPM_OK;
}

extern "C" pppm_status pppm_get_cell_tables(pppm_scene *s, const uint32_t **start, const uint32_t **end) {
    if (!s) return PPPM_ERR_INVALID;
    if (!s->far_ready) { snprintf(g_err, sizeof(g_err), "pppm_get_cell_tables: no far field built"); return PPPM_ERR_STATE; }
    if (start) *start = s->cell_start;
    if (end) *end = s->cell_end;
    return PPPM_OK;
}

extern "C" pppm_status pppm_get_sorted_index(pppm_scene *s, const uint32_t **key, const uint32_t **idx) {
    if (!s) return PPPM_ERR_INVALID;
    if (!s->far_ready) { snprintf(g_err, sizeof(g_err), "pppm_get_sorted_index: no far field built"); return PPPM_ERR_STATE; }
    if (!s->ref_valid) {
        cudaError_t e = pppm::launch_reference_order(s);
        if (e != cudaSuccess) return cuda_fail("pppm_get_sorted_index", e);
        s->ref_valid = true;
    }
    if (key) *key = s->ref_sorted_key;
    if (idx) *idx = s->ref_sorted_idx;
    return PPPM_OK;
}

extern "C" pppm_status pppm_get_sorted_vortices(pppm_scene *s, float *pos4, double *ax, double *ay, double *az) {
    if (!s) return PPPM_ERR_INVALID;
    if (!s->far_ready) {
        snprintf(g_err, sizeof(g_err), "pppm_get_sorted_vortices: no far field built");
        return PPPM_ERR_STATE;
    }
    std::lock_guard<std::recursive_mutex> lk(pppm::device_lock());
    double *tmp = nullptr;
    cudaError_t e = cudaSuccess;
    if (!s->ref_valid) {
        e = pppm::launch_reference_order(s);
        if (e != cudaSuccess) return cuda_fail("pppm_get_sorted_vortices", e);
        s->ref_valid = true;
    }
    if (ax || ay || az) e = ::pppm::device_malloc((void **)&tmp, sizeof(double) * 3 * (size_t)s->N);
    if (e == cudaSuccess) e = pppm::launch_gather_sorted(s, reinterpret_cast<float4 *>(pos4), tmp);
    const size_t N = s->N;
    if (e == cudaSuccess && ax) e = cudaMemcpyAsync(ax, tmp, sizeof(double) * N, cudaMemcpyDeviceToDevice, s->stream);
    if (e == cudaSuccess && ay) e = cudaMemcpyAsync(ay, tmp + N, sizeof(double) * N, cudaMemcpyDeviceToDevice, s->stream);
    if (e == cudaSuccess && az)
        e = cudaMemcpyAsync(az, tmp + 2 * N, sizeof(double) * N, cudaMemcpyDeviceToDevice, s->stream);
    if (e == cudaSuccess && tmp) e = cudaStreamSynchronize(s->stream);
    cudaFree(tmp);
    if (e != cudaSuccess) return cuda_fail("pppm_get_sorted_vortices", e);
    return PPPM_OK;
}

extern "C" pppm_status pppm_get_grid(pppm_scene *s, int which, const void **ptr) {
    if (!s || !ptr) return PPPM_ERR_INVALID;
    switch (which) {
        case PPPM_GRID_VORT: *ptr = s->vort; break;
        case PPPM_GRID_PSI: *ptr = s->psi; break;
        case PPPM_GRID_FAR: *ptr = s->far; break;
        default: snprintf(g_err, sizeof(g_err), "pppm_get_grid: unknown grid %d", which); return PPPM_ERR_INVALID;
    }
    return PPPM_OK;
}

namespace pppm {

std::recursive_mutex &device_lock() {
    static std::recursive_mutex m;
    return m;
}

static std::atomic<unsigned long long> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
unsigned long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

const char *stage_name(int i) {
    static const char *names[kNumStages] = {"domain", "vort_sort", "cells_reorder", "p2m",
                                            "multigrid", "farfield", "eval_sort", "eval",
                                            "segments", "seg_to_blob", "rehash", "gaussian_smooth"};
    return (i >= 0 && i < kNumStages) ? names[i] : "";
}

void prof_begin(pppm_scene *s, int stage) {
    if (!s->profiling) return;
    if (!s->ev_begin[stage]) {
        cudaEventCreate(&s->ev_begin[stage]);
        cudaEventCreate(&s->ev_end[stage]);
    }
    cudaEventRecord(s->ev_begin[stage], s->stream);
}

void prof_end(pppm_scene *s, int stage) {
    if (!s->profiling) return;
    cudaEventRecord(s->ev_end[stage], s->stream);
    s->ev_used[stage] = true;
}

}  // namespace pppm

extern "C" pppm_status pppm_scene_set_profiling(pppm_scene *s, int on) {
    if (!s) return PPPM_ERR_INVALID;
    s->profiling = on != 0;
    for (int i = 0; i < 16; i++) s->ev_used[i] = false;
    return PPPM_OK;
}

extern "C" const char *pppm_stage_name(int i) { return pppm::stage_name(i); }

extern "C" uint64_t pppm_kernel_launches(void) { return pppm::launch_count(); }

extern "C" pppm_status pppm_get_stage_times(pppm_scene *s, double *ms, int cap, int *count) {
    if (!s || !ms || cap < pppm::kNumStages) return PPPM_ERR_INVALID;
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return cuda_fail("pppm_get_stage_times", e);
    for (int i = 0; i < pppm::kNumStages; i++) {
        ms[i] = -1.0;
        if (s->profiling && s->ev_used[i]) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, s->ev_begin[i], s->ev_end[i]) == cudaSuccess) ms[i] = t;
        }
    }
    if (count) *count = pppm::kNumStages;
    return PPPM_OK;
}

extern "C" pppm_status pppm_get_stats(pppm_scene *s, uint64_t *pairs, int32_t *mg_cycles, double *mg_relres) {
    if (!s) return PPPM_ERR_INVALID;
    if (pairs) {
        unsigned long long h = 0;
        cudaError_t e = cudaMemcpyAsync(&h, s->pair_count, sizeof(h), cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) return cuda_fail("pppm_get_stats", e);
        *pairs = h;
    }
    if (mg_cycles) *mg_cycles = s->mg_cycles_last;
    if (mg_relres) *mg_relres = s->mg_relres_last;
    return PPPM_OK;
}

// ---------------------------------------------------------------------------
// gf::MultiGridSolver3DPeriod_double surface (MG/MultiGrid.h:188-209).
// ---------------------------------------------------------------------------
struct pppm_mg {
    pppm::MGPlan plan;
    float *pool = nullptr;
    float *x2_pool = nullptr;               // second x copies of the blocked-smoother levels
    uint32_t *err = nullptr;                // its device error flag
    double *r64 = nullptr, *e64 = nullptr;  // residual of the initial guess, its correction
    double *coarse_op = nullptr;            // coarsest-level operator (levels >= 2)
    cudaGraphExec_t graph = nullptr;        // reference-schedule solve of r64 into e64, captured on first use
    unsigned graph_kernels = 0;
    uint32_t n = 0;
};

namespace {
__global__ void to_float_kernel(const double *__restrict__ in, float *__restrict__ out, size_t count) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) out[t] = (float)in[t];
}

// r = b - (sum_nbr(x) - 6x) with zero ghost values, FP64; the FP32 copy seeds
// the finest multigrid level.
__global__ void residual64_kernel(const double *__restrict__ x, const double *__restrict__ b, double *__restrict__ r,
                                  float *__restrict__ r32, int d) {
    const size_t C = (size_t)d * d * d;
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= C) return;
    const int i = (int)(t % d), j = (int)((t / d) % d), k = (int)(t / ((size_t)d * d));
    const size_t dd = (size_t)d * d;
    const double lv = (i > 0) ? x[t - 1] : 0.0, rv = (i < d - 1) ? x[t + 1] : 0.0;
    const double uv = (j < d - 1) ? x[t + d] : 0.0, dv = (j > 0) ? x[t - d] : 0.0;
    const double fv = (k > 0) ? x[t - dd] : 0.0, bv = (k < d - 1) ? x[t + dd] : 0.0;
    const double v = b[t] - ((((lv + rv) + (uv + dv)) + (fv + bv)) - 6.0 * x[t]);
    r[t] = v;
    r32[t] = (float)v;
}

__global__ void add64_kernel(double *__restrict__ x, const double *__restrict__ e, size_t count) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) x[t] += e[t];
}
}  // namespace

extern "C" pppm_status pppm_mg_create(uint32_t n, void *stream, pppm_mg **out) {
    if (!out || n < 2 || n > 512 || !pppm::mg_shape_ok(n)) {
        snprintf(g_err, sizeof(g_err), "pppm_mg_create: unsupported grid edge %u", n);
        return PPPM_ERR_INVALID;
    }
    std::lock_guard<std::recursive_mutex> lk(pppm::device_lock());
    pppm_mg *m = new pppm_mg();
    m->n = n;
    pppm::MGPlan &P = m->plan;
    P.comps = 1;
    P.st = (cudaStream_t)stream;
    P.levels = pppm::mg_level_count(n);
    size_t pool = 0;
    uint32_t d = n;
    for (int l = 0; l < P.levels; l++) {
        P.lv[l].d = d;
        P.lv[l].cells = d * d * d;
        pool += 2 * (size_t)P.lv[l].cells;
        d = (d / 2 == 0) ? 1 : d / 2;
    }
    cudaError_t e = dalloc(&m->pool, pool);
    if (e == cudaSuccess) e = dalloc(&P.norms, 2);
    if (e == cudaSuccess) e = dalloc(&m->r64, P.lv[0].cells);
    if (e == cudaSuccess) e = dalloc(&m->e64, P.lv[0].cells);
    if (e == cudaSuccess && P.levels >= 2) {
        // the coarsest solve from x = 0 as one precomputed linear map, as for scenes
        const uint32_t cc = P.lv[P.levels - 1].cells;
        e = dalloc(&m->coarse_op, (size_t)cc * cc);
        if (e == cudaSuccess) e = pppm::build_coarse_operator((int)P.lv[P.levels - 1].d, m->coarse_op, P.st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(P.st);
        P.coarse_op = m->coarse_op;
    }
    if (e != cudaSuccess) {
        pppm_status st = cuda_fail("pppm_mg_create", e);
        cudaFree(m->pool);
        cudaFree(P.norms);
        cudaFree(m->r64);
        cudaFree(m->e64);
        cudaFree(m->coarse_op);
        delete m;
        return st;
    }
    float *p = m->pool;
    for (int l = 0; l < P.levels; l++) {
        P.lv[l].x = p; p += P.lv[l].cells;
        P.lv[l].b = p; p += P.lv[l].cells;
    }
    {
        const int variant = pppm::mg_tb_default_variant();
        const size_t extra = variant != -1 ? pppm::mg_tb_extra_floats(P) : 0;
        if (extra) {
            e = dalloc(&m->x2_pool, extra);
            if (e == cudaSuccess) e = dalloc(&m->err, 1);
            if (e == cudaSuccess) e = cudaMemset(m->err, 0, sizeof(uint32_t));
            P.err = m->err;
            if (e == cudaSuccess) e = pppm::mg_tb_setup(P, m->x2_pool, variant);
        }
        if (e != cudaSuccess) {
            pppm_status st = cuda_fail("pppm_mg_create", e);
            cudaFree(m->pool);
            cudaFree(P.norms);
            cudaFree(m->r64);
            cudaFree(m->e64);
            cudaFree(m->coarse_op);
            cudaFree(m->x2_pool);
            cudaFree(m->err);
            delete m;
            return st;
        }
    }
    *out = m;
    return PPPM_OK;
}

extern "C" pppm_status pppm_mg_destroy(pppm_mg *m) {
    if (!m) return PPPM_OK;
    if (m->plan.st) cudaStreamSynchronize(m->plan.st);
    std::lock_guard<std::recursive_mutex> lk(pppm::device_lock());
    if (m->graph) cudaGraphExecDestroy(m->graph);
    cudaFree(m->pool);
    cudaFree(m->plan.norms);
    cudaFree(m->r64);
    cudaFree(m->e64);
    cudaFree(m->coarse_op);
    cudaFree(m->x2_pool);
    cudaFree(m->err);
    delete m;
    return PPPM_OK;
}

extern "C" pppm_status pppm_mg_full_multigrid(pppm_mg *m, double *x, const double *b, int mode, double tol,
                                              int max_cycles, double *relres) {
    if (!m || !x || !b || (mode != PPPM_MG_REFERENCE && mode != PPPM_MG_CONVERGED)) {
        snprintf(g_err, sizeof(g_err), "pppm_mg_full_multigrid: invalid argument");
        return PPPM_ERR_INVALID;
    }
    // The reference's full multigrid starts from the x it is given (its first
    // residual is b - A x, MG/MultiGrid.cpp:211-226): solve for the correction
    // e of r = b - A x and add it, x + FMG(0, r), which is the same linear
    // iteration (and exactly the plain solve when x = 0).
    pppm::MGPlan P = m->plan;
    P.psi = m->e64;
    P.b64 = m->r64;
    P.vort = nullptr;
    P.P = nullptr;
    const size_t C = P.lv[0].cells;
    ::pppm::note_launch();
    residual64_kernel<<<(unsigned)((C + 255) / 256), 256, 0, P.st>>>(x, b, m->r64, P.lv[0].b, (int)P.lv[0].d);
    cudaError_t e = cudaGetLastError();
    int cyc = 0;
    double rel = -1.0;
    if (e == cudaSuccess && mode == PPPM_MG_REFERENCE) {
        // the fixed schedule touches only this object's buffers: one graph
        // launch, captured on first use
        if (!m->graph) {
            std::lock_guard<std::recursive_mutex> lk(pppm::device_lock());
            e = pppm::mg_capture_graph(P, &m->graph, &m->graph_kernels);
            if (e != cudaSuccess) m->graph = nullptr;
        }
        if (e == cudaSuccess) e = cudaGraphLaunch(m->graph, P.st);
        for (unsigned q = 0; e == cudaSuccess && q < m->graph_kernels; q++) ::pppm::note_launch();
    } else if (e == cudaSuccess) {
        e = pppm::mg_solve(P, mode, tol, max_cycles > 0 ? max_cycles : 1, &cyc, &rel);
    }
    if (e == cudaSuccess) {
        ::pppm::note_launch();
        add64_kernel<<<(unsigned)((C + 255) / 256), 256, 0, P.st>>>(x, m->e64, C);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return cuda_fail("pppm_mg_full_multigrid", e);
    if (relres) *relres = rel;
    return PPPM_OK;
}

extern "C" pppm_status pppm_mg_levels(const pppm_mg *m, int *levels, uint32_t *edges, int cap) {
    if (!m || !levels) {
        snprintf(g_err, sizeof(g_err), "pppm_mg_levels: invalid argument");
        return PPPM_ERR_INVALID;
    }
    *levels = m->plan.levels;
    for (int l = 0; edges && l < m->plan.levels && l < cap; l++) edges[l] = m->plan.lv[l].d;
    return PPPM_OK;
}

extern "C" pppm_status pppm_mg_vcycle(pppm_mg *m, double *x, const double *b, int level) {
    if (!m || !x || !b || level < 0 || level >= m->plan.levels) {
        snprintf(g_err, sizeof(g_err), "pppm_mg_vcycle: invalid argument (level %d of %d)", level,
                 m ? m->plan.levels : 0);
        return PPPM_ERR_INVALID;
    }
    // The cycle runs on the levels from `level` down; x and b are that level's
    // FP64 arrays.  r = b - A x seeds the level's FP32 right-hand side, the
    // FP32 V-cycle solves for the correction from zero, and x += e.
    pppm::MGPlan P = m->plan;
    P.levels = m->plan.levels - level;
    for (int l = 0; l < P.levels; l++) {
        P.lv[l] = m->plan.lv[level + l];
        P.tb_maps[l] = m->plan.tb_maps[level + l];
        P.tb_zchunk[l] = m->plan.tb_zchunk[level + l];
    }
    P.coarse_op = (P.levels >= 2) ? m->coarse_op : nullptr;
    const size_t C = P.lv[0].cells;
    ::pppm::note_launch();
    residual64_kernel<<<(unsigned)((C + 255) / 256), 256, 0, P.st>>>(x, b, m->r64, P.lv[0].b, (int)P.lv[0].d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = pppm::mg_vcycle_update(P, x);
    if (e != cudaSuccess) return cuda_fail("pppm_mg_vcycle", e);
    return PPPM_OK;
}

// ---------------------------------------------------------------------------
// FP64 direct sum (ground truth for the error reports).
// ---------------------------------------------------------------------------
namespace {

constexpr int kDSThreads = 128;

__global__ void __launch_bounds__(kDSThreads)
direct_sum_kernel(uint32_t N, const float4 *__restrict__ vp, const double *__restrict__ ax,
                  const double *__restrict__ ay, const double *__restrict__ az, uint32_t M,
                  const float4 *__restrict__ ea, const float4 *__restrict__ eb, int is_segment, double a,
                  double *__restrict__ u, double *__restrict__ v, double *__restrict__ w) {
    __shared__ double sx[kDSThreads], sy[kDSThreads], sz[kDSThreads], sa[kDSThreads], sb[kDSThreads],
        sc[kDSThreads];
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    double xa = 0, ya = 0, za = 0, xb = 0, yb = 0, zb = 0;
    if (t < M) {
        xa = ea[t].x; ya = ea[t].y; za = ea[t].z;
        if (is_segment == 1) { xb = eb[t].x; yb = eb[t].y; zb = eb[t].z; }
    }
    const double inva = 1.0 / a;
    double ox = 0, oy = 0, oz = 0;
    for (uint32_t base = 0; base < N; base += kDSThreads) {
        const uint32_t p = base + threadIdx.x;
        if (p < N) {
            const float4 q = vp[p];
            sx[threadIdx.x] = q.x; sy[threadIdx.x] = q.y; sz[threadIdx.x] = q.z;
            sa[threadIdx.x] = ax[p]; sb[threadIdx.x] = ay[p]; sc[threadIdx.x] = az[p];
        }
        __syncthreads();
        const uint32_t cnt = min((uint32_t)kDSThreads, N - base);
        if (t < M) {
            for (uint32_t q = 0; q < cnt; q++) {
                const double dx = xa - sx[q], dy = ya - sy[q], dz = za - sz[q];
                const double r2 = dx * dx + dy * dy + dz * dz;
                if (r2 == 0.0) continue;
                if (is_segment == 1 && xb == sx[q] && yb == sy[q] && zb == sz[q]) continue;
                const double r = sqrt(r2);
                const double s = r * inva;
                const double s3 = s * s * s;
                const double c = (s3 > 1e-8) ? -expm1(-s3) / (pppm::kFourPi * r2 * r)
                                             : (1.0 - 0.5 * s3) * inva * inva * inva / pppm::kFourPi;
                ox += (sb[q] * dz - sc[q] * dy) * c;
                oy += (sc[q] * dx - sa[q] * dz) * c;
                oz += (sa[q] * dy - sb[q] * dx) * c;
            }
        }
        __syncthreads();
    }
    if (t < M) { u[t] = ox; v[t] = oy; w[t] = oz; }
}

}  // namespace

extern "C" pppm_status pppm_direct_sum_fp64(uint32_t N, const float *vp, const double *ax, const double *ay,
                                            const double *az, uint32_t M, const float *ea, const float *eb,
                                            int is_segment, double a, double *u, double *v, double *w,
                                            void *stream) {
    if (!vp || !ax || !ay || !az || !ea || !u || !v || !w || (is_segment == 1 && !eb) || !(a > 0.0)) {
        snprintf(g_err, sizeof(g_err), "pppm_direct_sum_fp64: invalid argument");
        return PPPM_ERR_INVALID;
    }
    if (M == 0 || N == 0) return PPPM_OK;
    ::pppm::note_launch();
    direct_sum_kernel<<<(M + kDSThreads - 1) / kDSThreads, kDSThreads, 0, (cudaStream_t)stream>>>(
        N, reinterpret_cast<const float4 *>(vp), ax, ay, az, M, reinterpret_cast<const float4 *>(ea),
        reinterpret_cast<const float4 *>(eb), is_segment, a, u, v, w);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail("pppm_direct_sum_fp64", e);
    return PPPM_OK;
}
