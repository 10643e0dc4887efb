// Many independent scenes in one call (no reference counterpart: the
// reference drives one solver from one host thread,
// HFS/VortexSimulationSystemImp.cpp:1195-1244).
//
// Two phases.  (1) Each scene's set_vortices + build_far_field and the sort of
// its evaluation points run on a stream of its own from a set of streams the
// call borrows; scenes are dealt to the streams longest predicted build
// first, each to the least loaded stream.  (2) The evaluations of all scenes
// then run as ONE launch over a work list of (scene, block of 128 points)
// items, the blocks of the scenes with the most near-field pairs per point
// first, so the block scheduler hands out the longest work first and small
// scenes fill in behind; scenes that cannot share a launch (another
// smoothing series or segment mode) get one launch per group.  Each point is
// computed by exactly the arithmetic of the one-scene kernel, with no
// cross-scene reduction, so a scene's result does not depend on the batch.
//
// Concurrent callers borrow different stream sets, so their batches overlap
// on the device; nothing is serialised beyond the set's own bookkeeping.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "pppm_internal.cuh"

extern "C" __attribute__((visibility("hidden"))) void pppm_set_error(const char *fmt, ...);
pppm_status pppm_eval_batch_prepare(pppm_scene *s, uint32_t M, const float *ea, const float *eb, int is_segment,
                                    double *u, double *v, double *w, pppm::EvalArgs *args, pppm::EvalMode *mode);

namespace {

constexpr int kSetStreams = 16;

struct StreamSet {
    int device = -1;
    bool busy = false;
    cudaStream_t s[kSetStreams] = {};
    cudaEvent_t done[kSetStreams] = {};
    cudaEvent_t start = nullptr;
    cudaEvent_t lists_read = nullptr;  // the device has copied this set's host lists
    // work list and per-scene arguments: pinned host staging, device copies
    pppm::EvalArgs *args_h = nullptr, *args_d = nullptr;
    uint2 *work_h = nullptr, *work_d = nullptr;
    size_t cap_args = 0, cap_work = 0;
};

std::mutex g_sets_mutex;
std::vector<StreamSet *> g_sets;

cudaError_t acquire_set(StreamSet **out) {
    int dev = 0;
    PPPM_CUDA_TRY(cudaGetDevice(&dev));
    StreamSet *set = nullptr;
    {
        // a free set whose previous batch the device has finished reading
        // (its lists and work buffers are reused); else a new set
        std::lock_guard<std::mutex> lock(g_sets_mutex);
        for (StreamSet *p : g_sets)
            if (!p->busy && p->device == dev && cudaEventQuery(p->lists_read) == cudaSuccess) {
                set = p;
                break;
            }
        if (set) set->busy = true;
    }
    if (!set) {
        set = new StreamSet();
        set->device = dev;
        set->busy = true;
        cudaError_t e = cudaSuccess;
        for (int i = 0; i < kSetStreams && e == cudaSuccess; i++) {
            e = cudaStreamCreateWithFlags(&set->s[i], cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&set->done[i], cudaEventDisableTiming);
        }
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&set->start, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&set->lists_read, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            delete set;  // (handles created so far are left to the process)
            return e;
        }
        std::lock_guard<std::mutex> lock(g_sets_mutex);
        g_sets.push_back(set);
    }
    *out = set;
    return cudaSuccess;
}

void release_set(StreamSet *set) {
    std::lock_guard<std::mutex> lock(g_sets_mutex);
    set->busy = false;
}

cudaError_t ensure_lists(StreamSet *set, size_t nargs, size_t nwork) {
    if (nargs > set->cap_args) {
        cudaFreeHost(set->args_h);
        cudaFree(set->args_d);
        set->args_h = nullptr;
        set->args_d = nullptr;
        set->cap_args = 0;
        PPPM_CUDA_TRY(pppm::host_malloc((void **)&set->args_h, sizeof(pppm::EvalArgs) * nargs));
        PPPM_CUDA_TRY(pppm::device_malloc((void **)&set->args_d, sizeof(pppm::EvalArgs) * nargs));
        set->cap_args = nargs;
    }
    if (nwork > set->cap_work) {
        cudaFreeHost(set->work_h);
        cudaFree(set->work_d);
        set->work_h = nullptr;
        set->work_d = nullptr;
        set->cap_work = 0;
        PPPM_CUDA_TRY(pppm::host_malloc((void **)&set->work_h, sizeof(uint2) * nwork));
        PPPM_CUDA_TRY(pppm::device_malloc((void **)&set->work_d, sizeof(uint2) * nwork));
        set->cap_work = nwork;
    }
    return cudaSuccess;
}

// Predicted cost of a scene's far-field build (cells of all levels plus the
// particle passes) and of its evaluation per point (particles per cell).
double build_cost(const pppm_batch_item &it) {
    const double n = (double)it.scene->n;
    return 1.15 * n * n * n * 3.0 + 8.0 * (double)it.N;
}
double pairs_per_point(const pppm_batch_item &it) {
    const double n = (double)it.scene->n;
    return (double)it.N / (n * n * n);
}

}  // namespace

extern "C" pppm_status pppm_batch_run(pppm_batch_item *items, uint32_t count, void *stream) {
    if (!items && count) {
        pppm_set_error("pppm_batch_run: items is NULL");
        return PPPM_ERR_INVALID;
    }
    for (uint32_t i = 0; i < count; i++) {
        if (!items[i].scene) {
            pppm_set_error("pppm_batch_run: item %u has no scene", i);
            return PPPM_ERR_INVALID;
        }
        for (uint32_t j = 0; j < i; j++)
            if (items[j].scene == items[i].scene) {
                pppm_set_error("pppm_batch_run: scene of item %u repeats item %u (a scene runs once per batch)", i, j);
                return PPPM_ERR_INVALID;
            }
    }
    if (count == 0) return PPPM_OK;
    StreamSet *set = nullptr;
    cudaError_t e = acquire_set(&set);
    if (e != cudaSuccess) {
        pppm_set_error("pppm_batch_run: stream set: %s", cudaGetErrorString(e));
        return PPPM_ERR_CUDA;
    }
    cudaStream_t caller = (cudaStream_t)stream;
    const int used = (int)std::min<uint32_t>(count, (uint32_t)kSetStreams);
    e = cudaEventRecord(set->start, caller);
    for (int q = 0; q < used && e == cudaSuccess; q++) e = cudaStreamWaitEvent(set->s[q], set->start, 0);
    if (e != cudaSuccess) {
        release_set(set);
        pppm_set_error("pppm_batch_run: %s", cudaGetErrorString(e));
        return PPPM_ERR_CUDA;
    }

    // phase 1: builds and sorts, longest predicted build first onto the least
    // loaded stream
    std::vector<uint32_t> order(count);
    for (uint32_t i = 0; i < count; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return build_cost(items[a]) > build_cost(items[b]); });
    std::vector<double> load(used, 0.0);
    std::vector<pppm::EvalArgs> args(count);
    std::vector<pppm::EvalMode> modes(count);
    std::vector<char> has_eval(count, 0);
    pppm_status rc = PPPM_OK;
    uint32_t failed = 0;
    for (uint32_t k = 0; k < count && rc == PPPM_OK; k++) {
        const uint32_t i = order[k];
        pppm_batch_item &it = items[i];
        const int q = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        load[q] += build_cost(it) + (double)it.M * pairs_per_point(it);
        pppm_scene *s = it.scene;
        cudaStream_t own = s->stream;
        s->stream = set->s[q];
        rc = pppm_set_vortices(s, it.N, it.pos4_dev, it.ax_dev, it.ay_dev, it.az_dev);
        if (rc == PPPM_OK) rc = pppm_build_far_field(s);
        if (rc == PPPM_OK && it.M) {
            rc = pppm_eval_batch_prepare(s, it.M, it.eval_a4_dev, it.eval_b4_dev, it.is_segment, it.u_dev, it.v_dev,
                                         it.w_dev, &args[i], &modes[i]);
            has_eval[i] = (rc == PPPM_OK);
        }
        s->stream = own;
        failed = i;
    }
    // join: the caller's stream waits for every stream of the set
    for (int q = 0; q < used; q++) {
        cudaEventRecord(set->done[q], set->s[q]);
        cudaStreamWaitEvent(caller, set->done[q], 0);
    }
    if (rc != PPPM_OK) {
        char buf[256];
        snprintf(buf, sizeof(buf), "%s", pppm_last_error());
        release_set(set);
        pppm_set_error("pppm_batch_run: item %u: %s", failed, buf);
        return rc;
    }

    // phase 2: one evaluation launch per group of scenes sharing a mode, its
    // work list ordered by pairs per point
    std::vector<uint32_t> ev;
    size_t nwork = 0;
    for (uint32_t i = 0; i < count; i++)
        if (has_eval[i]) {
            ev.push_back(i);
            nwork += (items[i].M + 127) / 128;
        }
    std::stable_sort(ev.begin(), ev.end(),
                     [&](uint32_t a, uint32_t b) { return pairs_per_point(items[a]) > pairs_per_point(items[b]); });
    e = ensure_lists(set, ev.size(), nwork);
    size_t wpos = 0;
    std::vector<char> done(count, 0);
    uint32_t a_pos = 0;
    for (size_t g0 = 0; g0 < ev.size() && e == cudaSuccess; g0++) {
        const uint32_t lead = ev[g0];
        if (done[lead]) continue;
        const uint32_t a_first = a_pos;
        const size_t w_first = wpos;
        for (size_t g = g0; g < ev.size(); g++) {
            const uint32_t i = ev[g];
            if (done[i] || !modes[i].same(modes[lead])) continue;
            done[i] = 1;
            set->args_h[a_pos] = args[i];
            const uint32_t blocks = (items[i].M + 127) / 128;
            for (uint32_t b = 0; b < blocks; b++) set->work_h[wpos++] = make_uint2(a_pos - a_first, b);
            a_pos++;
        }
        const uint32_t nargs = a_pos - a_first;
        const uint32_t nblocks = (uint32_t)(wpos - w_first);
        e = cudaMemcpyAsync(set->args_d + a_first, set->args_h + a_first, sizeof(pppm::EvalArgs) * nargs,
                            cudaMemcpyHostToDevice, caller);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(set->work_d + w_first, set->work_h + w_first, sizeof(uint2) * nblocks,
                                cudaMemcpyHostToDevice, caller);
        if (e == cudaSuccess)
            e = pppm::launch_eval_batch(modes[lead], set->args_d + a_first, set->work_d + w_first, nblocks, caller);
    }
    if (e == cudaSuccess) e = cudaEventRecord(set->lists_read, caller);
    release_set(set);
    if (e != cudaSuccess) {
        pppm_set_error("pppm_batch_run: evaluation: %s", cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? PPPM_ERR_OOM : PPPM_ERR_CUDA;
    }
    return PPPM_OK;
}
