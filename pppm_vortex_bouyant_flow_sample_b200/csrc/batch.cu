// Many independent scenes in one call.  Scenes share nothing, so each one's
// far-field build and evaluation run on a stream of its own from a pool the
// library keeps per device; small scenes, which alone leave most of the GPU
// idle between their short kernels, then overlap.  The caller's stream first
// orders the pool streams after its earlier work and finally waits for all of
// them, so the batch behaves like one stream-ordered operation.  Results are
// computed by exactly the kernels a single scene uses, with no cross-scene
// reduction, so each scene's output does not depend on what else is in the
// batch.
#include <cstdio>
#include <mutex>
#include <vector>

#include "pppm_internal.cuh"

extern "C" __attribute__((visibility("hidden"))) void pppm_set_error(const char *fmt, ...);

namespace {

constexpr int kPoolStreams = 16;
constexpr int kMaxDevices = 64;

struct StreamPool {
    cudaStream_t s[kPoolStreams] = {};
    cudaEvent_t done[kPoolStreams] = {};
    cudaEvent_t start = nullptr;
    bool ready = false;
};

std::mutex g_pool_mutex;
StreamPool g_pools[kMaxDevices];

cudaError_t pool_for_device(StreamPool **out) {
    int dev = 0;
    PPPM_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    StreamPool &p = g_pools[dev];
    if (!p.ready) {
        for (int i = 0; i < kPoolStreams; i++) {
            PPPM_CUDA_TRY(cudaStreamCreateWithFlags(&p.s[i], cudaStreamNonBlocking));
            PPPM_CUDA_TRY(cudaEventCreateWithFlags(&p.done[i], cudaEventDisableTiming));
        }
        PPPM_CUDA_TRY(cudaEventCreateWithFlags(&p.start, cudaEventDisableTiming));
        p.ready = true;
    }
    *out = &p;
    return cudaSuccess;
}

std::mutex g_batch_mutex;  // one batch at a time per process: the pool is shared

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
    std::lock_guard<std::mutex> lock(g_batch_mutex);
    StreamPool *pool = nullptr;
    cudaError_t e = pool_for_device(&pool);
    if (e != cudaSuccess) {
        pppm_set_error("pppm_batch_run: stream pool: %s", cudaGetErrorString(e));
        return PPPM_ERR_CUDA;
    }
    cudaStream_t caller = (cudaStream_t)stream;
    e = cudaEventRecord(pool->start, caller);
    const int used = (int)(count < (uint32_t)kPoolStreams ? count : (uint32_t)kPoolStreams);
    for (int q = 0; q < used && e == cudaSuccess; q++) e = cudaStreamWaitEvent(pool->s[q], pool->start, 0);
    if (e != cudaSuccess) {
        pppm_set_error("pppm_batch_run: %s", cudaGetErrorString(e));
        return PPPM_ERR_CUDA;
    }
    pppm_status rc = PPPM_OK;
    uint32_t failed = 0;
    for (uint32_t i = 0; i < count && rc == PPPM_OK; i++) {
        pppm_batch_item &it = items[i];
        pppm_scene *s = it.scene;
        cudaStream_t own = s->stream;
        s->stream = pool->s[i % kPoolStreams];
        rc = pppm_set_vortices(s, it.N, it.pos4_dev, it.ax_dev, it.ay_dev, it.az_dev);
        if (rc == PPPM_OK) rc = pppm_build_far_field(s);
        if (rc == PPPM_OK && it.M)
            rc = pppm_eval(s, it.M, it.eval_a4_dev, it.eval_b4_dev, it.is_segment, it.u_dev, it.v_dev, it.w_dev);
        s->stream = own;
        failed = i;
    }
    // join: the caller's stream waits for every pool stream that was used
    for (int q = 0; q < used; q++) {
        cudaEventRecord(pool->done[q], pool->s[q]);
        cudaStreamWaitEvent(caller, pool->done[q], 0);
    }
    if (rc != PPPM_OK) {
        char buf[256];
        snprintf(buf, sizeof(buf), "%s", pppm_last_error());
        pppm_set_error("pppm_batch_run: item %u: %s", failed, buf);
    }
    return rc;
}
