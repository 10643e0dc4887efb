// Request loop for many resident scenes (no reference counterpart: the
// reference runs one scene per process, HFS/newTest.cpp:38-58).
//
// Scenes are registered with their particles on the host.  A request asks
// for the velocity at a scene's particles (EVAL) or for `steps` RK2 time
// steps of its particles (ADVANCE).  Requests are served by `slots` worker
// threads, each owning a CUDA stream, so requests that arrive while others
// run start as soon as a slot is free and their kernels overlap on the GPU
// (continuous batching).  Before a request runs, its scene must be resident:
// device buffers sized for it, positions and strengths on the device.  A
// scene's footprint is admitted against the HBM budget; when it does not fit,
// the least recently used idle resident scene is evicted (its positions are
// copied back to the host first, so an advanced scene continues from where it
// was).  Requests of one scene run in submission order, one at a time.  Every
// request runs exactly the single-scene kernels, so its result does not depend
// on what else is in flight.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "pppm_internal.cuh"

extern "C" __attribute__((visibility("hidden"))) void pppm_set_error(const char *fmt, ...);

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct SceneRec {
    uint64_t id = 0;
    pppm_params prm{};
    uint32_t N = 0;
    std::vector<float> pos;      // host copy (authoritative while not resident)
    std::vector<double> alpha;   // [3][N]
    // residency
    pppm_scene *scene = nullptr;
    float *dpos = nullptr;
    double *dalpha = nullptr;
    double *dvel = nullptr;      // [3][N]
    uint64_t footprint = 0;
    bool busy = false;           // a request of this scene is running
    double last_use = 0.0;
    std::deque<uint64_t> fifo;   // queued tickets of this scene
};

struct Request {
    uint64_t ticket = 0;
    uint64_t scene = 0;
    int kind = 0;
    uint32_t steps = 0;
    double dt = 0.0;
    pppm_request_info info{};
    std::vector<double> result;  // [3][N] velocities for EVAL
    bool done = false;
};

// Device bytes a scene needs: the scene's own buffers plus the server's
// position / strength / velocity arrays.
uint64_t scene_footprint(uint32_t n, uint32_t N) {
    const uint64_t C = (uint64_t)n * n * n;
    uint64_t levels = 0, d = n;
    while (d * d * d > 512) { levels += d * d * d; d /= 2; }
    levels += d * d * d;
    const uint64_t grid = C * (12 /*vort*/ + 24 /*psi*/ + 12 /*far*/ + 12 /*start,end,flag*/ + 64 /*sub tables*/) +
                          levels * 24 /*mg x,b*/ + 512ull * 512 * 8 /*coarse operator*/;
    const uint64_t part = (uint64_t)N * (16 + 24 + 32 /*sort*/ + 32 /*records*/ + 16 /*rk2*/ + 16 /*ref order*/ +
                                         32 /*eval sort*/ + 32 /*staging*/ + 16 + 24 + 24 /*server arrays*/);
    return grid + part + (4ull << 20);
}

}  // namespace

struct pppm_server {
    pppm_server_config cfg{};
    int device = 0;
    std::mutex mu;
    std::condition_variable cv_work;   // workers wait for runnable requests
    std::condition_variable cv_done;   // waiters wait for completions
    std::map<uint64_t, std::unique_ptr<SceneRec>> scenes;
    std::map<uint64_t, std::unique_ptr<Request>> requests;
    std::deque<uint64_t> queue;        // submission order of pending tickets
    uint64_t next_scene = 1, next_ticket = 1;
    uint64_t resident_bytes = 0;
    bool stopping = false;
    std::vector<std::thread> workers;
    uint64_t completed = 0;
};

namespace {

void release_device(SceneRec &r) {
    std::lock_guard<std::recursive_mutex> lk(pppm::device_lock());
    // the scene's last stream may belong to a worker that has exited
    if (r.scene) pppm_scene_set_stream(r.scene, nullptr);
    if (r.scene) pppm_scene_destroy(r.scene);
    cudaFree(r.dpos);
    cudaFree(r.dalpha);
    cudaFree(r.dvel);
    r.scene = nullptr;
    r.dpos = nullptr;
    r.dalpha = nullptr;
    r.dvel = nullptr;
}

// Makes scene r resident (called without the server lock held).
pppm_status make_resident(SceneRec &r, cudaStream_t st) {
    std::unique_lock<std::recursive_mutex> lk(pppm::device_lock());
    pppm_status rc = pppm_scene_create(&r.prm, r.N, r.N, st, &r.scene);
    if (rc != PPPM_OK) return rc;
    cudaError_t e = ::pppm::device_malloc((void **)&r.dpos, sizeof(float) * 4 * (size_t)r.N);
    if (e == cudaSuccess) e = ::pppm::device_malloc((void **)&r.dalpha, sizeof(double) * 3 * (size_t)r.N);
    if (e == cudaSuccess) e = ::pppm::device_malloc((void **)&r.dvel, sizeof(double) * 3 * (size_t)r.N);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(r.dpos, r.pos.data(), sizeof(float) * 4 * (size_t)r.N, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(r.dalpha, r.alpha.data(), sizeof(double) * 3 * (size_t)r.N, cudaMemcpyHostToDevice, st);
    lk.unlock();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        pppm_set_error("server: making scene %llu resident: %s", (unsigned long long)r.id, cudaGetErrorString(e));
        release_device(r);
        return PPPM_ERR_OOM;
    }
    return PPPM_OK;
}

// Copies an evicted scene's positions back to the host, then frees it.
void evict(SceneRec &r, cudaStream_t st) {
    if (r.dpos) {
        cudaMemcpyAsync(r.pos.data(), r.dpos, sizeof(float) * 4 * (size_t)r.N, cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
    }
    release_device(r);
}

pppm_status run_request(SceneRec &r, Request &q, cudaStream_t st) {
    pppm_scene_set_stream(r.scene, st);
    const uint32_t N = r.N;
    double *ax = r.dalpha, *ay = r.dalpha + N, *az = r.dalpha + 2 * (size_t)N;
    pppm_status rc = PPPM_OK;
    if (q.kind == PPPM_REQ_EVAL) {
        rc = pppm_set_vortices(r.scene, N, r.dpos, ax, ay, az);
        if (rc == PPPM_OK) rc = pppm_build_far_field(r.scene);
        if (rc == PPPM_OK) rc = pppm_eval(r.scene, N, r.dpos, r.dpos, 1, r.dvel, r.dvel + N, r.dvel + 2 * (size_t)N);
        if (rc == PPPM_OK) {
            q.result.resize(3 * (size_t)N);
            cudaError_t e = cudaMemcpyAsync(q.result.data(), r.dvel, sizeof(double) * 3 * (size_t)N,
                                            cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) rc = PPPM_ERR_CUDA;
        }
    } else {
        for (uint32_t k = 0; k < q.steps && rc == PPPM_OK; k++)
            rc = pppm_advect_rk2(r.scene, N, r.dpos, ax, ay, az, q.dt);
        if (rc == PPPM_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = PPPM_ERR_CUDA;
    }
    return rc;
}

void worker_main(pppm_server *S, int slot) {
    cudaSetDevice(S->device);
    cudaStream_t st = nullptr;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        // first pending request whose scene is idle and fits (or can be made to fit)
        Request *pick = nullptr;
        SceneRec *rec = nullptr;
        std::vector<SceneRec *> victims;
        for (auto it = S->queue.begin(); it != S->queue.end(); ++it) {
            Request *q = S->requests[*it].get();
            SceneRec *r = S->scenes[q->scene].get();
            if (r->busy || r->fifo.empty() || r->fifo.front() != q->ticket) continue;
            if (r->scene) { pick = q; rec = r; S->queue.erase(it); break; }
            // needs residency: admit by footprint, evicting idle scenes (LRU)
            uint64_t need = r->footprint;
            uint64_t free_b = S->cfg.hbm_budget_bytes > S->resident_bytes ? S->cfg.hbm_budget_bytes - S->resident_bytes : 0;
            std::vector<SceneRec *> idle;
            for (auto &kv : S->scenes)
                if (kv.second->scene && !kv.second->busy) idle.push_back(kv.second.get());
            std::sort(idle.begin(), idle.end(), [](SceneRec *a, SceneRec *b) { return a->last_use < b->last_use; });
            std::vector<SceneRec *> v;
            for (SceneRec *c : idle) {
                if (free_b >= need) break;
                v.push_back(c);
                free_b += c->footprint;
            }
            if (free_b >= need) { pick = q; rec = r; victims = v; S->queue.erase(it); break; }
        }
        if (!pick) {
            if (S->stopping) break;
            S->cv_work.wait(lk);
            continue;
        }
        rec->busy = true;
        for (SceneRec *v : victims) { v->busy = true; S->resident_bytes -= v->footprint; }
        const bool need_res = rec->scene == nullptr;
        if (need_res) S->resident_bytes += rec->footprint;
        pick->info.start_s = now_s();
        lk.unlock();
        for (SceneRec *v : victims) evict(*v, st);
        pppm_status rc = need_res ? make_resident(*rec, st) : PPPM_OK;
        if (rc == PPPM_OK) rc = run_request(*rec, *pick, st);
        const double end = now_s();
        lk.lock();
        for (SceneRec *v : victims) v->busy = false;
        if (rc != PPPM_OK && need_res && !rec->scene) S->resident_bytes -= rec->footprint;
        rec->busy = false;
        rec->last_use = end;
        rec->fifo.pop_front();
        pick->info.end_s = end;
        pick->info.status = rc;
        pick->done = true;
        S->completed++;
        S->cv_done.notify_all();
        S->cv_work.notify_all();
    }
    lk.unlock();
    cudaStreamDestroy(st);
}

}  // namespace

extern "C" pppm_status pppm_server_create(const pppm_server_config *cfg, pppm_server **out) {
    if (!cfg || !out || cfg->slots == 0 || cfg->slots > 64 || cfg->hbm_budget_bytes == 0) {
        pppm_set_error("pppm_server_create: invalid configuration");
        return PPPM_ERR_INVALID;
    }
    pppm_server *S = new pppm_server();
    S->cfg = *cfg;
    cudaGetDevice(&S->device);
    for (uint32_t i = 0; i < cfg->slots; i++) S->workers.emplace_back(worker_main, S, (int)i);
    *out = S;
    return PPPM_OK;
}

extern "C" pppm_status pppm_server_destroy(pppm_server *S) {
    if (!S) return PPPM_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopping = true;
        S->queue.clear();
    }
    S->cv_work.notify_all();
    for (auto &t : S->workers) t.join();
    for (auto &kv : S->scenes) release_device(*kv.second);
    delete S;
    return PPPM_OK;
}

extern "C" pppm_status pppm_server_add_scene(pppm_server *S, const pppm_params *p, uint32_t N, const float *pos4_host,
                                             const double *ax, const double *ay, const double *az, uint64_t *id) {
    if (!S || !p || !pos4_host || !ax || !ay || !az || !id || N == 0) {
        pppm_set_error("pppm_server_add_scene: invalid argument");
        return PPPM_ERR_INVALID;
    }
    auto r = std::make_unique<SceneRec>();
    r->prm = *p;
    r->N = N;
    r->pos.assign(pos4_host, pos4_host + 4 * (size_t)N);
    r->alpha.resize(3 * (size_t)N);
    std::memcpy(r->alpha.data(), ax, sizeof(double) * N);
    std::memcpy(r->alpha.data() + N, ay, sizeof(double) * N);
    std::memcpy(r->alpha.data() + 2 * (size_t)N, az, sizeof(double) * N);
    r->footprint = scene_footprint(p->n, N);
    if (r->footprint > S->cfg.hbm_budget_bytes) {
        pppm_set_error("pppm_server_add_scene: scene needs %llu bytes, more than the whole HBM budget",
                       (unsigned long long)r->footprint);
        return PPPM_ERR_OOM;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    r->id = S->next_scene++;
    *id = r->id;
    S->scenes[r->id] = std::move(r);
    return PPPM_OK;
}

extern "C" pppm_status pppm_server_submit(pppm_server *S, uint64_t scene, int kind, uint32_t steps, double dt,
                                          uint64_t *ticket) {
    if (!S || !ticket || (kind != PPPM_REQ_EVAL && kind != PPPM_REQ_ADVANCE)) {
        pppm_set_error("pppm_server_submit: invalid argument");
        return PPPM_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->scenes.find(scene);
    if (it == S->scenes.end()) {
        pppm_set_error("pppm_server_submit: unknown scene %llu", (unsigned long long)scene);
        return PPPM_ERR_INVALID;
    }
    auto q = std::make_unique<Request>();
    q->ticket = S->next_ticket++;
    q->scene = scene;
    q->kind = kind;
    q->steps = steps;
    q->dt = dt;
    q->info.submit_s = now_s();
    q->info.status = -1;
    *ticket = q->ticket;
    it->second->fifo.push_back(q->ticket);
    S->queue.push_back(q->ticket);
    S->requests[q->ticket] = std::move(q);
    S->cv_work.notify_one();
    return PPPM_OK;
}

extern "C" pppm_status pppm_server_wait(pppm_server *S, uint64_t ticket, double timeout_s, pppm_request_info *info,
                                        double *vel_host) {
    if (!S) return PPPM_ERR_INVALID;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->requests.find(ticket);
    if (it == S->requests.end()) {
        pppm_set_error("pppm_server_wait: unknown ticket %llu", (unsigned long long)ticket);
        return PPPM_ERR_INVALID;
    }
    Request *q = it->second.get();
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
    while (!q->done) {
        if (S->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && !q->done) {
            pppm_set_error("pppm_server_wait: ticket %llu not done within %.3f s", (unsigned long long)ticket,
                           timeout_s);
            return PPPM_ERR_STATE;
        }
    }
    if (info) *info = q->info;
    if (vel_host && q->kind == PPPM_REQ_EVAL && !q->result.empty())
        std::memcpy(vel_host, q->result.data(), sizeof(double) * q->result.size());
    const pppm_status st = (pppm_status)q->info.status;
    S->requests.erase(it);
    return st;
}

extern "C" pppm_status pppm_server_read_positions(pppm_server *S, uint64_t scene, float *pos4_host) {
    if (!S || !pos4_host) return PPPM_ERR_INVALID;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->scenes.find(scene);
    if (it == S->scenes.end()) return PPPM_ERR_INVALID;
    SceneRec &r = *it->second;
    while (r.busy || !r.fifo.empty()) S->cv_done.wait(lk);
    if (r.dpos) {
        cudaStream_t st = nullptr;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return PPPM_ERR_CUDA;
        cudaError_t e = cudaMemcpyAsync(r.pos.data(), r.dpos, sizeof(float) * 4 * (size_t)r.N,
                                        cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
        if (e != cudaSuccess) return PPPM_ERR_CUDA;
    }
    std::memcpy(pos4_host, r.pos.data(), sizeof(float) * 4 * (size_t)r.N);
    return PPPM_OK;
}

extern "C" pppm_status pppm_server_stats(pppm_server *S, uint64_t *resident_bytes, uint64_t *completed) {
    if (!S) return PPPM_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    if (resident_bytes) *resident_bytes = S->resident_bytes;
    if (completed) *completed = S->completed;
    return PPPM_OK;
}
