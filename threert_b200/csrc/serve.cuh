// The serving loop (include/threert_cuda.h trt_server_*): requests on resident scenes, admitted by free device memory,
// their samples packed into shared waves that the pass's kernels run at once. Included by pathtrace.cu, whose kernels,
// wave state and scene type it uses.
//
// The reference serves one job at a time (renderer/src/main.rs:345-397: read a JSON line, Gpu::render, write the
// image). Here a worker thread keeps the GPU busy across requests: each step is one wave through every bounce, holding
// the next samples of every active request that fit; a request that arrives while a step runs joins the next one.
// Step N+1 is queued before step N's finished requests are read back (on a copy stream), so the read-back and the
// host's bookkeeping overlap the next step's kernels.
#pragma once
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <thread>

namespace trt {

struct ServeRequest {
    uint64_t id = 0;
    trt_scene* scene = nullptr;
    Params P{};
    uint32_t spp = 0, issued = 0, n_idx = 0, w = 0, h = 0, steps = 0;
    float* host = nullptr;     // the accum's host buffer, or null
    float* rgb = nullptr;      // the denoised image's host buffer, or null
    float4* accum = nullptr;
    uint64_t accum_bytes = 0;
    double t_submit = 0, t_start = -1;
    int status = TRT_OK;
    cudaEvent_t copied = nullptr;  // its read-back's completion
};

// One step on the GPU: its events, the requests it finishes, its counts.
struct ServeStep {
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    std::vector<ServeRequest*> finishing;
    uint64_t paths = 0;
};

}  // namespace trt

struct trt_server {
    trt_ctx* ctx = nullptr;
    trt_server_options opt{};
    cudaStream_t stream = nullptr, copy = nullptr;
    // each depth's shadow walk on `aux` beside the next depth's closest-hit walk (forked and joined by events, inside
    // the step's graph)
    cudaStream_t aux = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    Wave wave;
    unsigned long long* totals = nullptr;
    // The step's table on the device: a StepHead, then at TABLE_JOBS the jobs; pinned staging copies alternate.
    uint8_t* table = nullptr;
    uint8_t* staging[2] = {nullptr, nullptr};
    std::map<std::pair<uint32_t, uint32_t>, cudaGraphExec_t> graphs;  // by (deepest depth, launch size)
    cudaEvent_t staged[2] = {nullptr, nullptr};
    uint32_t parity = 0;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;
    std::deque<trt::ServeRequest*> pending;
    std::multimap<double, trt::ServeRequest*> scheduled;  // requests that arrive later (trt_server_submit_at), by time
    std::vector<trt::ServeRequest*> active;
    std::vector<trt_request_done> done;
    std::vector<trt::ServeRequest*> copying;  // read-backs queued on the copy stream, not yet seen complete
    std::vector<cudaEvent_t> ev_free;
    std::multimap<uint64_t, float4*> pool;  // accum buffers by size, free for reuse
    uint64_t next_id = 1;
    std::chrono::steady_clock::time_point t0;
    trt_server_stats stats{};
    std::string err;
    int g_ext = 0, g_sha = 0;
};

namespace {

constexpr uint64_t TABLE_JOBS = 256;  // the jobs' offset in the step table
constexpr uint64_t TABLE_BYTES = TABLE_JOBS + sizeof(Job) * MAX_JOBS;

double serve_now(const trt_server* s) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - s->t0).count();
}

float4* serve_take_accum(trt_server* s, uint64_t bytes) {
    auto it = s->pool.find(bytes);
    if (it != s->pool.end()) {
        float4* p = it->second;
        s->pool.erase(it);
        return p;
    }
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess || free_b < bytes + s->opt.hbm_reserve) return nullptr;
    float4* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    return p;
}

// Moves waiting requests into the active set while there is room (with the lock held); scheduled requests whose
// time has come join the waiting ones first, in arrival order.
void serve_admit(trt_server* s) {
    if (!s->scheduled.empty()) {
        const double now = serve_now(s);
        while (!s->scheduled.empty() && s->scheduled.begin()->first <= now) {
            s->pending.push_back(s->scheduled.begin()->second);
            s->scheduled.erase(s->scheduled.begin());
        }
    }
    while (!s->pending.empty() && s->active.size() < s->opt.max_active) {
        ServeRequest* r = s->pending.front();
        float4* a = serve_take_accum(s, r->accum_bytes);
        if (!a) break;  // no room on the device yet: it waits, and those behind it too (first come, first served)
        r->accum = a;
        cudaMemsetAsync(a, 0, r->accum_bytes, s->stream);
        s->pending.pop_front();
        s->active.push_back(r);
    }
}

void serve_finish(trt_server* s, ServeRequest* r, int status) {
    trt_request_done d{};
    d.id = r->id;
    d.status = status;
    d.steps = r->steps;
    d.submit_ms = r->t_submit;
    d.start_ms = r->t_start;
    d.done_ms = serve_now(s);
    if (r->accum) s->pool.emplace(r->accum_bytes, r->accum);
    s->done.push_back(d);
    s->stats.requests_done++;
    delete r;
}

// A step's launches, all sized by `size` (the kernels stop at the counts on the device), reading the step table.
void serve_enqueue(trt_server* s, uint32_t last, uint32_t size, cudaStream_t st) {
    Wave& W = s->wave;
    const StepHead* head = reinterpret_cast<const StepHead*>(s->table);
    const Job* tj = reinterpret_cast<const Job*>(s->table + TABLE_JOBS);
    const int blk = 128;
    const Job none{};
    uint32_t grid = (size + blk - 1) / blk;
    cudaMemsetAsync(W.Q.cnt, 0, 4ull * (MAX_DEPTH * CNT_STRIDE + CNT_STRIDE), st);
    k_raygen<<<grid, blk, 0, st>>>(tj, 0u, W.B, W.Q, size, head);
    bool sort_hits = (s->opt.flags & TRT_RENDER_UNSORTED_HITS) == 0;
    // Each depth's shadow walk runs on the second stream beside the next depth's closest-hit walk, as trt_render
    // runs them: both read what the depth's shading wrote and write apart (visibility bits; hit records), and the
    // depth's resolve waits for the shadow walk (the join) before the next depth's hit sort rewrites its order.
    k_extend<false, false, true><<<s->g_ext, blk, 0, st>>>(tj, none, W.B, W.Q, 0u, W.Q.q[0]);
    for (uint32_t depth = 0; depth <= last; ++depth) {
        uint32_t* raw = W.Q.q[depth & 1u];
        uint32_t* next = W.Q.q[(depth + 1u) & 1u];
        uint32_t* shade_q = raw;
        if (sort_hits) {
            shade_q = W.Q.qx;
            k_sort_count<SORT_HITS><<<(size + SORT_ITEMS - 1u) / SORT_ITEMS, SORT_THREADS, 0, st>>>(tj, W.B, W.Q, raw,
                                                                                                  depth, 0u);
            k_sort_scatter<SORT_HITS><<<(size + 255u) / 256u, 256, 0, st>>>(W.Q, raw, shade_q, depth);
        }
        k_shade<true><<<grid, blk, 0, st>>>(tj, none, W.B, W.Q, depth, shade_q, next);
        cudaEventRecord(s->fork_ev, st);
        cudaStreamWaitEvent(s->aux, s->fork_ev, 0);
        k_shadow<false, false, true><<<s->g_sha, blk, 0, s->aux>>>(tj, none, W.B, W.Q, depth, nullptr);
        if (depth < last) k_extend<false, false, true><<<s->g_ext, blk, 0, st>>>(tj, none, W.B, W.Q, depth + 1u, next);
        cudaEventRecord(s->join_ev, s->aux);
        cudaStreamWaitEvent(st, s->join_ev, 0);
        k_resolve<true><<<grid, blk, 0, st>>>(tj, none, W.B, W.Q, depth, shade_q);
    }
    k_accumulate_flat<<<grid, blk, 0, st>>>(tj, head, W.B, size);
    k_tally<<<1, 32, 0, st>>>(W.Q, last + 1, 0u, head);
}

// Plans and queues one step from the active requests; false when none has samples left to issue.
bool serve_step(trt_server* s, ServeStep& step) {
    std::vector<Job> jobs;
    std::vector<ServeRequest*> owners;
    uint32_t slot = 0, last = 0, n_idx_max = 0;
    const uint32_t cap = s->wave.slots;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        serve_admit(s);
        for (ServeRequest* r : s->active) {
            if (r->issued >= r->spp) continue;
            if (jobs.size() == MAX_JOBS) break;
            uint32_t k = std::min(r->spp - r->issued, (cap - slot) / r->n_idx);
            if (k == 0) continue;  // not enough slots left in this step: a smaller request may still fit
            Job j{r->P, Walk{scene_view(r->scene), WideView{}, r->P.w[P_MOTION + 2], r->P.w[P_MOTION + 3]}, r->accum,
                  slot, r->n_idx, k, r->issued};
            j.depth = r->rgb ? 1u : 0u;  // the denoiser's depth guide
            jobs.push_back(j);
            owners.push_back(r);
            if (r->t_start < 0) r->t_start = serve_now(s);
            r->issued += k;
            r->steps++;
            slot += r->n_idx * k;
            last = std::max(last, r->P.w[P_COUNTS + 2]);
            n_idx_max = std::max(n_idx_max, r->n_idx);
            step.paths += (uint64_t)r->w * r->h * k;
            if (r->issued == r->spp) step.finishing.push_back(r);
        }
    }
    if (jobs.empty()) return false;
    cudaStream_t st = s->stream;
    // The step's table through a pinned staging buffer (the one two steps back is free once its copy has run).
    uint8_t* stage = s->staging[s->parity];
    cudaEventSynchronize(s->staged[s->parity]);
    StepHead head{(uint32_t)jobs.size(), (uint32_t)std::min<uint64_t>(step.paths, 0xffffffffu), 0u, 0u};
    uint32_t idx_first = 0;
    for (Job& j : jobs) {
        j.idx_first = idx_first;
        idx_first += j.n_idx;
    }
    std::memcpy(stage, &head, sizeof(head));
    std::memcpy(stage + TABLE_JOBS, jobs.data(), sizeof(Job) * jobs.size());
    cudaEventRecord(step.t0, st);
    cudaMemcpyAsync(s->table, stage, TABLE_JOBS + sizeof(Job) * jobs.size(), cudaMemcpyHostToDevice, st);
    cudaEventRecord(s->staged[s->parity], st);
    s->parity ^= 1u;
    // Launch sizes by the power of two at or above the slots used (at least 2^16, at most the wave): the kernels
    // read the true counts from the device, so one graph serves every step of that size class and depth.
    uint32_t size = 1u << 16;
    while (size < slot && size < s->wave.slots) size <<= 1;
    size = std::min(size, s->wave.slots);
    if (s->opt.launch_mode == 0) {
        auto key = std::make_pair(last, size);
        auto it = s->graphs.find(key);
        if (it == s->graphs.end()) {
            cudaGraph_t g = nullptr;
            cudaGraphExec_t exec = nullptr;
            cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                serve_enqueue(s, last, size, st);
                e = cudaStreamEndCapture(st, &g);
            }
            if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, g, 0);
            if (g) cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                // (Then the server launches directly from here on.)
                std::lock_guard<std::mutex> lk(s->mu);
                s->err = std::string("graph capture: ") + cudaGetErrorString(e);
                s->opt.launch_mode = 1;
                cudaGetLastError();
            } else {
                it = s->graphs.emplace(key, exec).first;
            }
        }
        if (s->opt.launch_mode == 0) cudaGraphLaunch(it->second, st);
    }
    if (s->opt.launch_mode != 0) serve_enqueue(s, last, size, st);
    cudaEventRecord(step.t1, st);
    return true;
}

// Waits for a queued step and queues the read-back of the requests it finished on the copy stream (into pinned host
// memory it runs at full speed and does not hold the worker; into pageable memory the copy call itself waits).
void serve_retire(trt_server* s, ServeStep& step) {
    cudaEventSynchronize(step.t1);
    float ms = 0;
    cudaEventElapsedTime(&ms, step.t0, step.t1);
    for (ServeRequest* r : step.finishing) {
        cudaEvent_t ev = nullptr;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (!s->ev_free.empty()) { ev = s->ev_free.back(); s->ev_free.pop_back(); }
        }
        if (!ev) cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        cudaError_t e = cudaStreamWaitEvent(s->copy, step.t1, 0);
        if (e == cudaSuccess && r->rgb) {
            // the learned denoiser on the copy stream, beside the next step's kernels
            const float* rgb = unet_denoise_on_stream(s->opt.denoiser, r->accum, r->w, r->h, s->copy);
            if (!rgb) r->status = TRT_ECUDA;
            else e = cudaMemcpyAsync(r->rgb, rgb, 12ull * r->w * r->h, cudaMemcpyDeviceToHost, s->copy);
        }
        if (e == cudaSuccess && r->host)
            e = cudaMemcpyAsync(r->host, r->accum, r->accum_bytes, cudaMemcpyDeviceToHost, s->copy);
        if (e == cudaSuccess) e = cudaEventRecord(ev, s->copy);
        r->copied = ev;
        if (e != cudaSuccess) r->status = TRT_ECUDA;
        std::lock_guard<std::mutex> lk(s->mu);
        s->copying.push_back(r);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->stats.steps++;
    s->stats.paths += step.paths;
    s->stats.busy_ms += ms;
    step.finishing.clear();
    step.paths = 0;
}

// Reports the requests whose read-back has completed (waiting for them all when `all`).
void serve_reap(trt_server* s, bool all) {
    std::vector<ServeRequest*> ready;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (ServeRequest* r : s->copying) {
            cudaError_t q = all ? cudaEventSynchronize(r->copied) : cudaEventQuery(r->copied);
            if (q == cudaErrorNotReady) continue;
            if (q != cudaSuccess) r->status = TRT_ECUDA;
            ready.push_back(r);
        }
        if (ready.empty()) return;
        for (ServeRequest* r : ready) {
            s->copying.erase(std::remove(s->copying.begin(), s->copying.end(), r), s->copying.end());
            s->active.erase(std::remove(s->active.begin(), s->active.end(), r), s->active.end());
            s->ev_free.push_back(r->copied);
            serve_finish(s, r, r->status);
        }
    }
    s->cv_done.notify_all();
}

void serve_loop(trt_server* s) {
    cudaSetDevice(s->ctx->device);
    ServeStep steps[2];
    for (auto& st : steps) {
        cudaEventCreate(&st.t0);
        cudaEventCreate(&st.t1);
    }
    int cur = 0;
    bool in_flight = false;  // steps[cur ^ 1] is queued and not yet retired
    for (;;) {
        bool queued = serve_step(s, steps[cur]);
        if (in_flight) serve_retire(s, steps[cur ^ 1]);
        serve_reap(s, false);
        in_flight = queued;
        if (queued) {
            cur ^= 1;
            continue;
        }
        // Nothing to queue: finish the read-backs, then wait for work (or the stop).
        serve_reap(s, true);
        std::unique_lock<std::mutex> lk(s->mu);
        bool have = false;
        for (ServeRequest* r : s->active) have |= r->issued < r->spp;
        if (have) continue;
        if (s->stop && s->active.empty() && s->pending.empty() && s->scheduled.empty()) break;
        // (A request that waits for device memory is retried when a request finishes or 1 ms passes; the wait ends
        // early at the next scheduled arrival.)
        double wait_ms = 1.0;
        if (!s->scheduled.empty()) wait_ms = std::min(wait_ms, s->scheduled.begin()->first - serve_now(s));
        if (wait_ms > 0.0) s->cv_work.wait_for(lk, std::chrono::microseconds((int64_t)(wait_ms * 1000.0) + 1));
    }
    for (auto& st : steps) {
        cudaEventDestroy(st.t0);
        cudaEventDestroy(st.t1);
    }
}

}  // namespace

extern "C" {

int trt_server_create(trt_ctx* c, const trt_server_options* opts, trt_server** out) {
    if (!c || !out) return TRT_EINVAL;
    *out = nullptr;
    cudaSetDevice(c->device);
    auto* s = new trt_server();
    s->ctx = c;
    s->opt = opts ? *opts : trt_server_options{};
    if (s->opt.wave_slots == 0) s->opt.wave_slots = 2u << 20;
    if (s->opt.max_active == 0 || s->opt.max_active > MAX_JOBS) s->opt.max_active = MAX_JOBS;
    if (s->opt.hbm_reserve == 0) s->opt.hbm_reserve = 1ull << 30;
    s->opt.wave_slots = (s->opt.wave_slots + 31u) / 32u * 32u;
    auto fail_s = [&](cudaError_t e, const char* what) {
        c->err = std::string("trt_server_create: ") + what + ": " + cudaGetErrorString(e);
        if (s->stream) cudaStreamDestroy(s->stream);
        if (s->copy) cudaStreamDestroy(s->copy);
        if (s->aux) cudaStreamDestroy(s->aux);
        if (s->fork_ev) cudaEventDestroy(s->fork_ev);
        if (s->join_ev) cudaEventDestroy(s->join_ev);
        delete s;
        return TRT_ECUDA;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->aux, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->fork_ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->join_ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc(&s->totals, sizeof(unsigned long long) * T_COUNT);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->totals, 0, sizeof(unsigned long long) * T_COUNT, s->stream);
    if (e == cudaSuccess) e = cudaMalloc(&s->table, TABLE_BYTES);
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
        e = cudaMallocHost(&s->staging[k], TABLE_BYTES);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->staged[k], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(s->staged[k], s->stream);
    }
    if (e != cudaSuccess) return fail_s(e, "streams and buffers");
    std::string werr;
    if (wave_ensure(s->wave, s->opt.wave_slots, MAX_DIR_LIGHTS, s->totals, s->stream, werr) != TRT_OK) {
        c->err = "trt_server_create: " + werr;
        if (s->stream) cudaStreamDestroy(s->stream);
        if (s->copy) cudaStreamDestroy(s->copy);
        if (s->aux) cudaStreamDestroy(s->aux);
        if (s->fork_ev) cudaEventDestroy(s->fork_ev);
        if (s->join_ev) cudaEventDestroy(s->join_ev);
        delete s;
        return TRT_ECUDA;
    }
    s->g_ext = grid_for((const void*)k_extend<false, false, true>, 128, c->sm_count);
    s->g_sha = grid_for((const void*)k_shadow<false, false, true>, 128, c->sm_count);
    e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return fail_s(e, "set-up");
    s->t0 = std::chrono::steady_clock::now();
    s->worker = std::thread(serve_loop, s);
    *out = s;
    return TRT_OK;
}

void trt_server_destroy(trt_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        while (!s->pending.empty()) {
            ServeRequest* r = s->pending.front();
            s->pending.pop_front();
            serve_finish(s, r, TRT_EINVAL);
        }
        for (auto& pr : s->scheduled) serve_finish(s, pr.second, TRT_EINVAL);
        s->scheduled.clear();
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->stream);
    for (auto& pr : s->pool) cudaFree(pr.second);
    for (cudaEvent_t e : s->ev_free) cudaEventDestroy(e);
    if (s->wave.work) cudaFree(s->wave.work);
    if (s->totals) cudaFree(s->totals);
    if (s->table) cudaFree(s->table);
    for (auto& g : s->graphs) cudaGraphExecDestroy(g.second);
    for (int k = 0; k < 2; ++k) {
        if (s->staging[k]) cudaFreeHost(s->staging[k]);
        if (s->staged[k]) cudaEventDestroy(s->staged[k]);
    }
    cudaStreamDestroy(s->stream);
    cudaStreamDestroy(s->copy);
    cudaStreamDestroy(s->aux);
    cudaEventDestroy(s->fork_ev);
    cudaEventDestroy(s->join_ev);
    delete s;
}

int trt_server_submit(trt_server* s, trt_scene* scene, const uint32_t params[TRT_PARAMS_WORDS], uint32_t spp,
                      float* accum_host, uint64_t* id) {
    if (!accum_host) return TRT_EINVAL;
    return trt_server_submit_rgb(s, scene, params, spp, accum_host, nullptr, id);
}

int trt_server_submit_rgb(trt_server* s, trt_scene* scene, const uint32_t params[TRT_PARAMS_WORDS], uint32_t spp,
                          float* accum_host, float* rgb_host, uint64_t* id) {
    return trt_server_submit_at(s, scene, params, spp, accum_host, rgb_host, -1.0, id);
}

int trt_server_clock(trt_server* s, double* now_ms) {
    if (!s || !now_ms) return TRT_EINVAL;
    *now_ms = serve_now(s);
    return TRT_OK;
}

int trt_server_submit_at(trt_server* s, trt_scene* scene, const uint32_t params[TRT_PARAMS_WORDS], uint32_t spp,
                         float* accum_host, float* rgb_host, double at_ms, uint64_t* id) {
    if (!s || !scene || !params || (!accum_host && !rgb_host) || spp == 0 || at_ms != at_ms) return TRT_EINVAL;
    if (rgb_host) {
        uint32_t w = params[P_SIZE], h = params[P_SIZE + 1];
        uint32_t most = s->opt.denoise_max_spp ? s->opt.denoise_max_spp : 4u;
        if (!s->opt.denoiser) return fail(s->ctx, TRT_EINVAL, "trt_server_submit_rgb: the server has no denoiser");
        if (spp > most)
            return fail(s->ctx, TRT_EINVAL, "trt_server_submit_rgb: more samples than the server denoises");
        if (!unet_fits(s->opt.denoiser, w, h))
            return fail(s->ctx, TRT_EINVAL, "trt_server_submit_rgb: the denoiser does not take a " + std::to_string(w) +
                                                " x " + std::to_string(h) + " image");
    }
    if (scene->ctx->device != s->ctx->device) return fail(s->ctx, TRT_EINVAL, "trt_server_submit: the scene is on another device");
    int rc = check_params(scene, params);
    if (rc) return rc;
    auto* r = new ServeRequest();
    std::memcpy(r->P.w, params, sizeof(r->P.w));
    r->scene = scene;
    r->spp = spp;
    r->w = r->P.w[P_SIZE];
    r->h = r->P.w[P_SIZE + 1];
    r->n_idx = ((r->w + 7u) / 8u) * ((r->h + 3u) / 4u) * 32u;
    if (r->n_idx > s->wave.slots) {
        delete r;
        return fail(s->ctx, TRT_EINVAL, "trt_server_submit: the image needs " + std::to_string(r->n_idx) +
                                            " path slots, more than a step holds (" + std::to_string(s->wave.slots) + ")");
    }
    r->host = accum_host;
    r->rgb = rgb_host;
    r->accum_bytes = 80ull * r->w * r->h;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->id = s->next_id++;
        const double now = serve_now(s);
        if (at_ms > now) {
            r->t_submit = at_ms;
            s->scheduled.emplace(at_ms, r);
        } else {
            r->t_submit = at_ms >= 0.0 ? at_ms : now;
            s->pending.push_back(r);
        }
        if (id) *id = r->id;
    }
    s->cv_work.notify_all();
    return TRT_OK;
}

int trt_server_poll(trt_server* s, trt_request_done* out, uint32_t cap, uint32_t* n, uint32_t wait_ms) {
    if (!s || !n || (cap && !out)) return TRT_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->done.empty() && wait_ms)
        s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s->done.empty(); });
    uint32_t k = (uint32_t)std::min<size_t>(cap, s->done.size());
    for (uint32_t i = 0; i < k; ++i) out[i] = s->done[i];
    s->done.erase(s->done.begin(), s->done.begin() + k);
    *n = k;
    return TRT_OK;
}

int trt_server_stats_get(trt_server* s, trt_server_stats* out) {
    if (!s || !out) return TRT_EINVAL;
    unsigned long long t[T_COUNT];
    // (The totals are read on the copy stream: it does not wait for queued steps.)
    cudaError_t e = cudaMemcpyAsync(t, s->totals, sizeof(t), cudaMemcpyDeviceToHost, s->copy);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->copy);
    if (e != cudaSuccess) return cuda_fail(s->ctx, e, "trt_server_stats_get");
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->stats;
    out->closest_rays = t[T_CLOSEST];
    out->shadow_rays = t[T_SHADOW];
    out->active = (uint32_t)s->active.size();
    out->pending = (uint32_t)(s->pending.size() + s->scheduled.size());
    return TRT_OK;
}

}  // extern "C"
