// rzk_server.cu - a request loop for many users against device-resident scenes.
//
// Callers submit gather or guided-render requests (rzk_server_submit) from any thread.  A
// request is admitted only if the device memory it will hold while in flight (its receivers
// and, for a gather, its per-chunk partial sums) fits the server's HBM budget next to the
// requests already admitted; otherwise the call returns RZK_ERR_BUSY at once and the caller
// decides whether to retry.  One worker thread owns a context and a stream: each iteration
// takes the queue, traces every request's primary hits, runs all of the iteration's gathers
// as ONE persistent batched launch (continuous batching: requests that arrive while a launch
// runs join the next one), launches guided renders one by one, and marks each request done
// from a stream host function when its last kernel has finished.  With batching off the
// worker takes one request at a time and runs it with its own launches (the plain
// per-request baseline).  Scratch comes from the stream-ordered allocator, so an iteration
// neither blocks on an allocation nor synchronises the device.
#include "rzk_internal.cuh"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

enum { kQueued = 0, kRunning = 1, kDone = 2, kCancelled = 3, kFailed = 4 };

struct Req {
    uint64_t id = 0;
    rzk_request r{};
    size_t bytes = 0;
    int state = kQueued;
    rzk_status status = RZK_OK;
    double t_submit = 0.0, t_done = 0.0;
    rzk_receiver *d_recv = nullptr;
    struct rzk_server *srv = nullptr;
};

int default_chunks(int n_vpl) {   // rzk_gather's automatic chunk count
    const int max_chunks = std::max(1, (n_vpl + 127) / 128);
    return std::min(32, max_chunks);
}

}  // namespace

struct rzk_server {
    int device = 0;
    rzk_context *ctx = nullptr;
    cudaStream_t st = nullptr;
    rzk_server_params prm{};
    int64_t budget = 0, held = 0;
    int64_t n_submitted = 0, n_rejected = 0, n_completed = 0, n_launches = 0;
    uint64_t next_id = 1;
    bool stop = false;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req *> queue;
    std::unordered_map<uint64_t, Req *> reqs;
    std::thread worker;
};

namespace {

void CUDART_CB on_done(void *p) {
    Req *q = (Req *)p;
    rzk_server *s = q->srv;
    std::lock_guard<std::mutex> lk(s->mu);
    q->t_done = now_ms();
    q->state = q->status == RZK_OK ? kDone : kFailed;
    s->held -= (int64_t)q->bytes;
    s->n_completed++;
    s->cv_done.notify_all();
}

void fail_now(rzk_server *s, Req *q, rzk_status st) {
    std::lock_guard<std::mutex> lk(s->mu);
    q->status = st;
    q->t_done = now_ms();
    q->state = kFailed;
    s->held -= (int64_t)q->bytes;
    s->n_completed++;
    s->cv_done.notify_all();
}

// the receivers of every request of the iteration, then its gathers (batched or one by
// one) and its guided renders; each request's completion is a host function on the stream
void run_iteration(rzk_server *s, std::vector<Req *> &batch) {
    cudaStream_t st = s->st;
    std::vector<Req *> live;
    for (Req *q : batch) {
        const size_t n = (size_t)q->r.camera.width * q->r.camera.height;
        cudaError_t e = cudaMallocAsync((void **)&q->d_recv, sizeof(rzk_receiver) * n, st);
        if (e != cudaSuccess) { fail_now(s, q, RZK_ERR_NOMEM); continue; }
        rzk_status r = rzk_primary(q->r.scene, &q->r.camera, q->d_recv, st);
        if (r != RZK_OK) { cudaFreeAsync(q->d_recv, st); fail_now(s, q, r); continue; }
        live.push_back(q);
    }
    std::vector<Req *> gathers, guided;
    for (Req *q : live) (q->r.kind == RZK_REQ_GATHER ? gathers : guided).push_back(q);
    int64_t launches = 0;
    if (!gathers.empty() && s->prm.batching) {
        std::vector<rzk_gather_job> jobs(gathers.size());
        for (size_t i = 0; i < gathers.size(); ++i) {
            const rzk_request &r = gathers[i]->r;
            jobs[i] = rzk_gather_job{r.scene, gathers[i]->d_recv, r.camera.width * r.camera.height, r.camera.width,
                                     r.d_vpls, r.n_vpl, r.clamp_mode, r.tau, r.scale, r.d_rgb};
        }
        rzk::BatchPlan *plan = nullptr;
        rzk_status r = rzk::batch_plan_create(jobs.data(), (int)jobs.size(), 0, &plan);
        float *partial = nullptr;
        int *work = nullptr;
        if (r == RZK_OK) {
            const size_t pf = rzk::batch_plan_partial_floats(plan);
            if (cudaMallocAsync((void **)&partial, sizeof(float) * std::max<size_t>(pf, 1), st) != cudaSuccess ||
                cudaMallocAsync((void **)&work, sizeof(int) * rzk::batch_plan_tables(plan), st) != cudaSuccess)
                r = RZK_ERR_NOMEM;
        }
        if (r == RZK_OK) r = rzk::batch_plan_launch(plan, partial, work, 0, 0, st);
        if (r == RZK_OK) launches += 1 + 2 * rzk::batch_plan_tables(plan);
        if (partial) cudaFreeAsync(partial, st);
        if (work) cudaFreeAsync(work, st);
        if (plan) rzk::batch_plan_destroy(plan);
        for (Req *q : gathers) {
            q->status = r;
            cudaFreeAsync(q->d_recv, st);
            cudaLaunchHostFunc(st, on_done, q);
        }
    } else {
        for (Req *q : gathers) {
            const rzk_request &r = q->r;
            q->status = rzk_gather_cfg(s->ctx, r.scene, q->d_recv, r.camera.width * r.camera.height, r.camera.width,
                                       r.d_vpls, r.n_vpl, r.clamp_mode, r.tau, r.scale, r.d_rgb, 0, 0, st);
            launches += 3;
            cudaFreeAsync(q->d_recv, st);
            cudaLaunchHostFunc(st, on_done, q);
        }
    }
    for (Req *q : guided) {
        const rzk_request &r = q->r;
        rzk_guided_params g{r.spp, r.max_bounce, r.rr_depth, r.rr_prob, 1, r.seed};
        q->status = rzk_guided_render(s->ctx, r.scene, r.lightslice, &r.camera, &g, r.d_rgb, nullptr, st);
        launches += 1;
        cudaFreeAsync(q->d_recv, st);
        cudaLaunchHostFunc(st, on_done, q);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->n_launches += launches + (int64_t)live.size();
}

void worker_main(rzk_server *s) {
    cudaSetDevice(s->device);
    const int max_batch = s->prm.max_batch > 0 ? s->prm.max_batch : 256;
    while (true) {
        std::vector<Req *> batch;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty(); });
            if (s->queue.empty()) break;   // stopping and drained
            const size_t take = s->prm.batching ? std::min<size_t>(s->queue.size(), (size_t)max_batch) : 1;
            for (size_t i = 0; i < take; ++i) {
                Req *q = s->queue.front();
                s->queue.pop_front();
                q->state = kRunning;
                batch.push_back(q);
            }
        }
        run_iteration(s, batch);
    }
    cudaStreamSynchronize(s->st);
}

}  // namespace

extern "C" {

rzk_status rzk_server_create(int device, const rzk_server_params *params, rzk_server **out) {
    if (!params || !out || params->batching < 0 || params->max_batch < 0 || params->hbm_budget_bytes < 0)
        return RZK_ERR_INVALID;
    *out = nullptr;
    rzk_server *s = new rzk_server();
    s->device = device;
    s->prm = *params;
    rzk_status r = rzk_context_create(device, &s->ctx);
    if (r != RZK_OK) {
        delete s;
        return r;
    }
    if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) {
        rzk_context_destroy(s->ctx);
        delete s;
        return RZK_ERR_CUDA;
    }
    s->budget = params->hbm_budget_bytes;
    if (s->budget == 0) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        s->budget = (int64_t)(0.9 * (double)fr);
    }
    s->worker = std::thread(worker_main, s);
    *out = s;
    return RZK_OK;
}

rzk_status rzk_server_destroy(rzk_server *s) {
    if (!s) return RZK_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaStreamSynchronize(s->st);
    for (auto &kv : s->reqs) delete kv.second;
    cudaStreamDestroy(s->st);
    rzk_context_destroy(s->ctx);
    delete s;
    return RZK_OK;
}

rzk_status rzk_server_submit(rzk_server *s, const rzk_request *req, uint64_t *ticket) {
    if (!s || !req || !ticket) return RZK_ERR_INVALID;
    const rzk_request &r = *req;
    const int64_t n = (int64_t)r.camera.width * r.camera.height;
    if (!r.scene || r.camera.width <= 0 || r.camera.height <= 0 || n > (1LL << 30) || !r.d_rgb) return RZK_ERR_INVALID;
    size_t bytes = sizeof(rzk_receiver) * (size_t)n;
    if (r.kind == RZK_REQ_GATHER) {
        if (r.n_vpl < 0 || (r.n_vpl > 0 && !r.d_vpls) || ((uintptr_t)r.d_vpls & 15u) ||
            r.clamp_mode < RZK_CLAMP_NONE || r.clamp_mode > RZK_CLAMP_RADIANCE)
            return RZK_ERR_INVALID;
        bytes += sizeof(float) * 3 * (size_t)n * (size_t)default_chunks(r.n_vpl);
    } else if (r.kind == RZK_REQ_GUIDED) {
        if (!r.lightslice || r.spp <= 0 || r.max_bounce < 1 || r.max_bounce > 16 || r.rr_depth < 0 ||
            (r.rr_depth > 0 && !(r.rr_prob > 0.0f && r.rr_prob <= 1.0f)))
            return RZK_ERR_INVALID;
    } else {
        return RZK_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return RZK_ERR_INVALID;
    s->n_submitted++;
    if (s->held + (int64_t)bytes > s->budget) {
        s->n_rejected++;
        return RZK_ERR_BUSY;
    }
    Req *q = new Req();
    q->id = s->next_id++;
    q->r = r;
    q->bytes = bytes;
    q->srv = s;
    q->t_submit = now_ms();
    s->held += (int64_t)bytes;
    s->reqs[q->id] = q;
    s->queue.push_back(q);
    *ticket = q->id;
    s->cv_work.notify_one();
    return RZK_OK;
}

rzk_status rzk_server_poll(rzk_server *s, uint64_t ticket, int32_t *state, double *latency_ms) {
    if (!s || !state) return RZK_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) {
        *state = -1;
        return RZK_ERR_INVALID;
    }
    Req *q = it->second;
    *state = q->state;
    rzk_status st = RZK_OK;
    if (q->state >= kDone) {
        if (latency_ms) *latency_ms = q->t_done - q->t_submit;
        st = q->status;
        s->reqs.erase(it);   // a finished request is reported once
        delete q;
    }
    return st;
}

rzk_status rzk_server_wait(rzk_server *s, uint64_t ticket, int32_t timeout_ms, double *latency_ms) {
    if (!s) return RZK_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return RZK_ERR_INVALID;
    Req *q = it->second;
    auto finished = [&] { return q->state >= kDone; };
    if (timeout_ms < 0) s->cv_done.wait(lk, finished);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), finished)) return RZK_ERR_TIMEOUT;
    if (latency_ms) *latency_ms = q->t_done - q->t_submit;
    rzk_status st = q->status;
    s->reqs.erase(ticket);
    delete q;
    return st;
}

rzk_status rzk_server_cancel(rzk_server *s, uint64_t ticket) {
    if (!s) return RZK_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return RZK_ERR_INVALID;
    Req *q = it->second;
    if (q->state != kQueued) return RZK_ERR_BUSY;
    s->queue.erase(std::find(s->queue.begin(), s->queue.end(), q));
    q->state = kCancelled;
    q->status = RZK_OK;
    q->t_done = now_ms();
    s->held -= (int64_t)q->bytes;
    s->cv_done.notify_all();
    return RZK_OK;
}

rzk_status rzk_server_stats(rzk_server *s, int64_t *submitted, int64_t *rejected, int64_t *completed,
                            int64_t *launches, int64_t *held_bytes, int64_t *budget_bytes) {
    if (!s) return RZK_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    if (submitted) *submitted = s->n_submitted;
    if (rejected) *rejected = s->n_rejected;
    if (completed) *completed = s->n_completed;
    if (launches) *launches = s->n_launches;
    if (held_bytes) *held_bytes = s->held;
    if (budget_bytes) *budget_bytes = s->budget;
    return RZK_OK;
}

}  // extern "C"
