// rzk_server.cu - a request loop for many users against device-resident scenes.
//
// Callers submit gather or guided-render requests (rzk_server_submit) from any thread.  A
// request is admitted only if the device memory it will hold while in flight (its receivers
// and, for a gather, its per-chunk partial sums) fits the server's HBM budget next to the
// requests already admitted; otherwise the call returns RZK_ERR_BUSY at once and the caller
// decides whether to retry.  One worker thread owns a context and a stream and keeps at
// most two launch groups on it (one running, one queued behind it, so the GPU never waits
// for the host).  Whenever a slot frees it re-orders everything not yet launched - requests
// waiting over 2 s first, then shortest estimated work first - and issues the next group:
// consecutive gathers as ONE persistent batched launch of at most ~2e9 evaluations, or one
// guided render (continuous batching: new requests compete for the very next slot).  A host
// function after a group's last kernel marks its requests done.  With batching off the
// worker issues one request at a time in arrival order with its own launches (the plain
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
    double cost = 0.0;        // estimated work, for ordering an iteration
    struct rzk_server *srv = nullptr;
};

constexpr double kLaunchCost = 2e9;   // work of one batched launch (~0.1 s of gather)
constexpr double kAgeMs = 2000.0;     // waiting longer than this overrides shortest-first
constexpr int kMaxInFlight = 2;       // launch groups on the stream: one running, one queued

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
    std::deque<Req *> queue;     // submitted, not yet seen by the worker
    std::vector<Req *> ready;    // seen by the worker, not yet launched
    int in_flight = 0;           // launch groups issued and not finished
    std::unordered_map<uint64_t, Req *> reqs;
    std::thread worker;
};

namespace {

// One launch group: the requests whose kernels were issued together; the host function
// after the group's last kernel marks them done.
struct Group {
    rzk_server *s = nullptr;
    std::vector<Req *> reqs;
    int64_t launches = 0;
};

void CUDART_CB on_group_done(void *p) {
    Group *g = (Group *)p;
    rzk_server *s = g->s;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        const double t = now_ms();
        for (Req *q : g->reqs) {
            q->t_done = t;
            q->state = q->status == RZK_OK ? kDone : kFailed;
            s->held -= (int64_t)q->bytes;
            s->n_completed++;
        }
        s->n_launches += g->launches;
        s->in_flight--;
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
    delete g;
}

// Issues one group: every request's primary hits, then its gathers as one batched launch
// (or, without batching, the request's own launches) or its guided render.
void launch_group(rzk_server *s, Group *g) {
    cudaStream_t st = s->st;
    std::vector<Req *> live;
    for (Req *q : g->reqs) {
        const size_t n = (size_t)q->r.camera.width * q->r.camera.height;
        if (cudaMallocAsync((void **)&q->d_recv, sizeof(rzk_receiver) * n, st) != cudaSuccess) {
            q->d_recv = nullptr;
            q->status = RZK_ERR_NOMEM;
            continue;
        }
        q->status = rzk_primary(q->r.scene, &q->r.camera, q->d_recv, st);
        g->launches++;
        if (q->status == RZK_OK) live.push_back(q);
    }
    std::vector<Req *> gathers;
    for (Req *q : live) {
        const rzk_request &r = q->r;
        if (r.kind == RZK_REQ_GUIDED) {
            rzk_guided_params gp{r.spp, r.max_bounce, r.rr_depth, r.rr_prob, 1, r.seed, r.sampler, 0};
            q->status = rzk_guided_render(s->ctx, r.scene, r.lightslice, &r.camera, &gp, r.d_rgb, nullptr, st);
            g->launches += r.sampler == RZK_GUIDE_METROPOLIS ? 3 : 2;   // (chains +) path kernel + per-pixel mean
        } else if (!s->prm.batching) {
            q->status = rzk_gather_cfg(s->ctx, r.scene, q->d_recv, r.camera.width * r.camera.height, r.camera.width,
                                       r.d_vpls, r.n_vpl, r.clamp_mode, r.tau, r.scale, r.d_rgb, 0, 0, st);
            g->launches += rzk::gather_launches(r.camera.width * r.camera.height, r.n_vpl, 0);
        } else {
            gathers.push_back(q);
        }
    }
    if (!gathers.empty()) {
        std::vector<rzk_gather_job> jobs(gathers.size());
        for (size_t i = 0; i < gathers.size(); ++i) {
            const rzk_request &r = gathers[i]->r;
            jobs[i] = rzk_gather_job{r.scene, gathers[i]->d_recv, r.camera.width * r.camera.height, r.camera.width,
                                     r.d_vpls, r.n_vpl, r.clamp_mode, r.tau, r.scale, r.d_rgb};
        }
        rzk::BatchPlan *plan = nullptr;
        rzk_status r = rzk::batch_plan_create(jobs.data(), (int)jobs.size(), 0, &plan);
        float *partial = nullptr;
        void *order = nullptr;
        int *work = nullptr;
        if (r == RZK_OK) {
            const size_t pf = rzk::batch_plan_partial_floats(plan), ob = rzk::batch_plan_order_bytes(plan);
            if (cudaMallocAsync((void **)&partial, sizeof(float) * std::max<size_t>(pf, 1), st) != cudaSuccess ||
                (ob > 0 && cudaMallocAsync(&order, ob, st) != cudaSuccess) ||
                cudaMallocAsync((void **)&work, sizeof(int) * rzk::batch_plan_tables(plan), st) != cudaSuccess)
                r = RZK_ERR_NOMEM;
        }
        if (r == RZK_OK) r = rzk::batch_plan_launch(plan, partial, order, work, 0, 0, st);
        if (r == RZK_OK) g->launches += rzk::batch_plan_launches(plan);
        if (partial) cudaFreeAsync(partial, st);
        if (order) cudaFreeAsync(order, st);
        if (work) cudaFreeAsync(work, st);
        if (plan) rzk::batch_plan_destroy(plan);
        for (Req *q : gathers) q->status = r;
    }
    for (Req *q : g->reqs)
        if (q->d_recv) cudaFreeAsync(q->d_recv, st);
    if (cudaLaunchHostFunc(st, on_group_done, g) != cudaSuccess) {
        // the stream cannot run host functions: finish the group here
        cudaStreamSynchronize(st);
        for (Req *q : g->reqs)
            if (q->status == RZK_OK) q->status = RZK_ERR_CUDA;
        on_group_done(g);
    }
}

// Picks the next group from the ready list (called with the lock held).  Batching:
// requests waiting longer than kAgeMs first in arrival order, then shortest estimated work
// first; consecutive gathers form one group while their total work stays within
// kLaunchCost; a guided render is a group of its own.  Without batching: arrival order,
// one request per group.
Group *next_group(rzk_server *s) {
    std::vector<Req *> &rd = s->ready;
    if (rd.empty()) return nullptr;
    Group *g = new Group();
    g->s = s;
    if (!s->prm.batching) {
        g->reqs.push_back(rd.front());
        rd.erase(rd.begin());
        return g;
    }
    const double now = now_ms();
    std::stable_sort(rd.begin(), rd.end(), [now](const Req *a, const Req *b) {
        const bool aa = now - a->t_submit > kAgeMs, ab = now - b->t_submit > kAgeMs;
        if (aa != ab) return aa;
        if (aa) return a->id < b->id;
        return a->cost < b->cost;
    });
    const int max_batch = s->prm.max_batch > 0 ? s->prm.max_batch : 256;
    size_t take = 1;
    if (rd.front()->r.kind == RZK_REQ_GATHER) {
        double cost = rd.front()->cost;
        while (take < rd.size() && (int)take < max_batch && rd[take]->r.kind == RZK_REQ_GATHER &&
               cost + rd[take]->cost <= kLaunchCost) {
            cost += rd[take]->cost;
            ++take;
        }
    }
    g->reqs.assign(rd.begin(), rd.begin() + take);
    rd.erase(rd.begin(), rd.begin() + take);
    return g;
}

void worker_main(rzk_server *s) {
    cudaSetDevice(s->device);
    while (true) {
        Group *g = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] {
                const bool work = !s->queue.empty() || !s->ready.empty();
                return (s->stop && !work) || (work && s->in_flight < kMaxInFlight);
            });
            while (!s->queue.empty()) {
                s->ready.push_back(s->queue.front());
                s->queue.pop_front();
            }
            if (s->ready.empty()) break;   // stopping and drained
            g = next_group(s);
            for (Req *q : g->reqs) q->state = kRunning;
            s->in_flight++;
        }
        launch_group(s, g);
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
        if (default_chunks(r.n_vpl) > 1)   // spatially ordered VPL copy and its sort scratch
            bytes += sizeof(rzk_vpl) * (size_t)r.n_vpl + rzk::order_scratch_bytes(r.n_vpl);
    } else if (r.kind == RZK_REQ_GUIDED) {
        if (!r.lightslice || r.spp <= 0 || r.max_bounce < 1 || r.max_bounce > 16 || r.rr_depth < 0 ||
            (r.rr_depth > 0 && !(r.rr_prob > 0.0f && r.rr_prob <= 1.0f)) ||
            (r.sampler != RZK_GUIDE_JENSEN && r.sampler != RZK_GUIDE_METROPOLIS))
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
    q->cost = r.kind == RZK_REQ_GATHER ? (double)n * (double)std::max(r.n_vpl, 1) : (double)n * r.spp * 32.0;
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
    auto qi = std::find(s->queue.begin(), s->queue.end(), q);
    if (qi != s->queue.end()) s->queue.erase(qi);
    auto ri = std::find(s->ready.begin(), s->ready.end(), q);
    if (ri != s->ready.end()) s->ready.erase(ri);
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
