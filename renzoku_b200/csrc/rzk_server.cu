// rzk_server.cu - a request loop for many users against device-resident scenes.
//
// Callers submit gather or guided-render requests (rzk_server_submit) from any thread.  A
// request is admitted only if the device memory it will hold while in flight (its receivers
// and, for a gather, its per-chunk partial sums and spatially ordered VPL copy; for a guided
// render, its per-path radiance and chain pool) fits the server's HBM budget next to the
// requests already admitted, and the device's free memory (sampled by the worker) has room
// for it; otherwise the call returns RZK_ERR_BUSY at once and the caller decides whether to
// retry.
//
// One worker thread owns a context and four streams ("lanes"): gathers run on one, guided
// renders on the other three, so the kinds of work overlap on the device - a guided
// render's paths fill the SMs a finishing gather frees and the reverse, and small guided
// renders (a few thousand paths, far fewer than the GPU holds) run side by side.  The
// gather lane and the first guided lane have the device's highest stream priority, the
// other two guided lanes its lowest: the oldest guided render takes the first guided lane
// and its blocks are scheduled ahead of the younger renders', which only backfill SMs it
// leaves idle, so it finishes about as fast as it would alone (the path kernel's blocks
// are short - one thread per path - so the priorities act as SMs free up).  The gather
// lane keeps at most two launch groups queued on its stream (one running, one behind it,
// so the GPU never waits for the host), each guided lane one.  Whenever a lane has room
// the worker issues its next group from the requests not yet launched, in arrival order:
// on the gather lane every waiting gather, oldest first, as ONE persistent batched launch
// of at most ~2e9 evaluations (a request larger than that goes alone); on a guided lane
// the oldest guided render (Metropolis renders only on the first guided lane: their chain
// pool is the context's scratch).  Continuous batching: a request that arrives while
// others run joins the lane's very next group.  A host function after a
// group's last kernel marks its requests done.  With batching off the worker issues one
// request at a time in arrival order, with its own launches, on one stream (the plain
// per-request baseline).  Scratch comes from the stream-ordered allocator, whose pool keeps
// freed blocks, so an iteration neither blocks on an allocation nor synchronises the device.
#include "rzk_internal.cuh"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdint>
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
enum { kLaneGather = 0, kLaneGuided = 1, kGuidedLanes = 3, kLanes = 1 + kGuidedLanes };

struct Req {
    uint64_t id = 0;
    rzk_request r{};
    size_t bytes = 0;
    int state = kQueued;
    rzk_status status = RZK_OK;
    double t_submit = 0.0, t_launch = 0.0, t_done = 0.0;
    rzk_receiver *d_recv = nullptr;
    float *d_paths = nullptr;
    double cost = 0.0;        // estimated work (evaluations, or paths x 32)
};

constexpr double kLaunchCost = 2e9;     // work of one batched launch (~30 ms of gather)
constexpr int kMaxInFlight = 2;         // launch groups on the gather lane: one running, one queued
constexpr int kGuidedInFlight = 1;      // per guided lane (concurrency comes from the lanes)
constexpr int64_t kFreeReserve = 256ll << 20;   // device memory never handed to requests
constexpr size_t kTimingCap = 1 << 20;  // completed requests whose timings are kept

int default_chunks(int n_vpl) {   // rzk_gather's automatic chunk count
    const int max_chunks = std::max(1, (n_vpl + 127) / 128);
    return std::min(32, max_chunks);
}

}  // namespace

struct rzk_server {
    int device = 0;
    rzk_context *ctx = nullptr;
    cudaStream_t st[kLanes] = {};
    rzk_server_params prm{};
    int64_t budget = 0, held = 0, free_bytes = 0;
    int64_t n_submitted = 0, n_rejected = 0, n_completed = 0, n_launches = 0;
    uint64_t next_id = 1;
    bool stop = false;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req *> queue;     // submitted, not yet seen by the worker
    std::vector<Req *> ready;    // seen by the worker, not yet launched (arrival order)
    int in_flight[kLanes] = {};   // launch groups issued and not finished, per lane
    std::unordered_map<uint64_t, Req *> reqs;
    // per completed request: kind, queue wait (submit -> launch) and run (launch -> done), ms
    std::vector<int32_t> t_kind;
    std::vector<double> t_queue, t_run;
    std::thread worker;
};

namespace {

// One launch group: the requests whose kernels were issued together on one lane; the host
// function after the group's last kernel marks them done.
struct Group {
    rzk_server *s = nullptr;
    int lane = kLaneGather;
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
            if (s->t_kind.size() < kTimingCap) {
                s->t_kind.push_back(q->r.kind);
                s->t_queue.push_back(q->t_launch - q->t_submit);
                s->t_run.push_back(t - q->t_launch);
            }
        }
        s->n_launches += g->launches;
        s->in_flight[g->lane]--;
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
    delete g;
}

// Issues one group on its lane's stream: every request's primary hits, then its gathers as
// one batched launch (or, without batching, the request's own launches) or its guided render.
void launch_group(rzk_server *s, Group *g) {
    cudaStream_t st = s->st[g->lane];
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
            const size_t n = (size_t)r.camera.width * r.camera.height;
            // the per-path radiance in the request's own buffer (no context scratch to grow)
            if (cudaMallocAsync((void **)&q->d_paths, sizeof(float) * 3 * n * (size_t)r.spp, st) != cudaSuccess) {
                q->d_paths = nullptr;
                q->status = RZK_ERR_NOMEM;
                continue;
            }
            rzk_guided_params gp{r.spp, r.max_bounce, r.rr_depth, r.rr_prob, 1, r.seed, r.sampler, 0};
            q->status = rzk_guided_render(s->ctx, r.scene, r.lightslice, &r.camera, &gp, r.d_rgb, q->d_paths, st);
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
        rzk_status r = rzk::batch_plan_create(jobs.data(), (int)jobs.size(), 0, 8, &plan);
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
    for (Req *q : g->reqs) {
        if (q->d_recv) cudaFreeAsync(q->d_recv, st);
        if (q->d_paths) cudaFreeAsync(q->d_paths, st);
        q->d_recv = nullptr;
        q->d_paths = nullptr;
    }
    if (cudaLaunchHostFunc(st, on_group_done, g) != cudaSuccess) {
        // the stream cannot run host functions: finish the group here
        cudaStreamSynchronize(st);
        for (Req *q : g->reqs)
            if (q->status == RZK_OK) q->status = RZK_ERR_CUDA;
        on_group_done(g);
    }
}

int lane_cap(int lane) { return lane == kLaneGather ? kMaxInFlight : kGuidedInFlight; }

// Whether a lane may run a request: the plain loop runs everything on the gather lane; with
// batching gathers take the gather lane, Jensen renders any guided lane, Metropolis renders
// the first one.
bool lane_takes(const rzk_server *s, int lane, const Req *q) {
    if (!s->prm.batching) return lane == kLaneGather;
    if (q->r.kind != RZK_REQ_GUIDED) return lane == kLaneGather;
    if (lane == kLaneGather) return false;
    return q->r.sampler != RZK_GUIDE_METROPOLIS || lane == kLaneGuided;
}

bool can_launch(const rzk_server *s, const Req *q) {
    for (int lane = 0; lane < kLanes; ++lane)
        if (s->in_flight[lane] < lane_cap(lane) && lane_takes(s, lane, q)) return true;
    return false;
}

// Picks the next group for a lane with room (called with the lock held), or nullptr.
// Batching: the gather lane takes every waiting gather in arrival order while their total
// work stays within kLaunchCost (at least one); the guided lane takes the oldest guided
// render.  Without batching: the oldest request, alone.
Group *next_group(rzk_server *s) {
    std::vector<Req *> &rd = s->ready;
    if (rd.empty()) return nullptr;
    if (!s->prm.batching) {
        if (s->in_flight[kLaneGather] >= kMaxInFlight) return nullptr;
        Group *g = new Group();
        g->s = s;
        g->reqs.push_back(rd.front());
        rd.erase(rd.begin());
        return g;
    }
    for (int lane = 0; lane < kLanes; ++lane) {
        if (s->in_flight[lane] >= lane_cap(lane)) continue;
        const int max_batch = lane != kLaneGather ? 1 : (s->prm.max_batch > 0 ? s->prm.max_batch : 256);
        std::vector<Req *> take;
        double cost = 0.0;
        for (Req *q : rd) {
            if (!lane_takes(s, lane, q)) continue;
            if (!take.empty() && ((int)take.size() >= max_batch || cost + q->cost > kLaunchCost)) break;
            take.push_back(q);
            cost += q->cost;
        }
        if (take.empty()) continue;
        Group *g = new Group();
        g->s = s;
        g->lane = lane;
        g->reqs = take;
        rd.erase(std::remove_if(rd.begin(), rd.end(),
                                [&](Req *q) { return std::find(take.begin(), take.end(), q) != take.end(); }),
                 rd.end());
        return g;
    }
    return nullptr;
}

void worker_main(rzk_server *s) {
    cudaSetDevice(s->device);
    while (true) {
        Group *g = nullptr;
        {
            size_t fr = 0, tot = 0;
            if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) {
                std::lock_guard<std::mutex> lk(s->mu);
                s->free_bytes = (int64_t)fr;
            }
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] {
                while (!s->queue.empty()) {
                    s->ready.push_back(s->queue.front());
                    s->queue.pop_front();
                }
                if (s->ready.empty()) return s->stop;
                for (Req *q : s->ready)
                    if (can_launch(s, q)) return true;
                return false;
            });
            if (s->ready.empty()) break;   // stopping and drained
            g = next_group(s);
            if (!g) continue;
            const double t = now_ms();
            for (Req *q : g->reqs) {
                q->state = kRunning;
                q->t_launch = t;
            }
            s->in_flight[g->lane]++;
        }
        launch_group(s, g);
    }
    for (cudaStream_t st : s->st)
        if (st) cudaStreamSynchronize(st);
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
    int prio_least = 0, prio_greatest = 0;
    cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest);
    for (int lane = 0; lane < kLanes; ++lane)
        if (cudaStreamCreateWithPriority(&s->st[lane], cudaStreamNonBlocking,
                                         lane <= kLaneGuided ? prio_greatest : prio_least) != cudaSuccess) {
            for (cudaStream_t x : s->st)
                if (x) cudaStreamDestroy(x);
            rzk_context_destroy(s->ctx);
            delete s;
            return RZK_ERR_CUDA;
        }
    // the stream-ordered pool keeps freed blocks for the next requests instead of returning
    // them to the driver at every synchronisation
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    s->free_bytes = (int64_t)fr;
    s->budget = params->hbm_budget_bytes;
    if (s->budget == 0) s->budget = (int64_t)(0.9 * (double)fr);
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
    for (cudaStream_t st : s->st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    for (auto &kv : s->reqs) delete kv.second;
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
        if (n * (int64_t)r.spp > (1LL << 31)) return RZK_ERR_CAPACITY;
        // the per-path radiance, and the Metropolis chains' pool (4,096 states per slice)
        bytes += sizeof(float) * 3 * (size_t)n * (size_t)r.spp;
        if (r.sampler == RZK_GUIDE_METROPOLIS) {
            int32_t ns = 0;
            if (rzk_lightslice_info(r.lightslice, nullptr, &ns, nullptr, nullptr, nullptr, nullptr) == RZK_OK)
                bytes += 16 * 4096 * (size_t)std::max(ns, 0);
        }
    } else {
        return RZK_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return RZK_ERR_INVALID;
    s->n_submitted++;
    // the budget, and the device's free memory as the worker last sampled it, minus what the
    // admitted but not yet launched requests will take from it
    int64_t pending = 0;
    for (Req *q : s->queue) pending += (int64_t)q->bytes;
    for (Req *q : s->ready) pending += (int64_t)q->bytes;
    if (s->held + (int64_t)bytes > s->budget || (int64_t)bytes + pending > s->free_bytes - kFreeReserve) {
        s->n_rejected++;
        return RZK_ERR_BUSY;
    }
    Req *q = new Req();
    q->id = s->next_id++;
    q->r = r;
    q->bytes = bytes;
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

rzk_status rzk_server_timings(rzk_server *s, int32_t *h_kind, double *h_queue_ms, double *h_run_ms, int cap,
                              int32_t *n) {
    if (!s || !n || cap < 0 || (cap > 0 && (!h_kind || !h_queue_ms || !h_run_ms))) return RZK_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    const int k = (int)std::min<size_t>((size_t)cap, s->t_kind.size());
    std::copy(s->t_kind.begin(), s->t_kind.begin() + k, h_kind);
    std::copy(s->t_queue.begin(), s->t_queue.begin() + k, h_queue_ms);
    std::copy(s->t_run.begin(), s->t_run.begin() + k, h_run_ms);
    *n = (int32_t)s->t_kind.size();
    return RZK_OK;
}

}  // extern "C"
