// fdzb_serve.cpp -- request server with continuous batching.
//
// No counterpart in the reference, which renders one frame per FD::FDLaunch
// from a single-threaded GL application (FS/api.cpp:405-575, K/FourD.cu:47-136).
// Scenes (triangle soups) are registered once and stay resident in HBM; shadow
// requests (scene id, view-sample buffers, light rectangle, grid size) are
// queued by any thread.  A worker thread owns `slots` engines, each with its
// own stream and arena: whenever a slot is free and requests are waiting, it
// forms a batch from the head of the queue -- as many requests as fit the
// frame and sample limits and the memory budget -- and launches it.  Batches
// on different slots run concurrently on the GPU, so requests that arrive
// while others are on the device start without waiting for them to finish.
// A host callback on each slot's stream marks completion; per-request latency
// runs from submission to that callback.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/fdzb.h"
#include "fdzb_engine.h"
#include "fdzb_internal.h"

// ABI layouts mirrored by the ctypes binding
static_assert(sizeof(fdzb_serve_config) == 40, "fdzb_serve_config layout");
static_assert(sizeof(fdzb_request) == 112, "fdzb_request layout");
static_assert(sizeof(fdzb_request_result) == 208, "fdzb_request_result layout");
static_assert(sizeof(fdzb_serve_stats) == 144, "fdzb_serve_stats layout");

namespace {

using fdzb::Engine;
using fdzb::FrameSpec;

double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

size_t align_mb(size_t v) { return (v + (1u << 20) - 1) / (1u << 20) * (1u << 20); }

struct SceneRec {
    const float *vtx = nullptr;
    size_t nv = 0, stride = 16;
    const int32_t *idx = nullptr;
    size_t nt = 0;
    int cull = 0;
    float esp = 1e-3f;
};

enum ReqState { REQ_QUEUED = 0, REQ_RUNNING = 1, REQ_DONE = 2 };

struct Request {
    FrameSpec spec;
    size_t outBytes = 0;        // shadow + masks the request writes
    double tSubmit = 0, tLaunch = 0, tDone = 0;
    int state = REQ_QUEUED;
    int status = FDZB_OK;
    int batchFrames = 0;
    fdzb_frame_stats stats{};
};

struct Slot {
    Engine eng;
    std::vector<uint64_t> tickets;
    bool busy = false;
    std::atomic<bool> done{false};
    double tDone = 0;
    size_t outBytes = 0;        // outputs of the requests in flight on this slot
    fdzb_server *srv = nullptr;
};

}  // namespace

struct fdzb_server {
    fdzb_serve_config cfg{};
    std::vector<SceneRec> scenes;
    std::vector<std::unique_ptr<Slot>> slots;
    std::mutex mu;
    std::condition_variable cv;       // worker: new request or slot completion
    std::condition_variable cvDone;   // waiters: a request finished
    std::deque<uint64_t> queue;
    std::unordered_map<uint64_t, Request> reqs;
    uint64_t nextTicket = 1;
    std::thread worker;
    bool stop = false;
    fdzb::TuneTable tuned;
    std::string workerError;
    // statistics
    std::vector<double> lat;          // ms, completed requests since reset
    long long submitted = 0, completed = 0, rejected = 0, failed = 0, batches = 0, batchedFrames = 0;
    long long overlappedBatches = 0, arenaTrims = 0, splits = 0;
    int frameLimit = 1 << 30;         // lowered after a batch overflowed the pair buffer
    int maxInflight = 0;
    size_t peakBytes = 0;
    double tFirstSubmit = -1, tLastDone = -1;
};

namespace {

// Bytes the server holds for slot arenas plus the outputs of in-flight requests.
size_t held_bytes(const fdzb_server *s)
{
    size_t b = 0;
    for (const auto &sl : s->slots) b += sl->eng.arenaBytes + (sl->busy ? sl->outBytes : 0);
    return b;
}

void CUDART_CB on_slot_done(void *p)
{
    Slot *sl = static_cast<Slot *>(p);
    sl->tDone = now_s();
    sl->done.store(true);
    fdzb_server *s = sl->srv;
    { std::lock_guard<std::mutex> g(s->mu); }
    s->cv.notify_all();
}

// Forms a batch for an idle slot from the head of the queue (lock held).
// Returns the tickets taken; rejects requests that cannot fit the budget on
// their own.
std::vector<uint64_t> take_batch(fdzb_server *s, Slot &sl, std::vector<FrameSpec> &specs, size_t &outBytes)
{
    std::vector<uint64_t> take;
    const size_t budget = s->cfg.memory_budget_bytes;
    const size_t others = held_bytes(s) - sl.eng.arenaBytes;
    long long samples = 0, tris = 0;
    outBytes = 0;
    while (!s->queue.empty() && (int)take.size() < s->cfg.max_batch_frames) {
        const uint64_t t = s->queue.front();
        Request &r = s->reqs[t];
        const long long S = (long long)r.spec.W * r.spec.H;
        if (!take.empty() && (samples + S > s->cfg.max_batch_samples ||
                              tris + (long long)r.spec.nt > s->cfg.max_batch_triangles ||
                              (int)take.size() >= s->frameLimit))
            break;
        specs.push_back(r.spec);
        const long long pairCap = std::max(sl.eng.pairCapacity, fdzb::default_pair_capacity(tris + (long long)r.spec.nt));
        const size_t arena = std::max(sl.eng.arenaBytes, align_mb(fdzb::launch_bytes(specs, pairCap, false) * 9 / 8));
        if (others + arena + outBytes + r.outBytes > budget) {
            specs.pop_back();
            if (take.empty()) {
                // alone on an otherwise idle server it still would not fit: reject
                bool idle = true;
                for (const auto &o : s->slots) idle = idle && !o->busy;
                const size_t alone = align_mb(fdzb::launch_bytes({r.spec}, fdzb::default_pair_capacity((long long)r.spec.nt), false) * 9 / 8);
                if (idle && alone + r.outBytes > budget) {
                    r.state = REQ_DONE;
                    r.status = FDZB_ERR_NO_MEMORY;
                    r.tDone = now_s();
                    ++s->rejected;
                    s->queue.pop_front();
                    s->cvDone.notify_all();
                    continue;
                }
            }
            break;
        }
        samples += S;
        tris += (long long)r.spec.nt;
        outBytes += r.outBytes;
        take.push_back(t);
        s->queue.pop_front();
    }
    return take;
}

void worker_main(fdzb_server *s)
{
    cudaSetDevice(s->cfg.device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        bool progressed = false;
        // 1. harvest finished slots
        for (auto &up : s->slots) {
            Slot &sl = *up;
            if (!sl.busy || !sl.done.load()) continue;
            lk.unlock();
            const int rc = fdzb::engine_sync(sl.eng);   // returns at once unless the pairs overflowed
            std::string err = rc ? fdzb_last_error() : std::string();
            const double tDone = sl.eng.replans ? now_s() : sl.tDone;
            lk.lock();
            if (rc == FDZB_ERR_CAPACITY && sl.tickets.size() > 1) {
                // the batch's pair list outgrew the largest buffer: requeue its
                // requests at the head and launch them in smaller batches
                for (size_t i = sl.tickets.size(); i-- > 0;) {
                    auto it = s->reqs.find(sl.tickets[i]);
                    if (it == s->reqs.end()) continue;
                    it->second.state = REQ_QUEUED;
                    s->queue.push_front(sl.tickets[i]);
                }
                s->frameLimit = std::max(1, (int)sl.tickets.size() / 2);
                ++s->splits;
                sl.tickets.clear();
                sl.busy = false;
                sl.done.store(false);
                progressed = true;
                continue;
            }
            for (size_t i = 0; i < sl.tickets.size(); ++i) {
                auto it = s->reqs.find(sl.tickets[i]);
                if (it == s->reqs.end()) continue;
                Request &r = it->second;
                r.state = REQ_DONE;
                r.status = rc;
                r.tDone = tDone;
                if (rc == FDZB_OK) {
                    fdzb::frame_stats(sl.eng, (int)i, r.stats);
                    ++s->completed;
                    s->lat.push_back(1e3 * (tDone - r.tSubmit));
                } else {
                    ++s->failed;
                    s->workerError = err;
                }
            }
            s->tLastDone = std::max(s->tLastDone, tDone);
            sl.tickets.clear();
            sl.busy = false;
            sl.done.store(false);
            progressed = true;
            s->cvDone.notify_all();
        }
        // 2. dispatch waiting requests to idle slots, largest arena first (its
        //    memory is reused); when the head of the queue does not fit, free
        //    the arenas of the other idle slots and try again
        while (!s->queue.empty()) {
            Slot *pick = nullptr;
            for (auto &up : s->slots)
                if (!up->busy && (!pick || up->eng.arenaBytes > pick->eng.arenaBytes)) pick = up.get();
            if (!pick) break;
            Slot &sl = *pick;
            std::vector<FrameSpec> specs;
            size_t outBytes = 0;
            std::vector<uint64_t> take = take_batch(s, sl, specs, outBytes);
            if (take.empty()) {
                if (s->queue.empty()) break;   // the rest was rejected
                std::vector<Slot *> trim;
                for (auto &up : s->slots)
                    if (up.get() != pick && !up->busy && up->eng.arenaBytes > 0) trim.push_back(up.get());
                if (trim.empty()) break;       // wait for a busy slot to finish
                for (Slot *t : trim) t->busy = true;
                lk.unlock();
                for (Slot *t : trim) fdzb::engine_free_arena(t->eng);
                lk.lock();
                for (Slot *t : trim) t->busy = false;
                ++s->arenaTrims;
                continue;
            }
            int inflight = 1;
            for (const auto &o : s->slots) inflight += o->busy ? 1 : 0;
            const double tl = now_s();
            for (uint64_t t : take) {
                Request &r = s->reqs[t];
                r.state = REQ_RUNNING;
                r.tLaunch = tl;
                r.batchFrames = (int)take.size();
            }
            sl.busy = true;
            sl.done.store(false);
            sl.tickets = take;
            sl.outBytes = outBytes;
            ++s->batches;
            s->batchedFrames += (long long)take.size();
            if (inflight > 1) ++s->overlappedBatches;
            s->maxInflight = std::max(s->maxInflight, inflight);
            lk.unlock();
            sl.eng.frames.swap(specs);
            int rc = fdzb::engine_enqueue(sl.eng);
            if (rc == FDZB_OK && cudaLaunchHostFunc(sl.eng.stream, on_slot_done, &sl) != cudaSuccess)
                rc = FDZB_ERR_CUDA;
            std::string err = rc ? fdzb_last_error() : std::string();
            if (rc != FDZB_OK && sl.eng.pending) {
                cudaStreamSynchronize(sl.eng.stream);
                sl.eng.pending = false;
            }
            lk.lock();
            s->peakBytes = std::max(s->peakBytes, held_bytes(s));
            if (rc != FDZB_OK) {
                for (uint64_t t : take) {
                    Request &r = s->reqs[t];
                    r.state = REQ_DONE;
                    r.status = rc;
                    r.tDone = now_s();
                    ++s->failed;
                }
                s->workerError = err;
                sl.busy = false;
                sl.tickets.clear();
                s->cvDone.notify_all();
            }
            progressed = true;
        }
        if (!progressed) {
            bool any = false;
            for (const auto &up : s->slots) any = any || (up->busy && up->done.load());
            if (!any) s->cv.wait_for(lk, std::chrono::milliseconds(2));
        }
    }
}

int srv_check(fdzb_server *s)
{
    if (!s) return fdzb::set_error(FDZB_ERR_NOT_INITIALIZED, "server is NULL");
    return FDZB_OK;
}

void percentile(std::vector<double> v, double *p50, double *p99, double *mean, double *mx)
{
    *p50 = *p99 = *mean = *mx = 0;
    if (v.empty()) return;
    std::sort(v.begin(), v.end());
    auto at = [&](double q) {
        const double pos = q * (double)(v.size() - 1);
        const size_t i = (size_t)pos;
        const double f = pos - (double)i;
        return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
    };
    *p50 = at(0.50);
    *p99 = at(0.99);
    double sum = 0;
    for (double x : v) sum += x;
    *mean = sum / (double)v.size();
    *mx = v.back();
}

void result_of(const Request &r, fdzb_request_result *out)
{
    std::memset(out, 0, sizeof(*out));
    out->status = r.status;
    out->batch_frames = r.batchFrames;
    out->latency_ms = 1e3 * (r.tDone - r.tSubmit);
    out->queue_ms = r.tLaunch > 0 ? 1e3 * (r.tLaunch - r.tSubmit) : out->latency_ms;
    out->stats = r.stats;
}

}  // namespace

extern "C" {

void fdzb_serve_default_config(fdzb_serve_config *cfg)
{
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->device = -1;
    cfg->slots = 2;
    cfg->max_batch_frames = 16;
    cfg->max_batch_samples = 16ll << 20;
    cfg->max_batch_triangles = 4ll << 20;
    cfg->memory_budget_bytes = 150ull * 1000 * 1000 * 1000;
    cfg->use_graphs = 0;
}

int fdzb_serve_create(fdzb_server **out, const fdzb_serve_config *cfg)
{
    if (!out) return fdzb::set_error(FDZB_ERR_INVALID_ARG, "out is NULL");
    fdzb_serve_config c;
    fdzb_serve_default_config(&c);
    if (cfg) c = *cfg;
    if (c.slots < 1 || c.slots > 16) return fdzb::set_error(FDZB_ERR_INVALID_ARG, "slots must be in [1, 16]");
    if (c.max_batch_frames < 1) return fdzb::set_error(FDZB_ERR_INVALID_ARG, "max_batch_frames must be >= 1");
    if (c.max_batch_samples < 1) return fdzb::set_error(FDZB_ERR_INVALID_ARG, "max_batch_samples must be >= 1");
    if (c.max_batch_triangles < 1) return fdzb::set_error(FDZB_ERR_INVALID_ARG, "max_batch_triangles must be >= 1");
    if (c.device < 0) {
        cudaError_t e = cudaGetDevice(&c.device);
        if (e != cudaSuccess) return fdzb::set_error(FDZB_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    }
    fdzb_server *s = new (std::nothrow) fdzb_server();
    if (!s) return fdzb::set_error(FDZB_ERR_NO_MEMORY, "host allocation failed");
    s->cfg = c;
    for (int i = 0; i < c.slots; ++i) {
        auto sl = std::make_unique<Slot>();
        sl->srv = s;
        int rc = fdzb::engine_init(sl->eng, c.device);
        sl->eng.useGraph = c.use_graphs != 0;
        if (rc) {
            for (auto &o : s->slots) fdzb::engine_release(o->eng);
            fdzb::engine_release(sl->eng);
            delete s;
            return rc;
        }
        s->slots.push_back(std::move(sl));
    }
    s->worker = std::thread(worker_main, s);
    *out = s;
    return FDZB_OK;
}

int fdzb_serve_destroy(fdzb_server *s)
{
    if (!s) return FDZB_OK;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (auto &sl : s->slots) fdzb::engine_release(sl->eng);   // waits for its stream (and callback)
    delete s;
    return FDZB_OK;
}

int fdzb_serve_add_scene(fdzb_server *s, const float *d_vtx, size_t n_vtx, size_t vtx_stride_bytes,
                         const int32_t *d_idx, size_t n_tri, int cull, float esp, int32_t *scene_id)
{
    if (int rc = srv_check(s)) return rc;
    if (!scene_id) return fdzb::set_error(FDZB_ERR_INVALID_ARG, "scene_id is NULL");
    if ((n_vtx && !d_vtx) || (n_tri && !d_idx)) return fdzb::set_error(FDZB_ERR_INVALID_ARG, "NULL scene buffer");
    if (vtx_stride_bytes < 12 || vtx_stride_bytes % 4)
        return fdzb::set_error(FDZB_ERR_INVALID_ARG, "vertex stride must be >= 12 and a multiple of 4 bytes");
    SceneRec r;
    r.vtx = d_vtx;
    r.nv = n_vtx;
    r.stride = vtx_stride_bytes;
    r.idx = d_idx;
    r.nt = n_tri;
    r.cull = cull ? 1 : 0;
    r.esp = esp;
    std::lock_guard<std::mutex> g(s->mu);
    s->scenes.push_back(r);
    *scene_id = (int32_t)s->scenes.size() - 1;
    return FDZB_OK;
}

int fdzb_serve_submit(fdzb_server *s, const fdzb_request *q, uint64_t *ticket)
{
    if (int rc = srv_check(s)) return rc;
    if (!q || !ticket) return fdzb::set_error(FDZB_ERR_INVALID_ARG, "NULL request or ticket");
    fdzb_frame_desc d{};
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (q->scene_id < 0 || q->scene_id >= (int)s->scenes.size())
            return fdzb::set_error(FDZB_ERR_INVALID_ARG, "unknown scene id " + std::to_string(q->scene_id));
        const SceneRec &sc = s->scenes[q->scene_id];
        d.d_vtx = sc.vtx;
        d.n_vtx = sc.nv;
        d.vtx_stride_bytes = sc.stride;
        d.d_idx = sc.idx;
        d.n_tri = sc.nt;
        d.cull = sc.cull;
        d.esp = sc.esp;
    }
    d.d_pos = q->d_pos;
    d.d_nrm = q->d_nrm;
    d.W = q->W;
    d.H = q->H;
    d.light = q->light;
    d.bins = q->bins;
    d.d_shadow = q->d_shadow;
    d.d_masks = q->d_masks;
    d.model_transform = q->model_transform;
    Request r;
    if (int rc = fdzb::desc_to_spec(d, r.spec, 0)) return rc;
    if (q->W <= 0 || q->H <= 0 || (long long)q->W * q->H > (1ll << 30))
        return fdzb::set_error(FDZB_ERR_INVALID_ARG, "bad view size");
    if (!q->d_pos || !q->d_nrm || !q->d_shadow) return fdzb::set_error(FDZB_ERR_INVALID_ARG, "NULL view or output buffer");
    if (q->bins != 0 && (q->bins < 1 || q->bins > fdzb::kMaxBins || (q->bins & (q->bins - 1))))
        return fdzb::set_error(FDZB_ERR_INVALID_ARG, "bin number must be 0 or a power of two in [1, 512]");
    const long long S = (long long)q->W * q->H;
    r.outBytes = (size_t)S * 4 + (q->d_masks ? (size_t)S * 4 * ((r.spec.light.N * r.spec.light.NC + 31) / 32) : 0);
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (r.spec.bins == 0) {
            const fdzb::TuneChoice c = fdzb::tuned_shape(s->tuned, r.spec);
            r.spec.bins = c.bins;
            r.spec.occChunk = c.chunk;
            r.spec.occItem = c.item;
        }
        r.tSubmit = now_s();
        if (s->tFirstSubmit < 0) s->tFirstSubmit = r.tSubmit;
        const uint64_t t = s->nextTicket++;
        s->reqs.emplace(t, r);
        s->queue.push_back(t);
        ++s->submitted;
        *ticket = t;
    }
    s->cv.notify_all();
    return FDZB_OK;
}

int fdzb_serve_poll(fdzb_server *s, uint64_t ticket, fdzb_request_result *out)
{
    if (int rc = srv_check(s)) return rc;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return fdzb::set_error(FDZB_ERR_INVALID_ARG, "unknown ticket");
    if (it->second.state != REQ_DONE) return 0;
    if (out) result_of(it->second, out);
    s->reqs.erase(it);
    return 1;
}

int fdzb_serve_wait(fdzb_server *s, uint64_t ticket, int timeout_ms, fdzb_request_result *out)
{
    if (int rc = srv_check(s)) return rc;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return fdzb::set_error(FDZB_ERR_INVALID_ARG, "unknown ticket");
    const auto pred = [&] {
        auto i2 = s->reqs.find(ticket);
        return i2 == s->reqs.end() || i2->second.state == REQ_DONE;
    };
    if (timeout_ms < 0) {
        s->cvDone.wait(lk, pred);
    } else if (!s->cvDone.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred)) {
        return 0;
    }
    it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return fdzb::set_error(FDZB_ERR_INVALID_ARG, "ticket collected by another caller");
    if (out) result_of(it->second, out);
    s->reqs.erase(it);
    return 1;
}

int fdzb_serve_drain(fdzb_server *s, int timeout_ms)
{
    if (int rc = srv_check(s)) return rc;
    std::unique_lock<std::mutex> lk(s->mu);
    const auto pred = [&] {
        if (!s->queue.empty()) return false;
        for (const auto &sl : s->slots)
            if (sl->busy) return false;
        return true;
    };
    if (timeout_ms < 0) {
        s->cvDone.wait(lk, pred);
        return 1;
    }
    return s->cvDone.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred) ? 1 : 0;
}

int fdzb_serve_autotune(fdzb_server *s, const fdzb_request *reqs, int n, float *d_scratch, size_t scratch_floats)
{
    if (int rc = srv_check(s)) return rc;
    if (!reqs || n <= 0) return fdzb::set_error(FDZB_ERR_INVALID_ARG, "empty request list");
    if (fdzb_serve_drain(s, -1) < 0) return FDZB_ERR_CUDA;
    std::vector<FrameSpec> specs;
    {
        std::lock_guard<std::mutex> g(s->mu);
        for (int i = 0; i < n; ++i) {
            const fdzb_request &q = reqs[i];
            if (q.scene_id < 0 || q.scene_id >= (int)s->scenes.size())
                return fdzb::set_error(FDZB_ERR_INVALID_ARG, "unknown scene id");
            const SceneRec &sc = s->scenes[q.scene_id];
            fdzb_frame_desc d{};
            d.d_pos = q.d_pos;
            d.d_nrm = q.d_nrm;
            d.W = q.W;
            d.H = q.H;
            d.d_vtx = sc.vtx;
            d.n_vtx = sc.nv;
            d.vtx_stride_bytes = sc.stride;
            d.d_idx = sc.idx;
            d.n_tri = sc.nt;
            d.light = q.light;
            d.cull = sc.cull;
            d.esp = sc.esp;
            d.d_shadow = q.d_shadow;
            FrameSpec f;
            if (int rc = fdzb::desc_to_spec(d, f, i)) return rc;
            specs.push_back(f);
        }
    }
    // slot 0 is idle after the drain and the worker only touches busy slots or
    // dispatches when the queue is non-empty; hold the queue empty meanwhile
    std::unique_lock<std::mutex> lk(s->mu);
    if (!s->queue.empty()) return fdzb::set_error(FDZB_ERR_NOT_READY, "requests submitted during autotuning");
    Slot &sl = *s->slots[0];
    sl.busy = true;   // keep the worker away from slot 0
    fdzb::TuneTable table = s->tuned;
    lk.unlock();
    long long launches = 0;
    int rc = fdzb::autotune_bins(sl.eng, table, specs, d_scratch, scratch_floats, &launches);
    lk.lock();
    sl.busy = false;
    if (rc == FDZB_OK) s->tuned = table;
    s->cv.notify_all();
    return rc;
}

int fdzb_serve_get_stats(fdzb_server *s, fdzb_serve_stats *out)
{
    if (int rc = srv_check(s)) return rc;
    if (!out) return fdzb::set_error(FDZB_ERR_INVALID_ARG, "out is NULL");
    std::lock_guard<std::mutex> g(s->mu);
    std::memset(out, 0, sizeof(*out));
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->rejected = s->rejected;
    out->failed = s->failed;
    out->batches = s->batches;
    out->batched_frames = s->batchedFrames;
    out->overlapped_batches = s->overlappedBatches;
    out->queued = (int64_t)s->queue.size();
    int busy = 0;
    for (const auto &sl : s->slots) busy += sl->busy ? 1 : 0;
    out->busy_slots = busy;
    out->max_inflight_batches = s->maxInflight;
    percentile(s->lat, &out->p50_ms, &out->p99_ms, &out->mean_ms, &out->max_ms);
    const double span = s->tLastDone - s->tFirstSubmit;
    out->frames_per_s = (s->completed > 0 && span > 0) ? (double)s->completed / span : 0.0;
    out->held_bytes = (int64_t)held_bytes(s);
    out->peak_bytes = (int64_t)s->peakBytes;
    out->budget_bytes = (int64_t)s->cfg.memory_budget_bytes;
    out->tuned_classes = (int32_t)s->tuned.size();
    out->slots = (int32_t)s->slots.size();
    return FDZB_OK;
}

int fdzb_serve_reset_stats(fdzb_server *s)
{
    if (int rc = srv_check(s)) return rc;
    std::lock_guard<std::mutex> g(s->mu);
    s->lat.clear();
    s->submitted = s->completed = s->rejected = s->failed = s->batches = s->batchedFrames = 0;
    s->overlappedBatches = 0;
    s->maxInflight = 0;
    s->peakBytes = held_bytes(s);
    s->tFirstSubmit = s->tLastDone = -1;
    return FDZB_OK;
}

const char *fdzb_serve_last_worker_error(fdzb_server *s)
{
    if (!s) return "";
    std::lock_guard<std::mutex> g(s->mu);
    static thread_local std::string copy;
    copy = s->workerError;
    return copy.c_str();
}

}  // extern "C"
