// server.cpp - hvvr_server: a render-request loop with admission control and continuous
// batching over resident scenes (no counterpart in the reference, whose Raycaster renders
// its cameras once per render() call).
//
// Requests name a view template (a sample set and viewport over one resident scene, clustered
// once when the template is added), an MSAA rate, a camera pose and an output image. One
// worker thread owns all GPU work of the server:
//   * admission - a request needs a camera instance of its template: a free one from the
//     template's pool, or a new clone (device copies of the template's setup) if the device
//     memory of all instances plus the slots' triangle-list pools stays within the HBM budget.
//     Requests that cannot be admitted wait; later requests that fit may go first.
//   * batching - up to max_batch_views admitted requests form one frame batch (one launch per
//     stage over all views, traversal as one longest-first work queue) on a free slot. Up to
//     `slots` batches are in flight on their own streams, so requests that arrive while a batch
//     runs are rendered by the next one, overlapping on the device. An idle GPU takes any
//     request at once; with a batch in flight the next one waits for min_batch_views requests
//     or for its oldest request to have waited max_wait_ms.
//   * latency class - requests with priority 1 (the two eyes of a stereo frame, say) go to the
//     latency slots: dispatched as soon as one is free, never held back to fill a batch, on
//     streams of the GPU's highest priority while the throughput slots run at its lowest, so
//     their CTAs are scheduled ahead of the throughput batches' pending ones. With latency
//     isolation (default) the throughput slots' frames cull non-persistently (a warp per tile) and
//     without the cull -> shade pipeline, so no throughput CTA holds an SM slot for longer than one
//     tile or waits on another CTA, and each slot one frees goes to the latency class first.
//     When the budget is short, idle instances of other templates are freed first.
//   * completion - a slot whose end event has fired returns its instances to the pools and its
//     requests to the completion queue (CPU outputs are copied out of pinned staging first).
//   * animation - vertex updates are staged on the device when submitted and applied between
//     batches: the worker waits until no batch is in flight, copies them into the scenes,
//     refits on the device and makes every slot stream wait for the refit.
// A request's image does not depend on the other requests of its batch: each view is a
// separate camera with its own buffers and the kernels are per tile, so the result is the
// same alone and in any mix.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>

#include <string.h>

#include "host_objects.h"

using namespace hvb;

namespace {

struct Template {
    hvvr_raycaster* rc = nullptr;
    hvvr_camera* proto = nullptr;
    uint32_t width = 0, height = 0;
    uint32_t samples = 0;
    size_t instBytes = 0;
    std::vector<struct Instance*> freeList;
};

struct Instance {
    hvvr_camera* cam = nullptr;
    uint32_t tmpl = 0;
    uint32_t width = 0, height = 0; // the template's image size (read without the server lock)
    DevBuf<uint32_t> image;         // device image the remap writes for CPU outputs
    uint32_t* staging = nullptr;    // pinned copy of image for CPU outputs (made on first use)
    size_t bytes = 0;
};

struct Request {
    uint64_t id = 0;
    hvvr_request r{};
    double submitMs = 0, dispatchMs = 0, doneMs = 0;
    int status = HVVR_OK;
    Instance* inst = nullptr;
    uint32_t batchViews = 0;
};

struct Update {
    hvvr_raycaster* rc = nullptr;
    size_t vertOffset = 0;   // in vertices, into the scene's concatenated vertex array
    uint32_t count = 0;
    DevBuf<float4> verts;    // 2 float4 per vertex
};

struct Slot {
    std::unique_ptr<hvvr_batch> batch;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    std::vector<Request*> reqs;
    bool busy = false;
    bool latency = false;           // renders only latency-class requests, at the highest priority
};

} // namespace

struct hvvr_server {
    hvvr_server_config cfg{};
    std::vector<hvvr_raycaster*> scenes;
    std::vector<Template> templates;
    std::vector<std::unique_ptr<Instance>> instances;
    std::vector<Slot> slots;
    cudaStream_t updateStream = nullptr;
    cudaEvent_t updateEv = nullptr;
    size_t poolBytes = 0, memUsed = 0, memPeak = 0;
    size_t reservedFor = 0;             // template count the slots' frame buffers are sized for

    std::mutex mu;                       // guards everything below
    std::condition_variable workCv, doneCv;
    std::deque<Request*> pending;
    std::vector<std::unique_ptr<Update>> updates;
    std::deque<hvvr_completion> completions;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> live;
    uint64_t nextId = 1;
    hvvr_server_stats stats{};
    uint64_t viewsDispatched = 0;
    bool stop = false;
    std::string workerError;

    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    std::thread worker;

    double nowMs() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

// frees idle instances of templates other than t, largest first, until `need` more bytes fit
bool evictFor(hvvr_server* s, uint32_t t, size_t need) {
    if (s->memUsed + need <= s->cfg.hbm_budget_bytes) return true;
    std::vector<Instance*> idle;
    for (uint32_t k = 0; k < s->templates.size(); k++)
        if (k != t)
            for (Instance* i : s->templates[k].freeList) idle.push_back(i);
    std::sort(idle.begin(), idle.end(), [](const Instance* a, const Instance* b) { return a->bytes > b->bytes; });
    size_t freeable = 0;
    for (Instance* i : idle) freeable += i->bytes;
    if (s->memUsed - freeable + need > s->cfg.hbm_budget_bytes) return false;
    for (Instance* i : idle) {
        if (s->memUsed + need <= s->cfg.hbm_budget_bytes) break;
        auto& fl = s->templates[i->tmpl].freeList;
        fl.erase(std::remove(fl.begin(), fl.end(), i), fl.end());
        if (i->staging) cudaFreeHost(i->staging);
        hvvr_camera_destroy(i->cam->rc, i->cam);
        s->memUsed -= i->bytes;
        s->stats.evicted++;
        s->instances.erase(std::remove_if(s->instances.begin(), s->instances.end(),
                                          [&](const std::unique_ptr<Instance>& p) { return p.get() == i; }),
                           s->instances.end());
    }
    return true;
}

// a new instance of template t (device copies of the template's setup), or nullptr when the
// budget does not allow one even after evicting idle instances of other templates
Instance* makeInstance(hvvr_server* s, uint32_t t) {
    Template& tp = s->templates[t];
    if (!evictFor(s, t, tp.instBytes)) return nullptr;
    auto inst = std::make_unique<Instance>();
    hvvr_camera* cam = nullptr;
    if (cloneCamera(tp.proto, &cam) != HVVR_OK) return nullptr;
    cam->hidden = true;
    inst->cam = cam;
    inst->tmpl = t;
    inst->width = tp.width;
    inst->height = tp.height;
    if (inst->image.alloc(size_t(tp.width) * tp.height) != HVVR_OK) {
        hvvr_camera_destroy(cam->rc, cam);
        return nullptr;
    }
    inst->bytes = tp.instBytes;
    s->memUsed += inst->bytes;
    s->memPeak = std::max(s->memPeak, s->memUsed);
    Instance* raw = inst.get();
    s->instances.push_back(std::move(inst));
    return raw;
}

// an idle instance of template t, else a new one; nullptr when the budget is exhausted
Instance* takeInstance(hvvr_server* s, uint32_t t) {
    Template& tp = s->templates[t];
    if (!tp.freeList.empty()) {
        Instance* i = tp.freeList.back();
        tp.freeList.pop_back();
        return i;
    }
    return makeInstance(s, t);
}

void complete(hvvr_server* s, Request* r, int status) {
    r->status = status;
    r->doneMs = s->nowMs();
    hvvr_completion c{};
    c.id = r->id;
    c.tag = r->r.tag;
    c.status = status;
    c.submit_ms = r->submitMs;
    c.dispatch_ms = r->dispatchMs;
    c.done_ms = r->doneMs;
    c.batch_views = r->batchViews;
    c.priority = r->r.priority;
    std::lock_guard<std::mutex> lock(s->mu);
    s->completions.push_back(c);
    if (status == HVVR_OK) s->stats.completed++;
    else s->stats.failed++;
    s->stats.in_flight--;
    s->live.erase(r->id);
    s->doneCv.notify_all();
}

void finishSlot(hvvr_server* s, Slot& sl) {
    const int st = checkStatus(sl.batch.get());
    float gpuMs = 0.0f;
    if (cudaEventElapsedTime(&gpuMs, sl.batch->ev[0], sl.batch->ev[5]) == cudaSuccess) {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stats.batch_gpu_ms += gpuMs;
    }
    for (Request* r : sl.reqs) {
        Instance* in = r->inst;
        if (st == HVVR_OK && r->r.memory_type == HVVR_MEMORY_CPU)
            memcpy(r->r.output, in->staging, size_t(in->width) * in->height * 4);
        {
            // the template table may grow on other threads (hvvr_server_add_view)
            std::lock_guard<std::mutex> lock(s->mu);
            s->templates[in->tmpl].freeList.push_back(in);
        }
        complete(s, r, st);
    }
    sl.reqs.clear();
    sl.busy = false;
}

// applies staged vertex updates (no batch in flight) and refits the touched scenes
int applyUpdates(hvvr_server* s, std::vector<std::unique_ptr<Update>>& ups) {
    std::vector<hvvr_raycaster*> touched;
    for (auto& u : ups) {
        CUDA_TRY(cudaMemcpyAsync(u->rc->vertsIn.p + 2 * u->vertOffset, u->verts.p, size_t(u->count) * 32,
                                 cudaMemcpyDeviceToDevice, s->updateStream));
        if (std::find(touched.begin(), touched.end(), u->rc) == touched.end()) touched.push_back(u->rc);
    }
    for (hvvr_raycaster* rc : touched) {
        CUDA_TRY(launchRefit(rc->scene, rc->spec.fp_mode == HVVR_FP_FMA, s->updateStream));
        rc->refitDirty = false;
    }
    CUDA_TRY(cudaEventRecord(s->updateEv, s->updateStream));
    for (Slot& sl : s->slots) CUDA_TRY(cudaStreamWaitEvent(sl.stream, s->updateEv, 0));
    CUDA_TRY(cudaStreamSynchronize(s->updateStream)); // staging buffers are released after this
    return HVVR_OK;
}

// whether slot sl may render request r: a latency slot takes the latency class only; a throughput
// slot takes the throughput class, and the latency class too when the server has no latency slots
bool slotTakes(const hvvr_server* s, const Slot& sl, const Request* r) {
    const bool urgent = r->r.priority != 0;
    if (sl.latency) return urgent;
    return !urgent || s->cfg.latency_slots == 0;
}

// forms and launches one batch on slot sl from the pending requests (latency class first, then in
// arrival order); false if none admitted
bool dispatch(hvvr_server* s, Slot& sl) {
    std::vector<Request*> take;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        std::stable_partition(s->pending.begin(), s->pending.end(), [](const Request* r) { return r->r.priority != 0; });
        for (auto it = s->pending.begin(); it != s->pending.end() && take.size() < s->cfg.max_batch_views;) {
            Request* r = *it;
            if (!slotTakes(s, sl, r)) {
                ++it;
                continue;
            }
            Instance* in = takeInstance(s, r->r.view);
            if (!in) {
                ++it;
                continue;
            }
            r->inst = in;
            take.push_back(r);
            it = s->pending.erase(it);
        }
        s->stats.queued = s->pending.size();
    }
    if (take.empty()) return false;
    const double hostStart = s->nowMs();
    hvvr_batch* b = sl.batch.get();
    // frame buffers sized once for the largest batch the templates allow, so that no batch
    // reallocates (a free synchronises the device behind the other slots)
    size_t tmplCount = 0, maxTiles = 0;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        tmplCount = s->templates.size();
        for (const Template& t : s->templates) maxTiles = std::max<size_t>(maxTiles, t.proto->dev.tiles);
    }
    if (s->reservedFor != tmplCount) {
        const size_t tiles = maxTiles * s->cfg.max_batch_views;
        for (Slot& o : s->slots)
            if (!o.busy || &o == &sl) {
                if (reserveBatch(o.batch.get(), tiles, tiles / kTilesPerBlock, s->cfg.max_batch_views) != HVVR_OK)
                    break;
            }
        bool all = true;
        for (Slot& o : s->slots) all = all && o.batch->order.n >= tiles;
        if (all) s->reservedFor = tmplCount;
    }
    b->cams.clear();
    const double now = s->nowMs();
    for (Request* r : take) {
        Instance* in = r->inst;
        hvvr_camera* c = in->cam;
        const Instance& tp = *in; // width and height of the template
        if (r->r.memory_type == HVVR_MEMORY_CPU && !in->staging &&
            cudaMallocHost((void**)&in->staging, size_t(tp.width) * tp.height * 4) != cudaSuccess) {
            cudaGetLastError();
            in->staging = nullptr;
        }
        c->xf = r->r.camera_to_world;
        c->msaa = r->r.msaa;
        uint32_t* img = r->r.memory_type == HVVR_MEMORY_CUDA ? static_cast<uint32_t*>(r->r.output) : in->image.p;
        c->target.memory_type = HVVR_MEMORY_CUDA;
        c->target.data = img;
        c->target.width = tp.width;
        c->target.height = tp.height;
        c->target.stride = tp.width;
        c->dev.image = img;
        c->dev.imageStride = tp.width;
        if (c->foveated) {
            // the resolve writes this request's image, and a request is one frame: no history
            // from whichever request this instance served before
            c->fovStatic.image = img;
            c->fovStatic.imageStride = tp.width;
            resetFoveatedHistory(c);
        }
        b->cams.push_back(c);
        r->dispatchMs = now;
        r->batchViews = uint32_t(take.size());
    }
    int rc = renderBatch(b, sl.stream, true);
    if (rc == HVVR_OK) {
        for (Request* r : take) {
            if (r->r.memory_type != HVVR_MEMORY_CPU) continue;
            const Instance& tp = *r->inst;
            if (!r->inst->staging) {
                rc = fail(HVVR_ERR_OOM, "pinned staging allocation failed");
                break;
            }
            if (cudaMemcpyAsync(r->inst->staging, r->inst->image.p, size_t(tp.width) * tp.height * 4,
                                cudaMemcpyDeviceToHost, sl.stream) != cudaSuccess)
                rc = fail(HVVR_ERR_CUDA, "output copy failed");
        }
    }
    if (rc == HVVR_OK && cudaEventRecord(sl.done, sl.stream) != cudaSuccess) rc = fail(HVVR_ERR_CUDA, "event record failed");
    if (rc != HVVR_OK) {
        cudaStreamSynchronize(sl.stream);
        for (Request* r : take) {
            {
                std::lock_guard<std::mutex> lock(s->mu);
                s->templates[r->inst->tmpl].freeList.push_back(r->inst);
            }
            complete(s, r, rc);
        }
        return true;
    }
    sl.reqs = take;
    sl.busy = true;
    std::lock_guard<std::mutex> lock(s->mu);
    s->stats.dispatch_host_ms += s->nowMs() - hostStart;
    s->stats.batches++;
    s->viewsDispatched += take.size();
    return true;
}

void workerLoop(hvvr_server* s) {
    cudaSetDevice(s->scenes[0]->spec.device);
    std::vector<std::unique_ptr<Update>> ups;
    for (;;) {
        bool progress = false;
        for (Slot& sl : s->slots) {
            if (sl.busy && cudaEventQuery(sl.done) == cudaSuccess) {
                finishSlot(s, sl);
                progress = true;
            }
        }
        {
            std::lock_guard<std::mutex> lock(s->mu);
            if (s->stop) break;
            for (auto& u : s->updates) ups.push_back(std::move(u));
            s->updates.clear();
        }
        bool anyBusy = false;
        for (Slot& sl : s->slots) anyBusy = anyBusy || sl.busy;
        if (!ups.empty()) {
            if (!anyBusy) {
                if (applyUpdates(s, ups) != HVVR_OK) {
                    std::lock_guard<std::mutex> lock(s->mu);
                    s->workerError = hvvr_last_error();
                }
                ups.clear();
                progress = true;
            }
        } else {
            // latency slots first: a latency-class request goes out as soon as one is free
            for (Slot& sl : s->slots) {
                if (sl.busy || !sl.latency) continue;
                if (dispatch(s, sl)) progress = true;
                else break;
            }
            for (Slot& sl : s->slots) {
                if (sl.busy || sl.latency) continue;
                // an idle GPU takes any request; with a batch in flight, gather a fuller batch
                // unless the oldest request has waited max_wait_ms
                bool busyNow = false;
                for (const Slot& o : s->slots) busyNow = busyNow || (o.busy && !o.latency);
                if (busyNow) {
                    std::lock_guard<std::mutex> lock(s->mu);
                    size_t eligible = 0;
                    double oldest = -1.0;
                    for (const Request* r : s->pending)
                        if (slotTakes(s, sl, r)) {
                            if (oldest < 0.0) oldest = r->submitMs;
                            eligible++;
                        }
                    if (!eligible) break;
                    const double waited = s->nowMs() - oldest;
                    if (eligible < s->cfg.min_batch_views && waited < s->cfg.max_wait_ms) break;
                }
                if (dispatch(s, sl)) progress = true;
                else break;
            }
        }
        if (!progress) {
            std::unique_lock<std::mutex> lock(s->mu);
            s->workCv.wait_for(lock, std::chrono::microseconds(50));
        }
    }
    for (Slot& sl : s->slots)
        if (sl.busy) {
            cudaEventSynchronize(sl.done);
            finishSlot(s, sl);
        }
}

} // namespace

extern "C" {

void hvvr_server_config_default(hvvr_server_config* cfg) {
    if (!cfg) return;
    memset(cfg, 0, sizeof(*cfg));
    cfg->hbm_budget_bytes = 120ull << 30;
    cfg->slots = 2;
    cfg->max_batch_views = 64;
    cfg->slot_list_capacity = 256ull << 20;
    cfg->tile_cull_warps = 4;
    cfg->heavy_divisor = 8;
    cfg->min_batch_views = 8;
    cfg->max_wait_ms = 2.0f;
    cfg->latency_slots = 1;
    cfg->tile_cull_ctas_per_sm = 0;
    cfg->latency_isolation = 1;
}

int hvvr_server_create(hvvr_raycaster* const* scenes, uint32_t count, const hvvr_server_config* cfg,
                       hvvr_server** out) {
    if (!out) return fail(HVVR_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!scenes || count == 0) return fail(HVVR_ERR_INVALID, "no scenes");
    auto s = std::make_unique<hvvr_server>();
    hvvr_server_config_default(&s->cfg);
    if (cfg) s->cfg = *cfg;
    if (s->cfg.slots < 1 || s->cfg.slots > 8) return fail(HVVR_ERR_INVALID, "slots must be 1..8");
    if (s->cfg.latency_slots > 4) return fail(HVVR_ERR_INVALID, "latency_slots must be 0..4");
    if (s->cfg.max_batch_views < 1) return fail(HVVR_ERR_INVALID, "max_batch_views must be >= 1");
    if (s->cfg.latency_isolation > 1) return fail(HVVR_ERR_INVALID, "latency_isolation must be 0 or 1");
    for (uint32_t i = 0; i < count; i++) {
        hvvr_raycaster* rc = scenes[i];
        if (!rc) return fail(HVVR_ERR_INVALID, "NULL scene %u", i);
        if (rc->spec.device != scenes[0]->spec.device || rc->spec.fp_mode != scenes[0]->spec.fp_mode)
            return fail(HVVR_ERR_INVALID, "served scenes must share one device and fp_mode");
        s->scenes.push_back(rc);
    }
    CUDA_TRY(cudaSetDevice(scenes[0]->spec.device));
    // scenes resident and refit before the first request
    for (hvvr_raycaster* rc : s->scenes) {
        if (rc->sceneDirty) {
            TRY(uploadScene(rc, rc->stream));
            rc->sceneDirty = false;
            rc->refitDirty = true;
        }
        if (rc->scene.nodeCount && rc->refitDirty) {
            CUDA_TRY(launchRefit(rc->scene, rc->spec.fp_mode == HVVR_FP_FMA, rc->stream));
            rc->refitDirty = false;
        }
        CUDA_TRY(cudaStreamSynchronize(rc->stream));
    }
    for (uint32_t rate : {1u, 2u, 4u, 8u, 16u, 32u}) TRY(ensureMsaaTable(rate, s->scenes[0]->stream));
    hvvr_batch_config bc;
    batchConfigDefault(&bc);
    bc.use_graph = 0; // every batch has its own mix of views
    bc.tile_cull_warps = s->cfg.tile_cull_warps;
    bc.heavy_divisor = s->cfg.heavy_divisor;
    bc.tri_index_capacity = s->cfg.slot_list_capacity;
    TRY(checkConfig(bc));
    int leastPriority = 0, greatestPriority = 0;
    CUDA_TRY(cudaDeviceGetStreamPriorityRange(&leastPriority, &greatestPriority));
    const uint32_t slotCount = s->cfg.slots + s->cfg.latency_slots;
    s->slots.resize(slotCount);
    for (uint32_t i = 0; i < slotCount; i++) {
        Slot& sl = s->slots[i];
        sl.latency = i >= s->cfg.slots;
        sl.batch = std::make_unique<hvvr_batch>();
        sl.batch->cfg = bc;
        // throughput slots leave SMs free for latency-class launches when asked to
        if (!sl.latency) sl.batch->cfg.tile_cull_ctas_per_sm = s->cfg.tile_cull_ctas_per_sm;
        // and, isolated, hold no SM slot for longer than one tile and never wait on another CTA: the
        // block scheduler then hands every slot they free to the latency class's launches first
        if (!sl.latency && s->cfg.latency_slots && s->cfg.latency_isolation) {
            sl.batch->cfg.tile_cull_persistent = 0;
            sl.batch->cfg.pipeline = 0;
            // no heavy-part split (a single frame's latency device, not a batch's): one stream per
            // rate class, so that all slots' streams fit the hardware work queues
            sl.batch->cfg.heavy_divisor = 0;
        }
        sl.batch->fixedViews = true;
        sl.batch->internal = true;
        sl.batch->rcs = s->scenes;
        // with latency slots, their launches go ahead of the throughput slots' pending CTAs
        sl.batch->streamPriorities = s->cfg.latency_slots == 0 ? 0 : (sl.latency ? 1 : 2);
        const int prio = s->cfg.latency_slots == 0 ? leastPriority : (sl.latency ? greatestPriority : leastPriority);
        CUDA_TRY(cudaStreamCreateWithPriority(&sl.stream, cudaStreamNonBlocking, prio));
        CUDA_TRY(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
    }
    CUDA_TRY(cudaStreamCreateWithFlags(&s->updateStream, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&s->updateEv, cudaEventDisableTiming));
    s->poolBytes = size_t(slotCount) * size_t(bc.tri_index_capacity) * 4 * (kChunk + 1) / kChunk;
    if (s->poolBytes > s->cfg.hbm_budget_bytes)
        return fail(HVVR_ERR_INVALID, "the slots' triangle-list pools alone exceed the HBM budget");
    s->memUsed = s->poolBytes;
    s->memPeak = s->memUsed;
    hvvr_server* raw = s.release();
    raw->worker = std::thread(workerLoop, raw);
    *out = raw;
    return HVVR_OK;
}

int hvvr_server_destroy(hvvr_server* s) {
    if (!s) return fail(HVVR_ERR_INVALID, "NULL server");
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
        s->workCv.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->scenes[0]->spec.device);
    cudaDeviceSynchronize();
    for (Slot& sl : s->slots) {
        if (sl.batch) releaseBatch(sl.batch.get());
        if (sl.stream) cudaStreamDestroy(sl.stream);
        if (sl.done) cudaEventDestroy(sl.done);
    }
    // instance and prototype cameras go back to their raycasters and are destroyed there
    for (auto& in : s->instances) {
        if (in->staging) cudaFreeHost(in->staging);
        hvvr_camera_destroy(in->cam->rc, in->cam);
    }
    for (Template& t : s->templates) hvvr_camera_destroy(t.rc, t.proto);
    if (s->updateStream) cudaStreamDestroy(s->updateStream);
    if (s->updateEv) cudaEventDestroy(s->updateEv);
    delete s;
    return HVVR_OK;
}

int hvvr_server_add_view(hvvr_server* s, uint32_t scene, const hvvr_float_rect* viewport, const hvvr_sample* samples,
                         uint32_t count, uint32_t split, uint32_t width, uint32_t height, uint32_t* view_id) {
    if (!s || !viewport || !samples || !view_id) return fail(HVVR_ERR_INVALID, "NULL argument");
    if (scene >= s->scenes.size()) return fail(HVVR_ERR_INVALID, "scene %u out of range", scene);
    if (!width || !height) return fail(HVVR_ERR_INVALID, "empty output image");
    hvvr_raycaster* rc = s->scenes[scene];
    hvvr_camera* cam = nullptr;
    // the worker thread may be cloning cameras of this raycaster: serialise with it
    std::lock_guard<std::mutex> lock(s->mu);
    TRY(hvvr_camera_create(rc, viewport, 0.0f, &cam));
    cam->hidden = true;
    hvvr_image_desc d{};
    d.pixel_format = HVVR_PIXEL_RGBA8_SRGB;
    d.memory_type = HVVR_MEMORY_CUDA;
    d.width = width;
    d.height = height;
    cam->target = d;
    int r = hvvr_camera_set_samples(cam, samples, count, split);
    if (r == HVVR_OK) r = setupCamera(cam, rc->stream);
    if (r == HVVR_OK && cudaStreamSynchronize(rc->stream) != cudaSuccess) r = fail(HVVR_ERR_CUDA, "setup failed");
    if (r != HVVR_OK) {
        hvvr_camera_destroy(rc, cam);
        return r;
    }
    Template t;
    t.rc = rc;
    t.proto = cam;
    t.width = width;
    t.height = height;
    t.samples = count;
    t.instBytes = cameraBytes(cam, 1) + size_t(width) * height * 4;
    s->templates.push_back(t);
    *view_id = uint32_t(s->templates.size() - 1);
    return HVVR_OK;
}

int hvvr_server_prewarm(hvvr_server* s, uint32_t view, uint32_t count) {
    if (!s) return fail(HVVR_ERR_INVALID, "NULL server");
    std::lock_guard<std::mutex> lock(s->mu);
    if (view >= s->templates.size()) return fail(HVVR_ERR_INVALID, "unknown view %u", view);
    Template& tp = s->templates[view];
    while (tp.freeList.size() < count) {
        if (s->memUsed + tp.instBytes > s->cfg.hbm_budget_bytes)
            return fail(HVVR_ERR_OOM, "HBM budget reached after %zu instances", tp.freeList.size());
        Instance* in = makeInstance(s, view);
        if (!in) return fail(HVVR_ERR_OOM, "could not make an instance");
        tp.freeList.push_back(in);
    }
    return HVVR_OK;
}

namespace {

// the checks of one request; the template checks need the server lock held
int checkRequest(const hvvr_server* s, const hvvr_request* req) {
    if (!req) return fail(HVVR_ERR_INVALID, "NULL request");
    if (req->memory_type != HVVR_MEMORY_CPU && req->memory_type != HVVR_MEMORY_CUDA)
        return fail(HVVR_ERR_INVALID, "output must be CPU or CUDA memory");
    if (!req->output) return fail(HVVR_ERR_INVALID, "NULL output");
    if (req->msaa != 1 && req->msaa != 2 && req->msaa != 4 && req->msaa != 8 && req->msaa != 16 && req->msaa != 32)
        return fail(HVVR_ERR_INVALID, "MSAA rate must be 1, 2, 4, 8, 16 or 32");
    if (req->priority > 1) return fail(HVVR_ERR_INVALID, "priority must be 0 (throughput) or 1 (latency)");
    if (req->view >= s->templates.size()) return fail(HVVR_ERR_INVALID, "unknown view %u", req->view);
    if (s->templates[req->view].instBytes + s->poolBytes > s->cfg.hbm_budget_bytes)
        return fail(HVVR_ERR_OOM, "one view of this template exceeds the HBM budget");
    return HVVR_OK;
}

// queues checked requests (server lock held) and wakes the worker once
void enqueueRequests(hvvr_server* s, const hvvr_request* reqs, uint32_t count, uint64_t* ids) {
    const double now = s->nowMs();
    for (uint32_t i = 0; i < count; i++) {
        auto r = std::make_unique<Request>();
        r->id = s->nextId++;
        r->r = reqs[i];
        r->submitMs = now;
        if (ids) ids[i] = r->id;
        s->pending.push_back(r.get());
        s->live[r->id] = std::move(r);
        s->stats.submitted++;
        s->stats.in_flight++;
    }
    s->stats.queued = s->pending.size();
    s->workCv.notify_all();
}

} // namespace

int hvvr_server_submit(hvvr_server* s, const hvvr_request* req, uint64_t* id) {
    if (!s || !req) return fail(HVVR_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lock(s->mu);
    TRY(checkRequest(s, req));
    enqueueRequests(s, req, 1, id);
    return HVVR_OK;
}

int hvvr_server_submit_group(hvvr_server* s, const hvvr_request* reqs, uint32_t count, uint64_t* ids) {
    if (!s || (count && !reqs)) return fail(HVVR_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lock(s->mu);
    for (uint32_t i = 0; i < count; i++) TRY(checkRequest(s, reqs + i));
    enqueueRequests(s, reqs, count, ids);
    return HVVR_OK;
}

int hvvr_server_poll(hvvr_server* s, hvvr_completion* out, uint32_t capacity, uint32_t* count, double wait_ms) {
    if (!s || !count || (capacity && !out)) return fail(HVVR_ERR_INVALID, "NULL argument");
    std::unique_lock<std::mutex> lock(s->mu);
    if (s->completions.empty() && wait_ms > 0)
        s->doneCv.wait_for(lock, std::chrono::duration<double, std::milli>(wait_ms),
                           [&] { return !s->completions.empty(); });
    uint32_t n = 0;
    while (n < capacity && !s->completions.empty()) {
        out[n++] = s->completions.front();
        s->completions.pop_front();
    }
    *count = n;
    if (!s->workerError.empty()) return fail(HVVR_ERR_CUDA, "server worker: %s", s->workerError.c_str());
    return HVVR_OK;
}

int hvvr_server_update_vertices(hvvr_server* s, hvvr_model* model, uint32_t first, uint32_t count,
                                const void* device_verts) {
    if (!s || !model || (count && !device_verts)) return fail(HVVR_ERR_INVALID, "NULL argument");
    hvvr_raycaster* rc = model->rc;
    if (std::find(s->scenes.begin(), s->scenes.end(), rc) == s->scenes.end())
        return fail(HVVR_ERR_INVALID, "model is not in a served scene");
    if (uint64_t(first) + count > model->verts.size()) return fail(HVVR_ERR_INVALID, "vertex range out of bounds");
    auto u = std::make_unique<Update>();
    u->rc = rc;
    size_t off = 0;
    for (auto& m : rc->models) {
        if (m.get() == model) break;
        off += m->verts.size();
    }
    u->vertOffset = off + first;
    u->count = count;
    TRY(u->verts.alloc(size_t(count) * 2));
    CUDA_TRY(cudaMemcpy(u->verts.p, device_verts, size_t(count) * 32, cudaMemcpyDeviceToDevice));
    std::lock_guard<std::mutex> lock(s->mu);
    s->updates.push_back(std::move(u));
    s->workCv.notify_all();
    return HVVR_OK;
}

int hvvr_server_get_stats(hvvr_server* s, hvvr_server_stats* out) {
    if (!s || !out) return fail(HVVR_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lock(s->mu);
    *out = s->stats;
    out->instances = s->instances.size();
    out->hbm_used = s->memUsed;
    out->hbm_peak = s->memPeak;
    out->mean_batch_views = s->stats.batches ? double(s->viewsDispatched) / double(s->stats.batches) : 0.0;
    return HVVR_OK;
}

} // extern "C"
