// evxg_serve.cu -- serving: a request loop over many live streams.
//
// No counterpart in the reference, which encodes one stream per
// evx3_encoder.  Streams are admitted by a device-memory budget and keep all
// their state (DPB slots, tables, levels, SAO state) on the device while they
// live.  Callers submit RGB frames as they arrive; each stream's GOP logic is
// the reference encoder's (evx3enc.cpp:105-414, the same planner evxg_encoder
// runs), so a frame becomes ready to encode once the frames it depends on
// have arrived.  Streams are spread over lanes -- a stream joins the lane
// whose streams are closest to its size -- and each lane has its own worker
// thread, CUDA stream and batch: the worker batches whatever of its streams'
// frames is ready -- at most one frame per stream per tick -- into batched
// ticks (evxg_batch.cu), building tick t+1 while tick t runs, and delivers
// every frame's serializer inputs, with its arrival / ready / launch / done
// times, through a callback.  Lanes tick independently and their ticks run
// on the device side by side (their streams are disjoint and each tick's
// persistent kernels claim only their own rows), so a small stream's frame
// does not wait for a large stream's wavefront.  Streams that join or leave
// change their lane's batch at its next tick boundary; the others' device
// state is untouched.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "evxg_internal.cuh"

using namespace evxg;

namespace {

uint64_t now_ns()
{
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Device memory a stream holds (evxg_stream_create's allocations).
size_t stream_bytes(uint32_t w, uint32_t h)
{
    const size_t W = (w + 15) & ~15u, H = (h + 15) & ~15u, nblk = (W / 16) * (H / 16);
    const size_t planeset = (W * H + 2 * (W / 2) * (H / 2)) * sizeof(int16_t);
    return 7 * planeset + (size_t)w * h * 3 + nblk * (3 * sizeof(evxg_block_desc) + sizeof(evxg_sao_info) + 8 + kSaoStatEntries * sizeof(int2)) +
           (3 * (H / 16) + 5) * sizeof(int) + kSaoPasses * sizeof(int);
}

struct Ready {
    std::vector<uint8_t> px;
    evxg_frame f;
    evxg_frame_times t;
};

struct Slot {
    uint32_t id = 0, w = 0, h = 0;
    int lane = 0;
    size_t bytes = 0;
    evxg_stream *st = nullptr;
    evxg_encoder *planner = nullptr;
    std::deque<Ready> ready;                   // frames whose encode order is known, oldest first
    std::map<uint32_t, uint64_t> arrival;      // arrival stamp by display order, until the frame is ready
    uint32_t next_order = 0;
    bool closing = false;                      // no more input; removed once drained
    int in_flight = 0;                         // frames in ticks not yet delivered
    evxg_config cfg{};                         // the build the stream reproduces
    // Evicted: the device state lives in `saved` (evxg_stream_save), st is
    // gone, its memory is back in the budget; the planner stays.
    bool evicted = false;
    std::vector<uint8_t> saved;
};

}  // namespace

struct Pending {
    bool used = false;
    std::vector<Ready> frames;                 // per batch index; f.type < 0 = none
};

// One lane: a set of streams with its own worker thread, CUDA stream and batch.
struct Lane {
    int index = 0;
    bool set_dirty = true;                     // its stream set changed (under the server lock)
    // worker-owned
    evxg_batch *batch = nullptr;
    std::vector<Slot *> bslots;                // batch order
    Pending pend[2];
    cudaStream_t cs = nullptr;
    std::thread worker;
};

struct evxg_server {
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::map<uint32_t, Slot *> slots;
    uint32_t next_id = 1, max_streams = 0;
    uint64_t budget = 0, used = 0;
    evxg_result_callback cb = nullptr;
    void *user = nullptr;
    std::vector<Lane *> lanes;
    bool stop = false;
    int drainers = 0;                          // threads waiting in evxg_server_drain
    int error = 0;
    uint64_t frames_done = 0, ticks = 0, rebuilds = 0;
    int device = 0;
};

namespace {

// Planner sink: the frame's encode order is known (called under the lock).
int sink(void *ctx, const uint8_t *rgb, uint32_t w, uint32_t h, const evxg_frame *f)
{
    Slot *s = static_cast<Slot *>(ctx);
    Ready r;
    r.px.assign(rgb, rgb + (size_t)w * h * 3);
    r.f = *f;
    auto it = s->arrival.find(f->display_order);
    r.t.arrival_ns = it != s->arrival.end() ? it->second : 0;
    if (it != s->arrival.end()) s->arrival.erase(it);
    r.t.ready_ns = now_ns();
    r.t.launch_ns = r.t.done_ns = 0;
    s->ready.push_back(std::move(r));
    return EVXG_SUCCESS;
}

bool drained(const Slot *s) { return s->ready.empty() && s->in_flight == 0; }
// Closed streams that have delivered everything stay in the batch (without
// frames) until the next rebuild, which a new stream's admission brings; until
// then their memory counts as free for admissions.
size_t dead_bytes(const evxg_server *v)
{
    size_t b = 0;
    for (auto &kv : v->slots)
        if (kv.second->closing && drained(kv.second)) b += kv.second->bytes;
    return b;
}

// Deliver lane l's tick q's results (its worker thread, without the lock).
int complete(evxg_server *v, Lane *l, int q)
{
    Pending &pd = l->pend[q];
    if (!pd.used) return EVXG_SUCCESS;
    pd.used = false;
    int rc = evxg_batch_wait(l->batch, (uint32_t)q);
    const uint64_t done = now_ns();
    for (size_t i = 0; i < pd.frames.size() && !rc; i++) {
        Ready &r = pd.frames[i];
        if (r.f.type < 0) continue;
        r.t.done_ns = done;
        const evxg_block_desc *bt, *pv;
        const evxg_sao_info *sao;
        const int16_t *lev;
        rc = evxg_batch_output(l->batch, (uint32_t)i, (uint32_t)q, &bt, &pv, &sao, &lev);
        if (!rc && v->cb) v->cb(v->user, l->bslots[i]->id, &r.f, bt, pv, sao, lev, &r.t);
    }
    std::lock_guard<std::mutex> lk(v->mu);
    for (size_t i = 0; i < pd.frames.size(); i++)
        if (pd.frames[i].f.type >= 0) { l->bslots[i]->in_flight--; v->frames_done++; }
    if (rc && !v->error) v->error = rc;
    pd.frames.clear();
    v->cv_done.notify_all();
    return rc;
}

}  // namespace

namespace {

// Worker of lane l: rebuild the lane's batch when its stream set changed
// (with no tick in flight), launch a tick of whatever is ready, then deliver
// the tick before it.
void work(evxg_server *v, Lane *l)
{
    cudaSetDevice(v->device);   // the caller's device
    int p = 0;
    for (;;) {
        std::unique_lock<std::mutex> lk(v->mu);
        auto any_ready = [&] {
            for (auto &kv : v->slots)
                if (kv.second->lane == l->index && !kv.second->evicted && !kv.second->ready.empty()) return true;
            return false;
        };
        v->cv_work.wait(lk, [&] {
            // a changed stream set is rebuilt when there is work for it or a drain waits on it, so a
            // burst of admissions costs one rebuild
            return v->stop || (l->set_dirty && v->drainers > 0) || any_ready() || l->pend[0].used || l->pend[1].used;
        });
        if (v->error) {   // a tick failed: deliver nothing more, let callers see the error
            v->cv_done.notify_all();
            if (v->stop) break;
            v->cv_work.wait(lk, [&] { return v->stop; });
            break;
        }
        if (v->stop && !any_ready() && !l->pend[0].used && !l->pend[1].used) break;
        if (l->set_dirty) {
            if (l->pend[0].used || l->pend[1].used) {   // finish the batch's ticks first, oldest first
                lk.unlock();
                complete(v, l, p ^ 1);
                complete(v, l, p);
                continue;
            }
            for (auto it = v->slots.begin(); it != v->slots.end();) {
                Slot *s = it->second;
                if (s->lane == l->index && s->closing && drained(s)) {
                    evxg_encoder_destroy(s->planner);
                    if (s->st) evxg_stream_destroy(s->st);
                    v->used -= s->bytes;
                    delete s;
                    it = v->slots.erase(it);
                } else {
                    ++it;
                }
            }
            if (l->batch) { evxg_batch_destroy(l->batch); l->batch = nullptr; }
            l->bslots.clear();
            std::vector<evxg_stream *> sts;
            for (auto &kv : v->slots)
                if (kv.second->lane == l->index && !kv.second->evicted) {
                    l->bslots.push_back(kv.second);
                    sts.push_back(kv.second->st);
                }
            if (!sts.empty()) {
                const int rc = evxg_batch_create(sts.data(), (uint32_t)sts.size(), &l->batch);
                if (rc) { v->error = rc; continue; }   // the batch's default shape: its tick model (evxg_batch.cu)
            }
            l->set_dirty = false;
            v->rebuilds++;
            p = 0;
            v->cv_done.notify_all();
            continue;
        }
        // a tick of whatever is ready: at most one frame per stream, its oldest
        std::vector<Ready> frames(l->bslots.size());
        bool any = false;
        for (size_t i = 0; i < l->bslots.size(); i++) {
            Slot *s = l->bslots[i];
            if (s->ready.empty()) { frames[i].f.type = -1; continue; }
            frames[i] = std::move(s->ready.front());
            s->ready.pop_front();
            s->in_flight++;
            any = true;
        }
        lk.unlock();
        if (!any) {   // nothing new: deliver what is in flight
            complete(v, l, p ^ 1);
            complete(v, l, p);
            continue;
        }
        if (complete(v, l, p)) continue;   // this parity's buffers are free again
        std::vector<evxg_frame> fr(frames.size());
        const uint64_t launch = now_ns();
        for (size_t i = 0; i < frames.size(); i++) {
            fr[i] = frames[i].f;
            if (frames[i].f.type < 0) continue;
            memcpy(evxg_batch_input(l->batch, (uint32_t)i, (uint32_t)p), frames[i].px.data(), frames[i].px.size());
            frames[i].t.launch_ns = launch;
            frames[i].px.clear();
            frames[i].px.shrink_to_fit();
        }
        int rc = evxg_batch_encode(l->batch, fr.data(), (uint32_t)p, l->cs);
        {
            std::lock_guard<std::mutex> g(v->mu);
            if (rc && !v->error) v->error = rc;
            v->ticks++;
        }
        if (rc) continue;
        l->pend[p].used = true;
        l->pend[p].frames = std::move(frames);
        complete(v, l, p ^ 1);   // the tick before runs ahead of this one; deliver it while this one runs
        p ^= 1;
    }
    complete(v, l, p ^ 1);
    complete(v, l, p);
}

// The lane a new stream of w x h joins: an empty lane while there is one (a
// stream alone in its lane is launched as soon as its frame arrives), else
// the least loaded lane whose streams have the closest size (macroblock count
// within a factor of two), else the one with the fewest macroblocks.
int pick_lane(const evxg_server *v, uint32_t w, uint32_t h)
{
    const size_t n = v->lanes.size();
    std::vector<double> load(n, 0.0), closest(n, 1e30);
    const double mbs = (double)((w + 15) / 16) * ((h + 15) / 16);
    for (const auto &kv : v->slots) {
        const Slot *s = kv.second;
        if (s->closing && drained(s)) continue;
        const double m = (double)((s->w + 15) / 16) * ((s->h + 15) / 16);
        load[s->lane] += m;
        const double r = m > mbs ? m / mbs : mbs / m;
        closest[s->lane] = std::min(closest[s->lane], r);
    }
    for (size_t i = 0; i < n; i++)
        if (load[i] == 0.0) return (int)i;
    int best = -1;
    for (size_t i = 0; i < n; i++)   // same size class, least loaded
        if (closest[i] < 2.0 && (best < 0 || load[i] < load[best])) best = (int)i;
    if (best >= 0) return best;
    best = 0;
    for (size_t i = 1; i < n; i++)
        if (load[i] < load[best]) best = (int)i;
    return best;
}

}  // namespace

extern "C" {

uint64_t evxg_server_now_ns(void) { return now_ns(); }

int evxg_server_create(uint64_t hbm_budget_bytes, uint32_t max_streams, evxg_result_callback cb, void *user,
                       evxg_server **out)
{
    return evxg_server_create_lanes(hbm_budget_bytes, max_streams, max_streams < 8 ? max_streams : 8, cb, user, out);
}

int evxg_server_create_lanes(uint64_t hbm_budget_bytes, uint32_t max_streams, uint32_t lanes, evxg_result_callback cb,
                             void *user, evxg_server **out)
{
    if (!out || !max_streams || !hbm_budget_bytes || !lanes || lanes > max_streams)
        return fail(EVXG_ERROR_INVALIDARG, "evxg_server_create: bad argument");
    evxg_server *v = new evxg_server();
    v->budget = hbm_budget_bytes;
    v->max_streams = max_streams;
    v->cb = cb;
    v->user = user;
    bool ok = cudaGetDevice(&v->device) == cudaSuccess;
    for (uint32_t i = 0; i < lanes && ok; i++) {
        Lane *l = new Lane();
        l->index = (int)i;
        v->lanes.push_back(l);
        ok = cudaStreamCreateWithFlags(&l->cs, cudaStreamNonBlocking) == cudaSuccess;
    }
    if (!ok) {
        for (Lane *l : v->lanes) {
            if (l->cs) cudaStreamDestroy(l->cs);
            delete l;
        }
        delete v;
        return fail(EVXG_ERROR_EXECUTION_FAILURE, "evxg_server_create: stream creation failed");
    }
    for (Lane *l : v->lanes) l->worker = std::thread(work, v, l);
    *out = v;
    return EVXG_SUCCESS;
}

int evxg_server_open(evxg_server *v, uint32_t width, uint32_t height, uint8_t quality, uint32_t *stream_id)
{
    return evxg_server_open_config(v, width, height, quality, nullptr, stream_id);
}

int evxg_server_open_config(evxg_server *v, uint32_t width, uint32_t height, uint8_t quality, const evxg_config *cfg,
                            uint32_t *stream_id)
{
    if (!v || !stream_id) return fail(EVXG_ERROR_INVALIDARG, "evxg_server_open: bad argument");
    const size_t bytes = stream_bytes(width, height);
    {
        std::lock_guard<std::mutex> lk(v->mu);
        if (v->error) return fail(v->error, "evxg_server_open: the server has failed");
        size_t dead_slots = 0;
        for (auto &kv : v->slots) dead_slots += kv.second->closing && drained(kv.second);
        if (v->slots.size() - dead_slots >= v->max_streams)
            return fail(EVXG_ERROR_CAPACITY_LIMIT, "evxg_server_open: every stream slot is taken");
        if (v->used - dead_bytes(v) + bytes > v->budget)
            return fail(EVXG_ERROR_CAPACITY_LIMIT, "evxg_server_open: the device memory budget is spent");
        v->used += bytes;   // reserved while the stream is created
    }
    Slot *s = new Slot();
    s->w = width; s->h = height; s->bytes = bytes;
    evxg_config_default(&s->cfg);
    if (cfg) s->cfg = *cfg;
    int rc = evxg_stream_create_config(width, height, cfg, &s->st);
    if (!rc) rc = evxg_encoder_create_config(nullptr, nullptr, cfg, &s->planner);
    if (!rc) { encoder_set_sink(s->planner, sink, s); rc = evxg_encoder_set_quality(s->planner, quality); }
    std::lock_guard<std::mutex> lk(v->mu);
    if (rc) {
        if (s->planner) evxg_encoder_destroy(s->planner);
        if (s->st) evxg_stream_destroy(s->st);
        delete s;
        v->used -= bytes;
        return rc;
    }
    s->id = v->next_id++;
    s->lane = pick_lane(v, width, height);
    v->slots[s->id] = s;
    v->lanes[s->lane]->set_dirty = true;
    *stream_id = s->id;
    v->cv_work.notify_all();
    return EVXG_SUCCESS;
}

int evxg_server_submit(evxg_server *v, uint32_t stream_id, const uint8_t *rgb, uint64_t arrival_ns)
{
    if (!v || !rgb) return fail(EVXG_ERROR_INVALIDARG, "evxg_server_submit: bad argument");
    std::lock_guard<std::mutex> lk(v->mu);
    if (v->error) return fail(v->error, "evxg_server_submit: the server has failed");
    auto it = v->slots.find(stream_id);
    if (it == v->slots.end() || it->second->closing) return fail(EVXG_ERROR_INVALID_INDEX, "evxg_server_submit: no such open stream");
    Slot *s = it->second;
    if (s->evicted) return fail(EVXG_ERROR_NOT_READY, "evxg_server_submit: the stream is evicted (restore it first)");
    s->arrival[s->next_order++] = arrival_ns ? arrival_ns : now_ns();
    const int rc = evxg_encoder_encode(s->planner, rgb, s->w, s->h);
    v->cv_work.notify_all();
    return rc;
}

int evxg_server_insert_intra(evxg_server *v, uint32_t stream_id)
{
    if (!v) return EVXG_ERROR_INVALIDARG;
    std::lock_guard<std::mutex> lk(v->mu);
    auto it = v->slots.find(stream_id);
    if (it == v->slots.end() || it->second->closing) return fail(EVXG_ERROR_INVALID_INDEX, "evxg_server_insert_intra: no such open stream");
    if (it->second->evicted) return fail(EVXG_ERROR_NOT_READY, "evxg_server_insert_intra: the stream is evicted");
    return evxg_encoder_insert_intra(it->second->planner);
}

int evxg_server_close(evxg_server *v, uint32_t stream_id)
{
    if (!v) return EVXG_ERROR_INVALIDARG;
    std::lock_guard<std::mutex> lk(v->mu);
    auto it = v->slots.find(stream_id);
    if (it == v->slots.end() || it->second->closing) return fail(EVXG_ERROR_INVALID_INDEX, "evxg_server_close: no such open stream");
    if (it->second->evicted) return fail(EVXG_ERROR_NOT_READY, "evxg_server_close: the stream is evicted (restore or cancel it)");
    const int rc = evxg_encoder_flush(it->second->planner);   // the frames still waiting for their anchor
    it->second->closing = true;
    v->cv_work.notify_all();
    return rc;
}

int evxg_server_cancel(evxg_server *v, uint32_t stream_id)
{
    if (!v) return EVXG_ERROR_INVALIDARG;
    std::lock_guard<std::mutex> lk(v->mu);
    auto it = v->slots.find(stream_id);
    if (it == v->slots.end() || it->second->closing) return fail(EVXG_ERROR_INVALID_INDEX, "evxg_server_cancel: no such open stream");
    Slot *s = it->second;
    s->ready.clear();     // frames not yet in a tick are dropped; those in flight are delivered
    s->arrival.clear();
    s->closing = true;    // no flush: frames still waiting for their anchor are dropped too
    v->cv_work.notify_all();
    return EVXG_SUCCESS;
}

int evxg_server_evict(evxg_server *v, uint32_t stream_id)
{
    if (!v) return EVXG_ERROR_INVALIDARG;
    std::unique_lock<std::mutex> lk(v->mu);
    auto it = v->slots.find(stream_id);
    if (it == v->slots.end() || it->second->closing || it->second->evicted)
        return fail(EVXG_ERROR_INVALID_INDEX, "evxg_server_evict: no such resident stream");
    Slot *s = it->second;
    Lane *l = v->lanes[s->lane];
    // The frames it already has are encoded and delivered first; then its lane
    // rebuilds its batch without it, so that no tick touches its memory again.
    v->drainers++;
    v->cv_work.notify_all();
    v->cv_done.wait(lk, [&] { return v->error || drained(s); });
    if (!v->error) {
        s->evicted = true;
        l->set_dirty = true;
        v->cv_work.notify_all();
        v->cv_done.wait(lk, [&] { return v->error || !l->set_dirty; });
    }
    v->drainers--;
    if (v->error) return fail(v->error, "evxg_server_evict: the server has failed");
    evxg_stream *st = s->st;
    s->st = nullptr;
    lk.unlock();
    std::vector<uint8_t> saved;
    int rc = EVXG_SUCCESS;
    try {
        saved.resize(evxg_stream_state_bytes(st));
    } catch (const std::bad_alloc &) {
        rc = fail(EVXG_ERROR_OUTOFMEMORY, "evxg_server_evict: host allocation");
    }
    if (!rc) rc = evxg_stream_save(st, saved.data(), saved.size(), nullptr);
    lk.lock();
    if (rc) {   // no copy: keep the stream resident as it was
        s->st = st;
        s->evicted = false;
        l->set_dirty = true;
        v->cv_work.notify_all();
        return rc;
    }
    lk.unlock();
    evxg_stream_destroy(st);
    lk.lock();
    s->saved = std::move(saved);
    v->used -= s->bytes;
    s->bytes = 0;
    return EVXG_SUCCESS;
}

int evxg_server_restore(evxg_server *v, uint32_t stream_id)
{
    if (!v) return EVXG_ERROR_INVALIDARG;
    Slot *s = nullptr;
    size_t bytes = 0;
    {
        std::lock_guard<std::mutex> lk(v->mu);
        if (v->error) return fail(v->error, "evxg_server_restore: the server has failed");
        auto it = v->slots.find(stream_id);
        if (it == v->slots.end() || it->second->closing || !it->second->evicted)
            return fail(EVXG_ERROR_INVALID_INDEX, "evxg_server_restore: no such evicted stream");
        s = it->second;
        bytes = stream_bytes(s->w, s->h);
        if (v->used - dead_bytes(v) + bytes > v->budget)
            return fail(EVXG_ERROR_CAPACITY_LIMIT, "evxg_server_restore: the device memory budget is spent");
        v->used += bytes;   // reserved while the stream is created
    }
    evxg_stream *st = nullptr;
    int rc = evxg_stream_create_config(s->w, s->h, &s->cfg, &st);
    if (!rc) rc = evxg_stream_restore(st, s->saved.data(), s->saved.size(), nullptr);
    std::lock_guard<std::mutex> lk(v->mu);
    if (rc) {
        if (st) evxg_stream_destroy(st);
        v->used -= bytes;
        return rc;
    }
    s->st = st;
    s->bytes = bytes;
    s->saved.clear();
    s->saved.shrink_to_fit();
    s->evicted = false;
    v->lanes[s->lane]->set_dirty = true;
    v->cv_work.notify_all();
    return EVXG_SUCCESS;
}

int evxg_server_drain(evxg_server *v)
{
    if (!v) return EVXG_ERROR_INVALIDARG;
    std::unique_lock<std::mutex> lk(v->mu);
    v->drainers++;
    v->cv_work.notify_all();
    v->cv_done.wait(lk, [&] {
        if (v->error) return true;
        for (const Lane *l : v->lanes)   // pend is read without the worker's ownership: only as a hint, in_flight decides
            if (l->set_dirty) return false;
        for (auto &kv : v->slots)
            if (!kv.second->ready.empty() || kv.second->in_flight) return false;
        return true;
    });
    v->drainers--;
    return v->error ? fail(v->error, "evxg_server_drain: a tick failed") : EVXG_SUCCESS;
}

int evxg_server_stats(evxg_server *v, uint64_t *frames, uint64_t *ticks, uint64_t *rebuilds, uint64_t *bytes_in_use)
{
    if (!v) return EVXG_ERROR_INVALIDARG;
    std::lock_guard<std::mutex> lk(v->mu);
    if (frames) *frames = v->frames_done;
    if (ticks) *ticks = v->ticks;
    if (rebuilds) *rebuilds = v->rebuilds;
    if (bytes_in_use) *bytes_in_use = v->used - dead_bytes(v);   // streams not yet closed and delivered
    return EVXG_SUCCESS;
}

int evxg_server_destroy(evxg_server *v)
{
    if (!v) return EVXG_ERROR_INVALIDARG;
    {
        std::lock_guard<std::mutex> lk(v->mu);
        for (auto &kv : v->slots)
            if (!kv.second->closing) { evxg_encoder_flush(kv.second->planner); kv.second->closing = true; }
        v->stop = true;
        v->cv_work.notify_all();
    }
    for (Lane *l : v->lanes) l->worker.join();
    for (Lane *l : v->lanes) {
        if (l->batch) evxg_batch_destroy(l->batch);
        cudaStreamDestroy(l->cs);
        delete l;
    }
    for (auto &kv : v->slots) {
        evxg_encoder_destroy(kv.second->planner);
        evxg_stream_destroy(kv.second->st);
        delete kv.second;
    }
    delete v;
    return EVXG_SUCCESS;
}

}  // extern "C"
