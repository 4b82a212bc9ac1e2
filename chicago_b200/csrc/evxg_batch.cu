// evxg_batch.cu -- batched ticks: many streams, of any sizes and at any GOP
// positions, advance one frame each through every stage of the pipeline with
// one kernel launch per stage, the whole tick replayed as one CUDA graph.
//
// The reference encodes one stream per evx3_encoder, frame by frame
// (src/video/evx3enc.cpp:105-414); a tick here is, for every stream with a
// frame, exactly that stream's engine_encode_frame minus serialization
// (src/video/encode.cpp:945-1001), so every stream's output is identical to
// encoding it alone.  What changes is how the work is launched:
//  * every frame-level kernel covers all streams (blockIdx.z = stream), with
//    the streams' parameters in one device array;
//  * the macroblock pass is one persistent launch whose CTAs (or three-CTA
//    clusters) claim (stream, row) items from one queue for the whole tick;
//  * the per-stream copies and memsets of the single path are kernels too,
//    so a tick is a fixed sequence: copies of the parameters and of the
//    input frames, 18 kernels, copies of the outputs.  It is captured once
//    per buffer parity and replayed.
// Host buffers (inputs, parameters, outputs) come in two parities, so the
// host fills tick t+1 while the device runs tick t.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "evxg_internal.cuh"

using namespace evxg;

struct evxg_batch {
    struct Side {
        FrameArgs *args = nullptr;          // pinned: one entry per stream
        int *queue = nullptr;               // pinned: [0] item count, then (stream, row) pairs
        int *err = nullptr;                 // pinned: the tick's error word, copied back
        std::vector<uint8_t *> rgb;         // pinned RGB24 inputs
        std::vector<uint8_t *> out;         // pinned outputs: blocks | previous blocks | SAO | levels
        cudaGraphExec_t exec = nullptr;
        cudaEvent_t done = nullptr;
        bool pending = false;
    };
    std::vector<evxg_stream *> st;
    Side side[2];
    FrameArgs *d_args = nullptr;
    int *d_queue = nullptr;                 // same layout as Side::queue
    int *d_ctl = nullptr;                   // [0] queue counter, [1] error word
    uint32_t qcap = 0;                      // rows of all streams together
    int form = EVXG_MB_FORM_SINGLE, grid = 1, policy = 0;
    int num_sms = 0, max_clusters = 0;
    long long timeout_ns = 5000000000LL;
};

static const int kTickKernels = 10 + kSaoPasses;   // kernels per tick, whatever the number of streams

// Shape of the macroblock pass from a model of the tick: a tick lasts at least
// its longest wavefront's critical path (cols + 3 x (rows - 1) MB steps) and at
// least the MBs of all streams over the units working on them (SMs in the
// single form, three-SM clusters in the cluster form), each MB step costing
// about kSingleVsCluster times as long in the single form (both forms timed on
// one 1080p, 720p and 360p stream: 1.53 at every size).
static const double kSingleVsCluster = 1.5;
static void model_shape(evxg_batch *b)
{
    double path = 0, mbs = 0;
    int busy = 0;
    for (const evxg_stream *s : b->st) {
        path = std::max(path, (double)(s->mbw + 3 * (s->mbh - 1)));
        mbs += (double)s->mbw * s->mbh;
        busy += (int)std::min<uint32_t>(s->mbh, s->mbw / 3 + 3);
    }
    const double t_single = kSingleVsCluster * std::max(path, mbs / b->num_sms);
    const double t_cluster = b->max_clusters > 0 ? std::max(path, mbs / b->max_clusters) : 1e30;
    if (t_cluster < t_single) {
        b->form = EVXG_MB_FORM_CLUSTER;
        b->grid = std::max(1, std::min(busy, b->max_clusters));
    } else {
        b->form = EVXG_MB_FORM_SINGLE;
        b->grid = std::max(1, std::min((int)b->qcap, b->num_sms));
    }
    b->policy = 0;
}

static size_t out_bytes(const evxg_stream *s)
{
    const size_t nblk = (size_t)s->mbw * s->mbh;
    return nblk * (2 * sizeof(evxg_block_desc) + sizeof(evxg_sao_info)) + s->plane_elems * sizeof(int16_t);
}

// Row queue of a tick.  Policy 0 interleaves the streams row by row (rows
// that can start at about the same time are claimed together: row r of any
// stream starts about 3r macroblock steps into the tick); policy 1 also puts,
// among rows of the same index, the streams with the longer remaining
// critical path (columns + 3 x rows left) first.  Both keep every stream's
// rows in order, which the wavefront's deadlock freedom needs.
static int build_queue(const evxg_batch *b, const std::vector<char> &active, int *q)
{
    struct Item { int s, r; long key, tie; };
    std::vector<Item> v;
    for (size_t i = 0; i < b->st.size(); i++) {
        if (!active[i]) continue;
        const evxg_stream *s = b->st[i];
        for (uint32_t r = 0; r < s->mbh; r++)
            v.push_back({(int)i, (int)r, (long)r, b->policy == 1 ? -(long)(s->mbw + 3 * (s->mbh - 1 - r)) : (long)i});
    }
    std::stable_sort(v.begin(), v.end(), [](const Item &x, const Item &y) {
        return x.key != y.key ? x.key < y.key : x.tie < y.tie;
    });
    q[0] = (int)v.size();
    for (size_t k = 0; k < v.size(); k++) { q[2 + 2 * k] = v[k].s; q[3 + 2 * k] = v[k].r; }
    return (int)v.size();
}

// The tick's work on stream cs (captured into the parity's graph).
static int enqueue_tick(evxg_batch *b, int parity, cudaStream_t cs)
{
    evxg_batch::Side &sd = b->side[parity];
    const unsigned n = (unsigned)b->st.size();
    unsigned cvx = 1, cvy = 1, rdo = 1, wf = 1;
    size_t msmem = 0, dsmem = 0;
    for (const evxg_stream *s : b->st) {
        const unsigned cw = std::min(s->vw, s->W), ch = std::min(s->vh, s->H);
        cvx = std::max(cvx, (cw / 2 + 127) / 128);
        cvy = std::max(cvy, ch / 2);
        rdo = std::max(rdo, (s->mbw * s->mbh + 7) / 8);   // one warp per MB, 8 per block
        wf = std::max(wf, (s->mbh + 7) / 8);
        msmem = std::max(msmem, merge_shared_bytes((int)s->mbw, (int)s->mbh));
        dsmem = std::max(dsmem, deblock_shared_bytes((int)s->W));
    }
    const unsigned share = std::max(8u, (unsigned)b->num_sms * 8 / n);
    CK(cudaMemsetAsync(b->d_ctl, 0, 2 * sizeof(int), cs));
    CK(cudaMemcpyAsync(b->d_args, sd.args, n * sizeof(FrameArgs), cudaMemcpyHostToDevice, cs));
    CK(cudaMemcpyAsync(b->d_queue, sd.queue, (2 + 2 * (size_t)b->qcap) * sizeof(int), cudaMemcpyHostToDevice, cs));
    for (unsigned i = 0; i < n; i++)
        CK(cudaMemcpyAsync(b->st[i]->rgb, sd.rgb[i], (size_t)b->st[i]->vw * b->st[i]->vh * 3, cudaMemcpyHostToDevice, cs));
    const int *qlen = b->d_queue;
    const int2 *items = reinterpret_cast<const int2 *>(b->d_queue + 2);
    k_tick_prep_b<<<dim3(64, 1, n), 256, 0, cs>>>(b->d_args, kSaoPasses);
    k_convert_b<<<dim3(cvx, cvy, n), 128, 0, cs>>>(b->d_args);
    if (b->form == EVXG_MB_FORM_CLUSTER)
        k_mb_cluster_b<<<3 * b->grid, mb_threads(), mb_shared_bytes(), cs>>>(b->d_args, items, qlen, b->d_ctl);
    else
        k_mb_wavefront_b<<<b->grid, mb_threads(), mb_shared_bytes(), cs>>>(b->d_args, items, qlen, b->d_ctl);
    k_deblock_b<<<dim3(kDeblockCtas, 1, n), kDeblockThreads, dsmem, cs>>>(b->d_args);
    k_sao_copy_b<<<dim3(share / 2, 1, n), 256, 0, cs>>>(b->d_args);
    k_sao_rdo_b<<<dim3(rdo, 1, n), 256, 0, cs>>>(b->d_args);
    k_sao_merge_b<<<dim3(kMergeCtas, 1, n), kMergeThreads, msmem, cs>>>(b->d_args);
    for (int p = 0; p < kSaoPasses; p++) k_sao_fix_b<<<dim3(share, 1, n), 256, 0, cs>>>(b->d_args, p);
    k_sao_restore_b<<<dim3(share / 2, 1, n), 256, 0, cs>>>(b->d_args, kSaoPasses - 1);
    k_sao_apply_b<<<dim3(wf, 1, n), 256, 0, cs>>>(b->d_args, kSaoPasses - 1);
    k_tick_post_b<<<dim3(64, 1, n), 256, 0, cs>>>(b->d_args);
    CK(cudaGetLastError());
    for (unsigned i = 0; i < n; i++) {   // the serializer's inputs, as evxg_fetch_tables returns them
        const evxg_stream *s = b->st[i];
        const size_t nblk = (size_t)s->mbw * s->mbh, tb = nblk * sizeof(evxg_block_desc);
        uint8_t *o = sd.out[i];
        CK(cudaMemcpyAsync(o, s->bt, tb, cudaMemcpyDeviceToHost, cs));
        CK(cudaMemcpyAsync(o + tb, s->prev_ser, tb, cudaMemcpyDeviceToHost, cs));
        CK(cudaMemcpyAsync(o + 2 * tb, s->sao, nblk * sizeof(evxg_sao_info), cudaMemcpyDeviceToHost, cs));
        CK(cudaMemcpyAsync(o + 2 * tb + nblk * sizeof(evxg_sao_info), s->lev, s->plane_elems * sizeof(int16_t),
                           cudaMemcpyDeviceToHost, cs));
    }
    CK(cudaMemcpyAsync(sd.err, b->d_ctl + 1, sizeof(int), cudaMemcpyDeviceToHost, cs));
    return EVXG_SUCCESS;
}

static int build_graph(evxg_batch *b, int parity)
{
    evxg_batch::Side &sd = b->side[parity];
    if (sd.exec) return EVXG_SUCCESS;
    cudaStream_t cs;
    CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed);   // other threads may allocate meanwhile
    int rc = e == cudaSuccess ? enqueue_tick(b, parity, cs) : cuda_fail(e, "cudaStreamBeginCapture");
    if (e == cudaSuccess) {
        const cudaError_t e2 = cudaStreamEndCapture(cs, &g);
        if (!rc && e2 != cudaSuccess) rc = cuda_fail(e2, "cudaStreamEndCapture");
    }
    if (!rc) {
        const cudaError_t e3 = cudaGraphInstantiate(&sd.exec, g, 0);
        if (e3 != cudaSuccess) rc = cuda_fail(e3, "cudaGraphInstantiate");
    }
    if (g) cudaGraphDestroy(g);
    cudaStreamDestroy(cs);
    return rc;
}

static void drop_graphs(evxg_batch *b)
{
    for (auto &sd : b->side)
        if (sd.exec) { cudaGraphExecDestroy(sd.exec); sd.exec = nullptr; }
}

// Synthetic content for the autotuner: a pattern that moves by (3, 2) px per
// tick, so the searches find motion as in real content.
static void synth_frame(uint8_t *p, uint32_t w, uint32_t h, int t)
{
    for (uint32_t y = 0; y < h; y++)
        for (uint32_t x = 0; x < w; x++) {
            const float u = (float)(x + 3 * t), v = (float)(y + 2 * t);
            const int base = (int)(128 + 60 * sinf(u * 0.11f) * cosf(v * 0.07f) + 40 * sinf((u + v) * 0.031f));
            const int n = (int)((x * 2654435761u ^ y * 40503u ^ (uint32_t)t * 97u) >> 28) - 8;   // a little noise
            uint8_t *q = p + ((size_t)y * w + x) * 3;
            q[0] = (uint8_t)std::min(255, std::max(0, base + n));
            q[1] = (uint8_t)std::min(255, std::max(0, base - n / 2 + 10));
            q[2] = (uint8_t)std::min(255, std::max(0, 255 - base + n));
        }
}

extern "C" {

int evxg_batch_create(evxg_stream *const *streams, uint32_t n, evxg_batch **out)
{
    if (!out || !streams || !n || n > 65535) return fail(EVXG_ERROR_INVALIDARG, "evxg_batch_create: need 1..65535 streams");
    *out = nullptr;
    for (uint32_t i = 0; i < n; i++)
        for (uint32_t j = 0; j < i; j++)
            if (!streams[i] || streams[i] == streams[j])
                return fail(EVXG_ERROR_INVALIDARG, "evxg_batch_create: null or repeated stream");
    if (!streams[0]) return fail(EVXG_ERROR_INVALIDARG, "evxg_batch_create: null stream");
    evxg_batch *b = new evxg_batch();
    b->st.assign(streams, streams + n);
    for (evxg_stream *s : b->st) b->qcap += s->mbh;
    b->num_sms = b->st[0]->num_sms;
    b->max_clusters = max_active_clusters();
    model_shape(b);   // the default shape; evxg_batch_autotune measures instead
    cudaError_t e = cudaMalloc(&b->d_args, n * sizeof(FrameArgs));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_queue, (2 + 2 * (size_t)b->qcap) * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_ctl, 2 * sizeof(int));
    for (auto &sd : b->side) {
        if (e == cudaSuccess) e = cudaMallocHost(&sd.args, n * sizeof(FrameArgs));
        if (e == cudaSuccess) e = cudaMallocHost(&sd.queue, (2 + 2 * (size_t)b->qcap) * sizeof(int));
        if (e == cudaSuccess) e = cudaMallocHost(&sd.err, sizeof(int));
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sd.done, cudaEventDisableTiming);
        sd.rgb.assign(n, nullptr);
        sd.out.assign(n, nullptr);
        for (uint32_t i = 0; i < n && e == cudaSuccess; i++) {
            e = cudaMallocHost(&sd.rgb[i], (size_t)b->st[i]->vw * b->st[i]->vh * 3);
            if (e == cudaSuccess) e = cudaMallocHost(&sd.out[i], out_bytes(b->st[i]));
            if (e == cudaSuccess) memset(sd.rgb[i], 0, (size_t)b->st[i]->vw * b->st[i]->vh * 3);
        }
        if (e == cudaSuccess) { memset(sd.queue, 0, (2 + 2 * (size_t)b->qcap) * sizeof(int)); *sd.err = 0; }
    }
    if (e != cudaSuccess) {
        const int rc = cuda_fail(e, "evxg_batch_create");
        evxg_batch_destroy(b);
        return rc;
    }
    // Both parities' tick graphs now: they do not depend on the frames, and the
    // first ticks then do not pay for the capture.
    for (int p = 0; p < 2; p++) {
        const int rc = build_graph(b, p);
        if (rc) {
            evxg_batch_destroy(b);
            return rc;
        }
    }
    *out = b;
    return EVXG_SUCCESS;
}

int evxg_batch_destroy(evxg_batch *b)
{
    if (!b) return EVXG_ERROR_INVALIDARG;
    for (auto &sd : b->side)
        if (sd.pending && sd.done) cudaEventSynchronize(sd.done);
    drop_graphs(b);
    for (auto &sd : b->side) {
        cudaFreeHost(sd.args); cudaFreeHost(sd.queue); cudaFreeHost(sd.err);
        for (uint8_t *p : sd.rgb) cudaFreeHost(p);
        for (uint8_t *p : sd.out) cudaFreeHost(p);
        if (sd.done) cudaEventDestroy(sd.done);
    }
    cudaFree(b->d_args); cudaFree(b->d_queue); cudaFree(b->d_ctl);
    delete b;
    return EVXG_SUCCESS;
}

uint8_t *evxg_batch_input(evxg_batch *b, uint32_t i, uint32_t parity)
{
    if (!b || i >= b->st.size() || parity > 1) return nullptr;
    return b->side[parity].rgb[i];
}

int evxg_batch_output(evxg_batch *b, uint32_t i, uint32_t parity, const evxg_block_desc **blocks,
                      const evxg_block_desc **prev_blocks, const evxg_sao_info **sao, const int16_t **levels)
{
    if (!b || i >= b->st.size() || parity > 1) return fail(EVXG_ERROR_INVALIDARG, "evxg_batch_output: bad index");
    const evxg_stream *s = b->st[i];
    const size_t nblk = (size_t)s->mbw * s->mbh, tb = nblk * sizeof(evxg_block_desc);
    const uint8_t *o = b->side[parity].out[i];
    if (blocks) *blocks = reinterpret_cast<const evxg_block_desc *>(o);
    if (prev_blocks) *prev_blocks = reinterpret_cast<const evxg_block_desc *>(o + tb);
    if (sao) *sao = reinterpret_cast<const evxg_sao_info *>(o + 2 * tb);
    if (levels) *levels = reinterpret_cast<const int16_t *>(o + 2 * tb + nblk * sizeof(evxg_sao_info));
    return EVXG_SUCCESS;
}

int evxg_batch_wait(evxg_batch *b, uint32_t parity)
{
    if (!b || parity > 1) return fail(EVXG_ERROR_INVALIDARG, "evxg_batch_wait: bad argument");
    evxg_batch::Side &sd = b->side[parity];
    if (!sd.pending) return EVXG_SUCCESS;
    CK(cudaEventSynchronize(sd.done));
    sd.pending = false;
    if (*sd.err) return fail(*sd.err, "evxg_batch_wait: a wavefront of the tick gave up waiting (timeout)");
    return EVXG_SUCCESS;
}

int evxg_batch_encode(evxg_batch *b, const evxg_frame *frames, uint32_t parity, void *cuda_stream)
{
    if (!b || !frames || parity > 1) return fail(EVXG_ERROR_INVALIDARG, "evxg_batch_encode: bad argument");
    evxg_batch::Side &sd = b->side[parity];
    if (sd.pending) {   // this parity's parameters and outputs are free again once its last tick is done
        CK(cudaEventSynchronize(sd.done));
        sd.pending = false;
        if (*sd.err) return fail(*sd.err, "evxg_batch_encode: the previous tick of this parity gave up waiting (timeout)");
    }
    const size_t n = b->st.size();
    std::vector<char> active(n, 0);
    std::vector<evxg_frame> fr(n);
    for (size_t i = 0; i < n; i++) {
        if (frames[i].type < 0) continue;   // no frame for this stream in this tick
        const int rc = check_frame(b->st[i], &frames[i], "evxg_batch_encode", &fr[i]);
        if (rc) return rc;
        active[i] = 1;
    }
    for (size_t i = 0; i < n; i++) {
        FrameArgs &a = sd.args[i];
        if (active[i]) {
            fill_args(b->st[i], &fr[i], b->st[i]->rgb, a);
        } else {
            a = FrameArgs{};
            a.active = 0;
        }
        a.error = b->d_ctl + 1;   // one error word for the tick: any wait that gives up fails all of it
        a.timeout_ns = b->timeout_ns;
    }
    build_queue(b, active, sd.queue);
    int rc = build_graph(b, (int)parity);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    CK(cudaGraphLaunch(sd.exec, st));
    CK(cudaEventRecord(sd.done, st));
    sd.pending = true;
    return EVXG_SUCCESS;
}

uint32_t evxg_batch_launch_count(const evxg_batch *b) { return b ? (uint32_t)kTickKernels : 0; }

int evxg_batch_set_timeout_ns(evxg_batch *b, int64_t ns)
{
    if (!b || ns <= 0) return fail(EVXG_ERROR_INVALIDARG, "evxg_batch_set_timeout_ns: null batch or ns <= 0");
    b->timeout_ns = ns;   // copied into every stream's parameters at the next tick
    return EVXG_SUCCESS;
}

int evxg_batch_set_shape(evxg_batch *b, int form, int grid, int policy)
{
    if (!b || (form != EVXG_MB_FORM_SINGLE && form != EVXG_MB_FORM_CLUSTER) || grid < 1 || policy < 0 || policy > 1)
        return fail(EVXG_ERROR_INVALIDARG, "evxg_batch_set_shape: bad form, grid or policy");
    const int cap = form == EVXG_MB_FORM_CLUSTER ? b->max_clusters : b->num_sms;
    if (cap < 1) return fail(EVXG_ERROR_INVALID_RESOURCE, "evxg_batch_set_shape: the device cannot run this form");
    for (auto &sd : b->side)
        if (sd.pending) { CK(cudaEventSynchronize(sd.done)); sd.pending = false; }
    b->form = form;
    b->grid = std::min(grid, cap);   // every CTA / cluster of the persistent grid must be resident
    b->policy = policy;
    drop_graphs(b);
    for (int p = 0; p < 2; p++) {
        const int rc = build_graph(b, p);
        if (rc) return rc;
    }
    return EVXG_SUCCESS;
}

int evxg_batch_get_shape(const evxg_batch *b, int *form, int *grid, int *policy)
{
    if (!b) return EVXG_ERROR_INVALIDARG;
    if (form) *form = b->form;
    if (grid) *grid = b->grid;
    if (policy) *policy = b->policy;
    return EVXG_SUCCESS;
}

// Autotuner: times each candidate shape of the macroblock pass on a short
// synthetic sequence (an I, a P and two B frames per stream -- I/P streams: an
// I and three P frames -- at the streams' own sizes), keeps the fastest and returns every stream to its initial
// state.  Candidates: one CTA per row or three-CTA clusters, the persistent
// grid at full and at two-thirds width, and both queue orders.
int evxg_batch_autotune(evxg_batch *b, void *cuda_stream, float *best_ms)
{
    if (!b) return fail(EVXG_ERROR_INVALIDARG, "evxg_batch_autotune: null batch");
    cudaStream_t st = (cudaStream_t)cuda_stream;
    const size_t n = b->st.size();
    struct Cand { int form, grid, policy; };
    std::vector<Cand> cands;
    const int rows = (int)b->qcap;
    for (int policy = 0; policy < 2; policy++) {
        for (int frac = 3; frac >= 2; frac--) {
            cands.push_back({EVXG_MB_FORM_SINGLE, std::max(1, std::min(rows, b->num_sms * frac / 3)), policy});
            if (b->max_clusters > 0)
                cands.push_back({EVXG_MB_FORM_CLUSTER, std::max(1, std::min(rows, b->max_clusters * frac / 3)), policy});
        }
    }
    for (uint32_t par = 0; par < 2; par++) {   // content of ticks 0, 2 and 1, 3, made before anything is timed
        const int r0 = evxg_batch_wait(b, par);
        if (r0) return r0;
        for (size_t i = 0; i < n; i++) synth_frame(b->side[par].rgb[i], b->st[i]->vw, b->st[i]->vh, (int)par);
    }
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    std::vector<evxg_frame> fr(n);
    float best = 1e30f;
    Cand pick = {b->form, b->grid, b->policy};
    int rc = EVXG_SUCCESS;
    for (const Cand &c : cands) {
        if ((rc = evxg_batch_set_shape(b, c.form, c.grid, c.policy))) break;
        for (evxg_stream *s : b->st)
            if ((rc = reset_stream(s, st))) break;
        if (rc) break;
        // I, P (from I), B (I, P), B (I, reference B): the reference's first mini-GOP shape
        const int types[4] = {EVXG_FRAME_INTRA, EVXG_FRAME_INTER, EVXG_FRAME_BIDIR, EVXG_FRAME_BIDIR};
        const int dpb[4] = {0, 1, 2, 3}, fwd[4] = {0, 0, 0, 0}, bwd[4] = {0, 0, 1, 2};
        for (int t = 0; t < 4 && !rc; t++) {
            const uint32_t par = (uint32_t)(t & 1);
            for (size_t i = 0; i < n; i++) {
                fr[i] = evxg_frame{};
                // I/P streams: I then P frames (their slots follow from the index)
                fr[i].type = b->st[i]->cfg.b_frames ? types[t] : (t ? EVXG_FRAME_INTER : EVXG_FRAME_INTRA);
                fr[i].index = (uint32_t)t; fr[i].quality = 8; fr[i].display_order = (uint32_t)t;
                fr[i].is_reference = t < 3; fr[i].dpb_slot = (uint8_t)dpb[t];
                fr[i].ref_slot_fwd = (uint8_t)fwd[t]; fr[i].ref_slot_bwd = (uint8_t)bwd[t];
            }
            if (t == 1) {
                const cudaError_t er = cudaEventRecord(e0, st);
                if (er != cudaSuccess) { rc = cuda_fail(er, "cudaEventRecord"); break; }
            }
            rc = evxg_batch_encode(b, fr.data(), par, cuda_stream);
        }
        if (!rc) {
            const cudaError_t er = cudaEventRecord(e1, st);
            if (er != cudaSuccess) rc = cuda_fail(er, "cudaEventRecord");
        }
        for (uint32_t par = 0; par < 2 && !rc; par++) rc = evxg_batch_wait(b, par);
        if (rc) break;
        float ms = 0;
        cudaError_t et = cudaEventSynchronize(e1);
        if (et == cudaSuccess) et = cudaEventElapsedTime(&ms, e0, e1);
        if (et != cudaSuccess) { rc = cuda_fail(et, "evxg_batch_autotune: timing"); break; }
        if (ms < best) { best = ms; pick = c; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (evxg_stream *s : b->st) {
        const int r2 = reset_stream(s, st);
        if (!rc) rc = r2;
    }
    if (!rc) rc = evxg_batch_set_shape(b, pick.form, pick.grid, pick.policy);
    if (!rc) {
        const cudaError_t es = cudaStreamSynchronize(st);
        if (es != cudaSuccess) rc = cuda_fail(es, "evxg_batch_autotune");
    }
    if (best_ms) *best_ms = best;
    return rc;
}

}  // extern "C"
