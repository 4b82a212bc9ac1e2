// evxg_api.cu -- host side of the B200 EVX3 encoder pipeline: the C ABI of
// include/evxg.h (per-stream device state, per-frame launch sequence, table
// fetch) and the GOP-level encoder that mirrors the reference's evx3_encoder
// (src/video/evx3enc.cpp:35-414) on top of it.
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "evxg_internal.cuh"

using namespace evxg;

static thread_local std::string g_last_error;

namespace evxg {
int fail(int code, const char *what)
{
    g_last_error = what;
    return code;
}
int cuda_fail(cudaError_t e, const char *where)
{
    g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? EVXG_ERROR_OUTOFMEMORY : EVXG_ERROR_EXECUTION_FAILURE;
}
}  // namespace evxg

static void pipeline_free(evxg_stream *s);

// Host-side fault injection: the next n device allocations of stream
// creation report cudaErrorMemoryAllocation without allocating.
static std::atomic<uint32_t> g_inject_alloc{0};
template <class T>
static cudaError_t dev_alloc(T **p, size_t n)
{
    uint32_t k = g_inject_alloc.load();
    while (k > 0)
        if (g_inject_alloc.compare_exchange_weak(k, k - 1)) return cudaErrorMemoryAllocation;
    return cudaMalloc(p, n);
}

int evxg::check_config(const evxg_config *c, const char *who)
{
    static thread_local char msg[200];
    const bool ok = (c->b_frames == 1 && c->ref_count == 4) || (c->b_frames == 0 && (c->ref_count == 2 || c->ref_count == 4));
    if (!ok) {
        snprintf(msg, sizeof msg, "%s: unsupported configuration (b_frames %u, ref_count %u): B frames need 4 DPB slots, "
                 "I/P streams 2 or 4", who, c->b_frames, c->ref_count);
        return fail(EVXG_ERROR_INVALIDARG, msg);
    }
    if (c->search_radius != 16 || c->reserved) {
        snprintf(msg, sizeof msg, "%s: unsupported search radius %u (16)", who, c->search_radius);
        return fail(EVXG_ERROR_INVALIDARG, msg);
    }
    return EVXG_SUCCESS;
}

extern "C" {

float evxg_lambda(uint16_t q) { return 0.85f * powf(2.0f, ((float)q - 12.0f) / 3.0f); }   // common.h:264-266

const char *evxg_last_error(void) { return g_last_error.c_str(); }

int evxg_inject_alloc_failures(uint32_t n)
{
    g_inject_alloc.store(n);
    return EVXG_SUCCESS;
}

void evxg_config_default(evxg_config *cfg)
{
    if (!cfg) return;
    *cfg = evxg_config{};
    cfg->b_frames = 1; cfg->ref_count = 4; cfg->search_radius = 16;
}

int evxg_stream_create(uint32_t width, uint32_t height, evxg_stream **out)
{
    return evxg_stream_create_config(width, height, nullptr, out);
}

int evxg_stream_config(const evxg_stream *s, evxg_config *out)
{
    if (!s || !out) return fail(EVXG_ERROR_INVALIDARG, "evxg_stream_config: null argument");
    *out = s->cfg;
    return EVXG_SUCCESS;
}

int evxg_stream_create_config(uint32_t width, uint32_t height, const evxg_config *cfg, evxg_stream **out)
{
    if (!out || !width || !height || width > 65535 || height > 65535 || (width & 1) || (height & 1))
        return fail(EVXG_ERROR_INVALIDARG, "evxg_stream_create: width/height must be even and in 2..65534");
    *out = nullptr;
    evxg_config c;
    evxg_config_default(&c);
    if (cfg) {
        int rc = check_config(cfg, "evxg_stream_create");
        if (rc) return rc;
        c = *cfg;
    }
    evxg_stream *s = new evxg_stream();
    s->cfg = c;
    s->vw = width; s->vh = height;
    s->W = (width + 15) & ~15u; s->H = (height + 15) & ~15u;
    s->mbw = s->W / 16; s->mbh = s->H / 16;
    s->plane_elems = (size_t)s->W * s->H + 2 * (size_t)(s->W / 2) * (s->H / 2);
    const size_t pb = s->plane_elems * sizeof(int16_t), nblk = (size_t)s->mbw * s->mbh;
    s->timeout_ns = 5000000000LL;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = dev_alloc(&s->src, pb);
    if (e == cudaSuccess) e = dev_alloc(&s->lev, pb);
    for (int i = 0; i < 4 && e == cudaSuccess; i++) e = dev_alloc(&s->dpb[i], pb);
    if (e == cudaSuccess) e = dev_alloc(&s->bt, nblk * sizeof(evxg_block_desc));
    if (e == cudaSuccess) e = dev_alloc(&s->prev, nblk * sizeof(evxg_block_desc));
    if (e == cudaSuccess) e = dev_alloc(&s->prev_ser, nblk * sizeof(evxg_block_desc));
    if (e == cudaSuccess) e = dev_alloc(&s->sao, nblk * sizeof(evxg_sao_info));
    if (e == cudaSuccess) e = dev_alloc(&s->sao_stats, nblk * kSaoStatEntries * sizeof(int2));
    if (e == cudaSuccess) e = dev_alloc(&s->sao_orig, pb);
    if (e == cudaSuccess) e = dev_alloc(&s->sao_flags, kSaoPasses * sizeof(int));
    if (e == cudaSuccess) e = dev_alloc(&s->sao_mail, nblk * sizeof(unsigned long long));
    if (e == cudaSuccess) e = dev_alloc(&s->rgb, (size_t)width * height * 3);
    if (e == cudaSuccess) e = dev_alloc(&s->sync, (3 * s->mbh + 5) * sizeof(int));
    // Zeroing on a private stream, synchronised alone: no device-wide
    // synchronisation, which another thread capturing a graph would forbid.
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->aux, cudaStreamNonBlocking);
    for (int i = 0; i < 2 && e == cudaSuccess; i++) e = cudaEventCreateWithFlags(&s->ev_aux[i], cudaEventDisableTiming);
    cudaStream_t zs = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&zs, cudaStreamNonBlocking);
    if (e == cudaSuccess && reset_stream(s, zs)) e = cudaErrorUnknown;
    const int max_clusters = e == cudaSuccess ? max_active_clusters() : 0;
    if (e == cudaSuccess) e = cudaStreamSynchronize(zs);
    if (zs) cudaStreamDestroy(zs);
    if (e != cudaSuccess) {
        int rc = cuda_fail(e, "evxg_stream_create");
        evxg_stream_destroy(s);
        return rc;
    }
    // The wavefront (row r trails row r-1 by four MBs) keeps at most about
    // cols/4 + 1 rows busy at once; a few more rows than that hide the row
    // hand-over, more would only spin, and leaving SMs free lets other
    // streams' frames run beside this one.
    const uint32_t rows_busy = std::min<uint32_t>(s->mbh, s->mbw / 4 + 4);
    s->mb_grid = (int)std::min<uint32_t>(rows_busy, (uint32_t)s->num_sms);
    s->mb_clusters = (int)std::min<uint32_t>(rows_busy, (uint32_t)max_clusters);
    s->mb_form = s->mb_clusters > 0 ? EVXG_MB_FORM_CLUSTER : EVXG_MB_FORM_SINGLE;
    *out = s;
    return EVXG_SUCCESS;
}

int evxg_stream_destroy(evxg_stream *s)
{
    if (!s) return EVXG_ERROR_INVALIDARG;
    cudaFree(s->src); cudaFree(s->lev);
    for (int i = 0; i < 4; i++) cudaFree(s->dpb[i]);
    cudaFree(s->bt); cudaFree(s->prev); cudaFree(s->prev_ser);
    cudaFree(s->sao); cudaFree(s->sao_stats); cudaFree(s->rgb); cudaFree(s->sync);
    cudaFree(s->sao_orig); cudaFree(s->sao_flags); cudaFree(s->sao_mail);
    if (s->profile)
        for (int i = 0; i < 7; i++) cudaEventDestroy(s->ev[i]);
    pipeline_free(s);
    if (s->aux) { cudaStreamSynchronize(s->aux); cudaStreamDestroy(s->aux); }
    for (int i = 0; i < 2; i++)
        if (s->ev_aux[i]) cudaEventDestroy(s->ev_aux[i]);
    delete s;
    return EVXG_SUCCESS;
}

int evxg_stream_dims(const evxg_stream *s, uint32_t *aw, uint32_t *ah, uint32_t *mbw, uint32_t *mbh)
{
    if (!s) return EVXG_ERROR_INVALIDARG;
    if (aw) *aw = s->W;
    if (ah) *ah = s->H;
    if (mbw) *mbw = s->mbw;
    if (mbh) *mbh = s->mbh;
    return EVXG_SUCCESS;
}

uint32_t evxg_last_launch_count(const evxg_stream *s) { return s ? s->launches : 0; }

int evxg_stream_set_timeout_ns(evxg_stream *s, int64_t ns)
{
    if (!s || ns <= 0) return fail(EVXG_ERROR_INVALIDARG, "evxg_stream_set_timeout_ns: null stream or ns <= 0");
    s->timeout_ns = ns;
    return EVXG_SUCCESS;
}

int evxg_stream_reset(evxg_stream *s, void *cuda_stream)
{
    if (!s) return fail(EVXG_ERROR_INVALIDARG, "evxg_stream_reset: null stream");
    const cudaStream_t st = (cudaStream_t)cuda_stream;
    const int rc = reset_stream(s, st);
    if (rc) return rc;
    CK(cudaStreamSynchronize(st));
    return EVXG_SUCCESS;
}

// Saved stream state: a 48-byte header (magic "EVXS", format version, aligned
// size, build, SAO epoch, sizes of what follows), then the four DPB plane
// sets, the level planes, the temporal predictor table and the block table --
// everything a later frame of the stream reads (the source, the SAO scratch
// and the serializer's snapshot are rewritten by every frame).
struct SavedHeader {
    char magic[4];
    uint32_t version, W, H;
    evxg_config cfg;
    int32_t epoch;
    uint64_t plane_bytes, table_bytes;
    uint32_t reserved[2];
};
static_assert(sizeof(SavedHeader) == 48, "saved-state header");

uint64_t evxg_stream_state_bytes(const evxg_stream *s)
{
    if (!s) return 0;
    const uint64_t pb = s->plane_elems * sizeof(int16_t), tb = (uint64_t)s->mbw * s->mbh * sizeof(evxg_block_desc);
    return sizeof(SavedHeader) + 5 * pb + 2 * tb;
}

int evxg_stream_save(evxg_stream *s, void *host, uint64_t capacity, void *cuda_stream)
{
    if (!s || !host) return fail(EVXG_ERROR_INVALIDARG, "evxg_stream_save: null argument");
    if (capacity < evxg_stream_state_bytes(s)) return fail(EVXG_ERROR_CAPACITY_LIMIT, "evxg_stream_save: buffer too small");
    const cudaStream_t st = (cudaStream_t)cuda_stream;
    const uint64_t pb = s->plane_elems * sizeof(int16_t), tb = (uint64_t)s->mbw * s->mbh * sizeof(evxg_block_desc);
    SavedHeader h{};
    memcpy(h.magic, "EVXS", 4);
    h.version = 1; h.W = s->W; h.H = s->H; h.cfg = s->cfg; h.epoch = s->epoch;
    h.plane_bytes = pb; h.table_bytes = tb;
    uint8_t *o = static_cast<uint8_t *>(host);
    memcpy(o, &h, sizeof h);
    o += sizeof h;
    for (int i = 0; i < 4; i++, o += pb) CK(cudaMemcpyAsync(o, s->dpb[i], pb, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(o, s->lev, pb, cudaMemcpyDeviceToHost, st));
    o += pb;
    CK(cudaMemcpyAsync(o, s->prev, tb, cudaMemcpyDeviceToHost, st));
    o += tb;
    CK(cudaMemcpyAsync(o, s->bt, tb, cudaMemcpyDeviceToHost, st));
    return evxg_stream_sync(s, cuda_stream);
}

int evxg_stream_restore(evxg_stream *s, const void *host, uint64_t size, void *cuda_stream)
{
    if (!s || !host) return fail(EVXG_ERROR_INVALIDARG, "evxg_stream_restore: null argument");
    SavedHeader h;
    if (size < sizeof h) return fail(EVXG_ERROR_INVALID_RESOURCE, "evxg_stream_restore: not a saved stream state");
    memcpy(&h, host, sizeof h);
    if (memcmp(h.magic, "EVXS", 4) != 0 || h.version != 1 || size != evxg_stream_state_bytes(s))
        return fail(EVXG_ERROR_INVALID_RESOURCE, "evxg_stream_restore: not a saved stream state of this size");
    if (h.W != s->W || h.H != s->H || memcmp(&h.cfg, &s->cfg, sizeof h.cfg) != 0)
        return fail(EVXG_ERROR_INVALIDARG, "evxg_stream_restore: saved from a stream of another size or build");
    const cudaStream_t st = (cudaStream_t)cuda_stream;
    const uint64_t pb = h.plane_bytes, tb = h.table_bytes;
    const uint8_t *i = static_cast<const uint8_t *>(host) + sizeof h;
    for (int k = 0; k < 4; k++, i += pb) CK(cudaMemcpyAsync(s->dpb[k], i, pb, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(s->lev, i, pb, cudaMemcpyHostToDevice, st));
    i += pb;
    CK(cudaMemcpyAsync(s->prev, i, tb, cudaMemcpyHostToDevice, st));
    i += tb;
    CK(cudaMemcpyAsync(s->bt, i, tb, cudaMemcpyHostToDevice, st));
    // mail words of frames after the saved one could carry the epochs that
    // follow it: none may match (a zero word matches no epoch 1..255)
    CK(cudaMemsetAsync(s->sao_mail, 0, (size_t)s->mbw * s->mbh * sizeof(unsigned long long), st));
    s->epoch = h.epoch;
    return evxg_stream_sync(s, cuda_stream);
}

int evxg_stream_set_mb_form(evxg_stream *s, int form)
{
    if (!s || (form != EVXG_MB_FORM_SINGLE && form != EVXG_MB_FORM_CLUSTER))
        return fail(EVXG_ERROR_INVALIDARG, "evxg_stream_set_mb_form: unknown form");
    if (form == EVXG_MB_FORM_CLUSTER && s->mb_clusters <= 0)
        return fail(EVXG_ERROR_INVALID_RESOURCE, "evxg_stream_set_mb_form: the device cannot run the cluster form");
    s->mb_form = form;
    return EVXG_SUCCESS;
}

int evxg_stream_mb_form(const evxg_stream *s) { return s ? s->mb_form : -EVXG_ERROR_INVALIDARG; }

}  // extern "C"

// The reference zero-fills every image and table at allocation (image.cpp:89,
// common.cpp:167-187); stale-pixel reads of never-written DPB slots see zeros.
int evxg::reset_stream(evxg_stream *s, cudaStream_t st)
{
    const size_t pb = s->plane_elems * sizeof(int16_t), nblk = (size_t)s->mbw * s->mbh;
    CK(cudaMemsetAsync(s->src, 0, pb, st));
    CK(cudaMemsetAsync(s->lev, 0, pb, st));
    for (int i = 0; i < 4; i++) CK(cudaMemsetAsync(s->dpb[i], 0, pb, st));
    CK(cudaMemsetAsync(s->bt, 0, nblk * sizeof(evxg_block_desc), st));
    CK(cudaMemsetAsync(s->prev, 0, nblk * sizeof(evxg_block_desc), st));
    CK(cudaMemsetAsync(s->prev_ser, 0, nblk * sizeof(evxg_block_desc), st));
    CK(cudaMemsetAsync(s->sao, 0, nblk * sizeof(evxg_sao_info), st));
    CK(cudaMemsetAsync(s->sao_mail, 0, nblk * sizeof(unsigned long long), st));
    CK(cudaMemsetAsync(s->sync, 0, (3 * s->mbh + 5) * sizeof(int), st));
    s->epoch = 0;
    return EVXG_SUCCESS;
}

// Shared-memory limits of the macroblock kernels (once per process and device)
// and the number of three-CTA clusters the device co-schedules; 0 when the
// cluster form cannot run.
static int cluster_setup()   // with the device current, once per device
{
    const int smem = (int)mb_shared_bytes();
    cudaFuncSetAttribute(k_sao_merge, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_deblock, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_deblock_b, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_sao_merge_b, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_mb_wavefront, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(k_mb_wavefront_b, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int n = 0;
    if (cudaFuncSetAttribute(k_mb_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) == cudaSuccess &&
        cudaFuncSetAttribute(k_mb_cluster_b, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) == cudaSuccess) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = 3; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(3); cfg.blockDim = dim3(mb_threads()); cfg.dynamicSmemBytes = mb_shared_bytes();
        cfg.attrs = at; cfg.numAttrs = 1;
        if (cudaOccupancyMaxActiveClusters(&n, (void *)k_mb_cluster, &cfg) != cudaSuccess) n = 0;
    }
    cudaGetLastError();   // the cluster form is optional: fall back to one CTA per row
    return n;
}
int evxg::max_active_clusters()
{
    static int cached[64];
    static std::once_flag once[64];   // streams may be created on several threads at once
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    std::call_once(once[dev], [&] { cached[dev] = cluster_setup(); });
    return cached[dev];
}

// Frame descriptor checks shared by the single and the batched path.  Without
// B frames the reference's evx_frame has no slot fields: the destination and
// the references follow from the index (query_prediction_index_by_offset,
// common.cpp:256-259), and are written into the copy.
int evxg::check_frame(const evxg_stream *s, const evxg_frame *fin, const char *who, evxg_frame *out)
{
    return check_frame_config(s->cfg, fin, who, out);
}
int evxg::check_frame_config(const evxg_config &cfg, const evxg_frame *fin, const char *who, evxg_frame *out)
{
    static thread_local char msg[160];
    auto bad = [&](int code, const char *what) {
        snprintf(msg, sizeof msg, "%s: %s", who, what);
        return fail(code, msg);
    };
    evxg_frame g = *fin;
    const evxg_frame *f = &g;
    if (f->type < EVXG_FRAME_INTRA || f->type > EVXG_FRAME_BIDIR) return bad(EVXG_ERROR_INVALIDARG, "bad frame type");
    if (!cfg.b_frames) {
        if (f->type == EVXG_FRAME_BIDIR) return bad(EVXG_ERROR_INVALIDARG, "B frame in a stream without B frames");
        const uint32_t R = cfg.ref_count;
        g.dpb_slot = (uint8_t)(f->index % R);
        g.ref_slot_fwd = (uint8_t)((f->index + R - 1) % R);
        g.ref_slot_bwd = 0;
    }
    if (f->dpb_slot > 3 || f->ref_slot_fwd > 3 || f->ref_slot_bwd > 3)
        return bad(EVXG_ERROR_INVALID_INDEX, "DPB slot out of range");
    if (f->quality < 1 || f->quality > 63) return bad(EVXG_ERROR_INVALIDARG, "quality (QP) must be 1..63");
    if (f->type != EVXG_FRAME_INTRA && f->ref_slot_fwd == f->dpb_slot)
        return bad(EVXG_ERROR_INVALIDARG, "forward reference equals the destination slot");
    if (f->type == EVXG_FRAME_BIDIR && f->ref_slot_bwd == f->dpb_slot)
        return bad(EVXG_ERROR_INVALIDARG, "backward reference equals the destination slot");
    if (out) *out = g;
    return EVXG_SUCCESS;
}

void evxg::fill_args(evxg_stream *s, const evxg_frame *f, const uint8_t *drgb, FrameArgs &a)
{
    a = FrameArgs{};
    a.W = (int)s->W; a.H = (int)s->H; a.mbw = (int)s->mbw; a.mbh = (int)s->mbh;
    a.vis_w = (int)s->vw; a.vis_h = (int)s->vh;
    a.type = f->type; a.quality = f->quality; a.dpb = f->dpb_slot;
    a.ref_fwd = f->ref_slot_fwd; a.ref_bwd = f->ref_slot_bwd;
    if (s->cfg.b_frames) {
        a.nref = 1; a.ref_slot[0] = f->ref_slot_fwd; a.ip_mode = 0;
    } else {   // offsets 1 .. ref_count-1 from the index (encode.cpp:211-247); f's slots come from check_frame
        const uint32_t R = s->cfg.ref_count;
        a.nref = (int)R - 1; a.ip_mode = 1;
        for (uint32_t k = 0; k + 1 < R; k++) a.ref_slot[k] = (int)((f->index + R - (k + 1)) % R);
    }
    a.lambda = evxg_lambda(f->quality);
    for (int i = 0; i < 4; i++) a.planes[i] = s->dpb[i];
    a.src = s->src; a.lev = s->lev; a.bt = s->bt;
    a.prev = f->type == EVXG_FRAME_INTER ? s->prev : nullptr;
    a.sao = s->sao; a.sao_stats = s->sao_stats; a.rgb = drgb;
    a.sao_orig = s->sao_orig; a.sao_flags = s->sao_flags; a.sao_mail = s->sao_mail;
    s->epoch = s->epoch % 255 + 1;
    a.epoch = s->epoch;
    a.progress = s->sync; a.counters = s->sync + 3 * s->mbh; a.error = s->sync + 3 * s->mbh + 4;
    a.timeout_ns = s->timeout_ns;
    a.active = 1;
    a.prev_tab = s->prev; a.prev_ser = s->prev_ser; a.plane_elems = s->plane_elems;
}

// The frame's work on stream st; after_convert (optional) is recorded once the
// conversion has read the RGB input.
static int encode_impl(evxg_stream *s, const uint8_t *rgb, int rgb_on_device, const evxg_frame *fin, cudaStream_t st,
                       cudaEvent_t after_convert)
{
    if (!s || !rgb || !fin) return fail(EVXG_ERROR_INVALIDARG, "evxg_encode_frame: null argument");
    evxg_frame fr;
    int rc = check_frame(s, fin, "evxg_encode_frame", &fr);
    if (rc) return rc;
    const evxg_frame *f = &fr;
    const uint8_t *drgb = rgb;
    if (!rgb_on_device) {
        CK(cudaMemcpyAsync(s->rgb, rgb, (size_t)s->vw * s->vh * 3, cudaMemcpyHostToDevice, st));
        drgb = s->rgb;
    }
    FrameArgs a;
    fill_args(s, f, drgb, a);
    const size_t nblk = (size_t)s->mbw * s->mbh;
    // the serializer of this frame reads the previous table before this frame's update
    CK(cudaMemcpyAsync(s->prev_ser, s->prev, nblk * sizeof(evxg_block_desc), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemsetAsync(s->sync, 0xFF, 3 * s->mbh * sizeof(int), st));
    CK(cudaMemsetAsync(s->sync + 3 * s->mbh, 0, 4 * sizeof(int), st));
    // Deblocking runs beside the cluster-form pass when both fit on the
    // device at once: it trails the wavefront and writes the deblocked frame
    // to the SAO pristine copy (later macroblock rows still read the slot's
    // reconstruction), which then becomes the SAO pass's starting image.
    const bool overlap = s->aux && s->mb_form == EVXG_MB_FORM_CLUSTER && deblock_shared_bytes((int)s->W) > 0 &&
                         3 * s->mb_clusters + kDeblockCtas <= s->num_sms;
    if (overlap) CK(cudaEventRecord(s->ev_aux[0], st));   // the progress words are reset
    const int cw = (int)std::min(s->vw, s->W), ch = (int)std::min(s->vh, s->H);
    dim3 cg((cw / 2 + 127) / 128, ch / 2);
    const unsigned wf = (s->mbh + 7) / 8;
    auto mark = [&](int i) { if (s->profile) cudaEventRecord(s->ev[i], st); };
    mark(0);
    k_convert<<<cg, 128, 0, st>>>(a);
    if (after_convert) CK(cudaEventRecord(after_convert, st));
    mark(1);
    if (s->mb_form == EVXG_MB_FORM_CLUSTER)
        k_mb_cluster<<<3 * s->mb_clusters, mb_threads(), mb_shared_bytes(), st>>>(a);
    else
        k_mb_wavefront<<<s->mb_grid, mb_threads(), mb_shared_bytes(), st>>>(a);
    if (overlap) {   // launched after the pass, so that the pass's clusters are placed first
        FrameArgs da = a;
        da.db_out = s->sao_orig;
        da.db_wait = 1;
        CK(cudaStreamWaitEvent(s->aux, s->ev_aux[0], 0));
        k_deblock<<<kDeblockCtas, kDeblockThreads, deblock_shared_bytes((int)s->W), s->aux>>>(da);
        CK(cudaEventRecord(s->ev_aux[1], s->aux));
    }
    mark(2);
    if (overlap) {
        CK(cudaStreamWaitEvent(st, s->ev_aux[1], 0));
        mark(3);
        CK(cudaMemcpyAsync(s->dpb[f->dpb_slot], s->sao_orig, s->plane_elems * sizeof(int16_t), cudaMemcpyDeviceToDevice, st));
    } else {
        k_deblock<<<kDeblockCtas, kDeblockThreads, deblock_shared_bytes((int)s->W), st>>>(a);
        mark(3);
        CK(cudaMemcpyAsync(s->sao_orig, s->dpb[f->dpb_slot], s->plane_elems * sizeof(int16_t), cudaMemcpyDeviceToDevice, st));
    }
    CK(cudaMemsetAsync(s->sao_flags, 0, kSaoPasses * sizeof(int), st));
    k_sao_rdo<<<(unsigned)((nblk + 7) / 8), 256, 0, st>>>(a);   // one warp per MB
    mark(4);
    k_sao_merge<<<kMergeCtas, kMergeThreads, merge_shared_bytes((int)s->mbw, (int)s->mbh), st>>>(a);
    mark(5);
    for (int p = 0; p < kSaoPasses; p++) k_sao_fix<<<s->num_sms * 8, 256, 0, st>>>(a, p);
    k_sao_restore<<<s->num_sms * 4, 256, 0, st>>>(a, kSaoPasses - 1);
    k_sao_apply<<<wf, 256, 0, st>>>(a, kSaoPasses - 1);
    mark(6);
    s->launches = 7 + kSaoPasses;
    CK(cudaGetLastError());
    if (f->type != EVXG_FRAME_BIDIR)   // temporal MV predictor table (encode.cpp:990-998)
        CK(cudaMemcpyAsync(s->prev, s->bt, nblk * sizeof(evxg_block_desc), cudaMemcpyDeviceToDevice, st));
    return EVXG_SUCCESS;
}

// Device bytes of one table snapshot: block table, previous table, SAO table,
// level planes, the error word.
static size_t snapshot_bytes(const evxg_stream *s)
{
    const size_t nblk = (size_t)s->mbw * s->mbh;
    return 2 * nblk * sizeof(evxg_block_desc) + nblk * sizeof(evxg_sao_info) + s->plane_elems * sizeof(int16_t) + 16;
}

static int pipeline_setup(evxg_stream *s)
{
    if (s->copy) return EVXG_SUCCESS;
    cudaError_t e = cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->down, cudaStreamNonBlocking);
    for (int p = 0; p < 2 && e == cudaSuccess; p++) {
        e = dev_alloc(&s->prgb[p], (size_t)s->vw * s->vh * 3);
        if (e == cudaSuccess) e = dev_alloc(&s->snap[p], snapshot_bytes(s));
        for (cudaEvent_t *ev : {&s->ev_up[p], &s->ev_conv[p], &s->ev_snap[p], &s->ev_free[p]})
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    }
    for (int k = 0; k < evxg_stream::kRing && e == cudaSuccess; k++)
        e = cudaEventCreateWithFlags(&s->done[k], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMallocHost(&s->herr, evxg_stream::kRing * sizeof(int));
    if (e != cudaSuccess) return cuda_fail(e, "evxg_encode_frame_pipelined: set-up");
    return EVXG_SUCCESS;
}

static void pipeline_free(evxg_stream *s)
{
    if (!s->copy) return;
    cudaStreamSynchronize(s->copy);
    if (s->down) cudaStreamSynchronize(s->down);
    for (int p = 0; p < 2; p++) {
        cudaFree(s->prgb[p]);
        cudaFree(s->snap[p]);
        for (cudaEvent_t ev : {s->ev_up[p], s->ev_conv[p], s->ev_snap[p], s->ev_free[p]})
            if (ev) cudaEventDestroy(ev);
    }
    for (int k = 0; k < evxg_stream::kRing; k++)
        if (s->done[k]) cudaEventDestroy(s->done[k]);
    cudaFreeHost(s->herr);
    cudaStreamDestroy(s->copy);
    if (s->down) cudaStreamDestroy(s->down);
}

extern "C" {

int evxg_encode_frame(evxg_stream *s, const uint8_t *rgb, int rgb_on_device, const evxg_frame *fin, void *cuda_stream)
{
    return encode_impl(s, rgb, rgb_on_device, fin, (cudaStream_t)cuda_stream, nullptr);
}

// Frame t uses buffer pair t & 1.  Upload stream: into prgb[p] once frame
// t-2's conversion read it; compute stream: the frame, then (once frame t-2's
// download read it) the snapshot of its tables into snap[p]; download
// stream: the snapshot, then done[t % kRing].  Uploads and downloads on
// streams of their own, so the next frame's upload never queues behind this
// frame's download.
int evxg_encode_frame_pipelined(evxg_stream *s, const uint8_t *rgb, const evxg_frame *frame, evxg_block_desc *blocks,
                                evxg_block_desc *prev_blocks, evxg_sao_info *sao, int16_t *levels, void *cuda_stream,
                                uint64_t *ticket)
{
    if (!s || !rgb || !frame || !ticket) return fail(EVXG_ERROR_INVALIDARG, "evxg_encode_frame_pipelined: null argument");
    int rc = pipeline_setup(s);
    if (rc) return rc;
    const uint64_t t = s->tickets.load();
    const int p = (int)(t & 1), k = (int)(t % evxg_stream::kRing);
    if (t >= (uint64_t)evxg_stream::kRing) CK(cudaEventSynchronize(s->done[k]));   // the ring entry is free again
    cudaStream_t st = (cudaStream_t)cuda_stream, cp = s->copy, dn = s->down;
    CK(cudaStreamWaitEvent(cp, s->ev_conv[p], 0));
    CK(cudaMemcpyAsync(s->prgb[p], rgb, (size_t)s->vw * s->vh * 3, cudaMemcpyHostToDevice, cp));
    CK(cudaEventRecord(s->ev_up[p], cp));
    CK(cudaStreamWaitEvent(st, s->ev_up[p], 0));
    if ((rc = encode_impl(s, s->prgb[p], 1, frame, st, s->ev_conv[p]))) return rc;
    const size_t nblk = (size_t)s->mbw * s->mbh, tb = nblk * sizeof(evxg_block_desc),
                 sb = nblk * sizeof(evxg_sao_info), lb = s->plane_elems * sizeof(int16_t);
    uint8_t *sn = s->snap[p];
    CK(cudaStreamWaitEvent(st, s->ev_free[p], 0));
    CK(cudaMemcpyAsync(sn, s->bt, tb, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(sn + tb, s->prev_ser, tb, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(sn + 2 * tb, s->sao, sb, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(sn + 2 * tb + sb, s->lev, lb, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(sn + 2 * tb + sb + lb, s->sync + 3 * s->mbh + 4, sizeof(int), cudaMemcpyDeviceToDevice, st));
    CK(cudaEventRecord(s->ev_snap[p], st));
    CK(cudaStreamWaitEvent(dn, s->ev_snap[p], 0));
    if (blocks) CK(cudaMemcpyAsync(blocks, sn, tb, cudaMemcpyDeviceToHost, dn));
    if (prev_blocks) CK(cudaMemcpyAsync(prev_blocks, sn + tb, tb, cudaMemcpyDeviceToHost, dn));
    if (sao) CK(cudaMemcpyAsync(sao, sn + 2 * tb, sb, cudaMemcpyDeviceToHost, dn));
    if (levels) CK(cudaMemcpyAsync(levels, sn + 2 * tb + sb, lb, cudaMemcpyDeviceToHost, dn));
    CK(cudaMemcpyAsync(&s->herr[k], sn + 2 * tb + sb + lb, sizeof(int), cudaMemcpyDeviceToHost, dn));
    CK(cudaEventRecord(s->ev_free[p], dn));
    CK(cudaEventRecord(s->done[k], dn));
    s->tickets.store(t + 1);
    *ticket = t;
    return EVXG_SUCCESS;
}

int evxg_stream_output_wait(evxg_stream *s, uint64_t ticket)
{
    const uint64_t issued = s ? s->tickets.load() : 0;
    if (!s || ticket >= issued || issued - ticket > (uint64_t)evxg_stream::kRing)
        return fail(EVXG_ERROR_INVALID_INDEX, "evxg_stream_output_wait: not one of the last 16 pipelined frames");
    const int k = (int)(ticket % evxg_stream::kRing);
    CK(cudaEventSynchronize(s->done[k]));
    if (s->herr[k]) return fail(s->herr[k], "evxg_stream_output_wait: the frame's wavefront gave up waiting (timeout)");
    return EVXG_SUCCESS;
}

int evxg_stream_profile(evxg_stream *s, int enable)
{
    if (!s) return EVXG_ERROR_INVALIDARG;
    if (enable && !s->profile)
        for (int i = 0; i < 7; i++) CK(cudaEventCreate(&s->ev[i]));
    if (!enable && s->profile)
        for (int i = 0; i < 7; i++) cudaEventDestroy(s->ev[i]);
    s->profile = enable != 0;
    return EVXG_SUCCESS;
}

int evxg_stream_kernel_ms(evxg_stream *s, float *out, uint32_t n)
{
    if (!s || !out) return -EVXG_ERROR_INVALIDARG;
    if (!s->profile) return 0;
    if (cudaEventSynchronize(s->ev[6]) != cudaSuccess) return -EVXG_ERROR_EXECUTION_FAILURE;
    uint32_t k = 0;
    for (; k < n && k < 6; k++)
        if (cudaEventElapsedTime(&out[k], s->ev[k], s->ev[k + 1]) != cudaSuccess) return -EVXG_ERROR_EXECUTION_FAILURE;
    return (int)k;
}

int evxg_stream_sync(evxg_stream *s, void *cuda_stream)
{
    if (!s) return EVXG_ERROR_INVALIDARG;
    CK(cudaStreamSynchronize((cudaStream_t)cuda_stream));
    int err = 0;
    CK(cudaMemcpy(&err, s->sync + 3 * s->mbh + 4, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) {
        CK(cudaMemset(s->sync + 3 * s->mbh + 4, 0, sizeof(int)));
        return fail(err, "device wavefront gave up waiting (timeout)");
    }
    return EVXG_SUCCESS;
}

static int copy_out(void *dst, const void *src, size_t n, int to_device, cudaStream_t st)
{
    if (!dst) return EVXG_SUCCESS;
    CK(cudaMemcpyAsync(dst, src, n, to_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
    return EVXG_SUCCESS;
}

int evxg_fetch_tables(evxg_stream *s, evxg_block_desc *blocks, evxg_block_desc *prev_blocks, evxg_sao_info *sao,
                      int16_t *levels, int to_device, void *cuda_stream)
{
    if (!s) return EVXG_ERROR_INVALIDARG;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    const size_t nblk = (size_t)s->mbw * s->mbh;
    int rc;
    if ((rc = copy_out(blocks, s->bt, nblk * sizeof(evxg_block_desc), to_device, st))) return rc;
    if ((rc = copy_out(prev_blocks, s->prev_ser, nblk * sizeof(evxg_block_desc), to_device, st))) return rc;
    if ((rc = copy_out(sao, s->sao, nblk * sizeof(evxg_sao_info), to_device, st))) return rc;
    if ((rc = copy_out(levels, s->lev, s->plane_elems * sizeof(int16_t), to_device, st))) return rc;
    if (!to_device) return evxg_stream_sync(s, cuda_stream);
    return EVXG_SUCCESS;
}

int evxg_fetch_planes(evxg_stream *s, uint32_t slot, int16_t *out, int to_device, void *cuda_stream)
{
    if (!s || !out) return EVXG_ERROR_INVALIDARG;
    if (slot > 4) return fail(EVXG_ERROR_INVALID_INDEX, "evxg_fetch_planes: slot must be 0..3 (DPB) or 4 (source)");
    int rc = copy_out(out, slot == 4 ? s->src : s->dpb[slot], s->plane_elems * sizeof(int16_t), to_device,
                      (cudaStream_t)cuda_stream);
    if (rc) return rc;
    if (!to_device) return evxg_stream_sync(s, cuda_stream);
    return EVXG_SUCCESS;
}

}  // extern "C"

// ------------------------------------------------------------------ GOP encoder
// Mirrors evx3_encoder_impl with EVX_ENABLE_B_FRAMES 1, EVX_B_FRAME_COUNT 3 and
// EVX_PERIODIC_INTRA_RATE 3600 (config.h:41, :120-121): frame types, display
// order, DPB slot assignment (common.cpp:256-283) and the hierarchical
// P / reference-B / B reorder (evx3enc.cpp:279-383); or, configured without
// B frames, its I/P path (evx3enc.cpp:137-160).
struct evxg_encoder {
    evxg_frame_callback cb = nullptr;
    void *user = nullptr;
    evxg_config cfg{};
    evxg_stream *stream = nullptr;
    evxg_frame frame{};                 // the running frame state (clear_frame, common.cpp:48-66)
    uint32_t width = 0, height = 0;
    struct Buf { std::vector<uint8_t> px; uint32_t display_order; };
    Buf reorder[4];
    uint32_t reorder_count = 0, display_counter = 0, ip_index = 0;
    bool first = true;
    std::vector<evxg_block_desc> h_bt, h_prev;
    std::vector<evxg_sao_info> h_sao;
    std::vector<int16_t> h_lev;
    // Where a frame goes once its place in encode order is known: encoded at
    // once on the encoder's own stream, or handed to a sink (the server queues
    // it for a batched tick; the encoder then has no stream of its own).
    evxg::FrameSink sink = nullptr;
    void *sink_ctx = nullptr;
    // Bitstream output (evxg_encoder_set_output): the stream's bytes in order.
    evxg_bytes_callback out_cb = nullptr;
    void *out_user = nullptr;
    bool header_done = false;
    std::vector<uint8_t> slice;
};

void evxg::encoder_set_sink(evxg_encoder *e, FrameSink sink, void *ctx) { e->sink = sink; e->sink_ctx = ctx; }

static const uint32_t kBFrames = 3, kIntraRate = 3600;
static uint8_t ip_slot(uint32_t ip) { return (uint8_t)(ip % 2); }

static void clear_frame(evxg_frame &f)
{
    f = evxg_frame{};
    f.type = EVXG_FRAME_INTRA;
    f.quality = 8;   // EVX_DEFAULT_QUALITY_LEVEL
}

static int encode_one(evxg_encoder *e, const uint8_t *px, const evxg_frame &f)
{
    int rc = evxg_encode_frame(e->stream, px, 0, &f, nullptr);
    if (rc) return rc;
    rc = evxg_fetch_tables(e->stream, e->h_bt.data(), e->h_prev.data(), e->h_sao.data(), e->h_lev.data(), 0, nullptr);
    if (rc) return rc;
    if (e->cb) e->cb(e->user, &f, e->h_bt.data(), e->h_prev.data(), e->h_sao.data(), e->h_lev.data());
    if (e->out_cb) {   // the reference's bytes for this frame (evx3enc.cpp:137-160, :249-277)
        if (!e->header_done) {
            uint8_t h[14];
            if ((rc = evxg_stream_header(&e->cfg, e->width, e->height, h))) return rc;
            e->out_cb(e->out_user, h, sizeof h);
            e->header_done = true;
        }
        const size_t fb = e->cfg.b_frames ? sizeof(evxg_frame) : 10, pre = e->cfg.b_frames ? 4 : 0;
        if (e->slice.size() < (size_t)e->stream->W * e->stream->H * 4) e->slice.resize((size_t)e->stream->W * e->stream->H * 4);
        uint64_t n = 0;
        rc = evxg_serialize_slice(&e->cfg, e->stream->W, e->stream->H, &f, e->h_bt.data(), e->h_prev.data(),
                                  e->h_sao.data(), e->h_lev.data(), e->slice.data() + pre + fb, e->slice.size() - pre - fb, &n);
        if (rc) return rc;
        if (pre) {   // default build: a 4-byte size before the frame record
            const uint32_t size = (uint32_t)(fb + n);
            memcpy(e->slice.data(), &size, 4);
        }
        memcpy(e->slice.data() + pre, &f, fb);   // evx_frame of the build: the first fb bytes
        e->out_cb(e->out_user, e->slice.data(), pre + fb + n);
    }
    return EVXG_SUCCESS;
}

static int emit(evxg_encoder *e, const uint8_t *px, const evxg_frame &f)
{
    return e->sink ? e->sink(e->sink_ctx, px, e->width, e->height, &f) : encode_one(e, px, f);
}

static int encode_gop(evxg_encoder *e)   // evx3enc.cpp:279-383
{
    const uint32_t p_idx = e->reorder_count - 1;
    evxg_frame p = e->frame;
    p.type = EVXG_FRAME_INTER;
    p.display_order = e->reorder[p_idx].display_order;
    p.dpb_slot = ip_slot(e->ip_index);
    p.is_reference = 1;
    p.ref_slot_fwd = ip_slot(e->ip_index - 1);
    p.ref_slot_bwd = 0;
    int rc = emit(e, e->reorder[p_idx].px.data(), p);
    if (rc) return rc;
    e->frame.index++;
    const uint32_t b_count = e->reorder_count - 1;
    if (b_count > 0) {
        const uint32_t ref_b = b_count / 2;
        evxg_frame b = e->frame;
        b.type = EVXG_FRAME_BIDIR;
        b.display_order = e->reorder[ref_b].display_order;
        b.dpb_slot = 2;
        b.is_reference = 1;
        b.ref_slot_fwd = ip_slot(e->ip_index - 1);
        b.ref_slot_bwd = ip_slot(e->ip_index);
        b.quality = (uint16_t)std::min<int>(e->frame.quality + 1, 31);
        if ((rc = emit(e, e->reorder[ref_b].px.data(), b))) return rc;
        e->frame.index++;
        for (uint32_t bi = 0; bi < b_count; bi++) {
            if (bi == ref_b) continue;
            evxg_frame nb = e->frame;
            nb.type = EVXG_FRAME_BIDIR;
            nb.display_order = e->reorder[bi].display_order;
            nb.dpb_slot = 3;
            nb.is_reference = 0;
            nb.quality = (uint16_t)std::min<int>(e->frame.quality + 2, 31);
            if (bi < ref_b) { nb.ref_slot_fwd = ip_slot(e->ip_index - 1); nb.ref_slot_bwd = 2; }
            else { nb.ref_slot_fwd = 2; nb.ref_slot_bwd = ip_slot(e->ip_index); }
            if ((rc = emit(e, e->reorder[bi].px.data(), nb))) return rc;
            e->frame.index++;
        }
    }
    e->ip_index++;
    e->frame.type = EVXG_FRAME_INTER;
    e->reorder_count = 0;
    return EVXG_SUCCESS;
}

extern "C" {

int evxg_encoder_create(evxg_frame_callback cb, void *user, evxg_encoder **out)
{
    return evxg_encoder_create_config(cb, user, nullptr, out);
}

int evxg_encoder_create_config(evxg_frame_callback cb, void *user, const evxg_config *cfg, evxg_encoder **out)
{
    if (!out) return EVXG_ERROR_INVALIDARG;
    evxg_config c;
    evxg_config_default(&c);
    if (cfg) {
        const int rc = check_config(cfg, "evxg_encoder_create_config");
        if (rc) return rc;
        c = *cfg;
    }
    evxg_encoder *e = new evxg_encoder();
    e->cb = cb; e->user = user; e->cfg = c;
    clear_frame(e->frame);
    *out = e;
    return EVXG_SUCCESS;
}

int evxg_encoder_clear(evxg_encoder *e)   // evx3enc.cpp:35-55
{
    if (!e) return EVXG_ERROR_INVALIDARG;
    if (e->stream) evxg_stream_destroy(e->stream);
    e->stream = nullptr;
    e->header_done = false;   // the next frame starts a new stream
    clear_frame(e->frame);
    e->reorder_count = 0; e->display_counter = 0; e->ip_index = 0; e->first = true;
    return EVXG_SUCCESS;
}

int evxg_encoder_destroy(evxg_encoder *e)
{
    if (!e) return EVXG_ERROR_INVALIDARG;
    evxg_encoder_clear(e);
    delete e;
    return EVXG_SUCCESS;
}

int evxg_encoder_insert_intra(evxg_encoder *e)
{
    if (!e) return EVXG_ERROR_INVALIDARG;
    e->frame.type = EVXG_FRAME_INTRA;
    return EVXG_SUCCESS;
}

int evxg_encoder_set_quality(evxg_encoder *e, uint8_t q)   // evx3enc.cpp:64-82
{
    if (!e) return EVXG_ERROR_INVALIDARG;
    int qq = std::min(std::max((int)q, 1), 31);
    int qp = qq <= 16 ? qq : qq + ((qq - 16) * (qq - 16)) / 10;
    e->frame.quality = (uint16_t)std::min(qp, 63);
    return EVXG_SUCCESS;
}

evxg_stream *evxg_encoder_stream(evxg_encoder *e) { return e ? e->stream : nullptr; }

int evxg_encoder_set_output(evxg_encoder *e, evxg_bytes_callback cb, void *user)
{
    if (!e) return fail(EVXG_ERROR_INVALIDARG, "evxg_encoder_set_output: null encoder");
    if (e->sink) return fail(EVXG_ERROR_INVALID_RESOURCE, "evxg_encoder_set_output: a served stream's encoder has no output");
    e->out_cb = cb;
    e->out_user = user;
    return EVXG_SUCCESS;
}

int evxg_encoder_encode(evxg_encoder *e, const uint8_t *rgb, uint32_t width, uint32_t height)
{
    if (!e || !rgb || !width || !height) return fail(EVXG_ERROR_INVALIDARG, "evxg_encoder_encode: bad argument");
    int rc;
    if (e->sink && !e->width) {   // frames go to the sink: no stream of its own
        e->width = width; e->height = height;
        e->reorder_count = 0; e->display_counter = 0; e->ip_index = 0; e->first = true;
    }
    if (!e->stream && !e->sink) {
        if ((rc = evxg_stream_create_config(width, height, &e->cfg, &e->stream))) return rc;
        e->width = width; e->height = height;
        const size_t nblk = (size_t)e->stream->mbw * e->stream->mbh;
        e->h_bt.resize(nblk); e->h_prev.resize(nblk); e->h_sao.resize(nblk);
        e->h_lev.resize(e->stream->plane_elems);
        e->reorder_count = 0; e->display_counter = 0; e->ip_index = 0; e->first = true;
    }
    if (width != e->width || height != e->height)
        return fail(EVXG_ERROR_INVALID_RESOURCE, "evxg_encoder_encode: frame size changed within a stream");
    if (!e->cfg.b_frames) {   // I/P: every frame as it arrives (evx3enc.cpp:137-160)
        const uint32_t R = e->cfg.ref_count;
        evxg_frame f = e->frame;
        f.display_order = e->display_counter++;
        f.is_reference = 1;
        f.dpb_slot = (uint8_t)(f.index % R);
        f.ref_slot_fwd = (uint8_t)((f.index + R - 1) % R);
        f.ref_slot_bwd = 0;
        if ((rc = emit(e, rgb, f))) return rc;
        e->frame.type = EVXG_FRAME_INTER;
        if ((e->frame.index + 1) % kIntraRate == 0) e->frame.type = EVXG_FRAME_INTRA;   // periodic intra
        e->frame.index++;
        return EVXG_SUCCESS;
    }
    if (e->display_counter > 0 && e->display_counter % kIntraRate == 0) {   // periodic intra
        if (e->reorder_count > 0 && (rc = encode_gop(e))) return rc;
        e->frame.type = EVXG_FRAME_INTRA;
        e->ip_index = 0;
    }
    const bool as_intra = e->frame.type == EVXG_FRAME_INTRA;
    if (as_intra && !e->first && e->reorder_count > 0) {
        if ((rc = encode_gop(e))) return rc;
        e->ip_index = 0;
    }
    evxg_encoder::Buf &b = e->reorder[e->reorder_count];
    b.px.assign(rgb, rgb + (size_t)width * height * 3);
    b.display_order = e->display_counter;
    e->reorder_count++;
    e->display_counter++;
    if (e->first || as_intra) {
        e->first = false;
        e->frame.type = EVXG_FRAME_INTRA;
        evxg_frame i = e->frame;
        i.display_order = e->reorder[0].display_order;
        i.dpb_slot = ip_slot(e->ip_index);
        i.is_reference = 1;
        i.ref_slot_fwd = 0;
        i.ref_slot_bwd = 0;
        if ((rc = emit(e, e->reorder[0].px.data(), i))) return rc;
        e->ip_index++;
        e->frame.type = EVXG_FRAME_INTER;
        e->frame.index++;
        e->reorder_count = 0;
    } else if (e->reorder_count == kBFrames + 1) {
        if ((rc = encode_gop(e))) return rc;
    }
    return EVXG_SUCCESS;
}

int evxg_encoder_peek(evxg_encoder *e, int which, uint8_t *rgb)   // evx3enc.cpp:417-547
{
    if (!e || !rgb) return fail(EVXG_ERROR_INVALIDARG, "evxg_encoder_peek: null argument");
    if (!e->stream) return EVXG_SUCCESS;   // nothing encoded yet (evx3enc.cpp:428-431)
    if (which < EVXG_PEEK_SOURCE || which > EVXG_PEEK_DESTINATION || which == EVXG_PEEK_PREDICTION)
        return fail(EVXG_ERROR_NOTIMPL, "evxg_encoder_peek: not a view the reference draws");
    evxg_stream *s = e->stream;
    const int16_t *planes = nullptr;
    if (which == EVXG_PEEK_SOURCE) {
        planes = s->src;
    } else if (which == EVXG_PEEK_DESTINATION) {   // evx3enc.cpp:444-452
        const uint32_t R = e->cfg.ref_count;
        planes = s->dpb[e->cfg.b_frames ? e->frame.dpb_slot % 4 : (e->frame.index + R - 1) % R];
    }
    // the stream's RGB staging buffer is free between frames; the encoder's work is on the legacy stream
    int rc = peek_rgb(planes, s->bt, which, (int)s->W, (int)s->H, (int)s->mbw, (int)s->vw, (int)s->vh, s->rgb, nullptr);
    if (rc) return rc;
    CK(cudaMemcpy(rgb, s->rgb, (size_t)s->vw * s->vh * 3, cudaMemcpyDeviceToHost));
    return evxg_stream_sync(s, nullptr);
}

int evxg_encoder_flush(evxg_encoder *e)   // evx3enc.cpp:385-414
{
    if (!e) return EVXG_ERROR_INVALIDARG;
    if (e->reorder_count == 0) return EVXG_SUCCESS;
    int rc;
    if (e->reorder_count == 1) {
        evxg_frame p = e->frame;
        p.type = EVXG_FRAME_INTER;
        p.display_order = e->reorder[0].display_order;
        p.dpb_slot = ip_slot(e->ip_index);
        p.is_reference = 1;
        p.ref_slot_fwd = ip_slot(e->ip_index - 1);
        p.ref_slot_bwd = 0;
        if ((rc = emit(e, e->reorder[0].px.data(), p))) return rc;
        e->frame.index++;
        e->ip_index++;
    } else if ((rc = encode_gop(e))) {
        return rc;
    }
    e->reorder_count = 0;
    return EVXG_SUCCESS;
}

}  // extern "C"
