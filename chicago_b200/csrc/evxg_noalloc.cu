// evxg_noalloc.cu -- an allocation-free entry point for the macroblock pass.
//
// Some callers cannot allocate device memory at the time they encode: a host
// that manages one fixed device arena itself (a plugin in a media server or a
// capture pipeline that gets all of its buffers from the host application), a
// caller running inside a section where allocation would synchronise the
// device or fail, or one whose memory budget is fixed at start-up.  Such a
// caller already owns every input and output buffer; what the macroblock
// wavefront kernel needs beyond them is a small scratch area (one progress
// word per macroblock row, a row counter and an error word).  Here that
// scratch lives in a fixed array in the library's device image, so this entry
// point calls no allocator at all.
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>

#include "evxg.h"
#include "evxg_device.cuh"

namespace evxg {
__global__ void k_mb_wavefront(FrameArgs a);
size_t mb_shared_bytes();
int mb_threads();
int fail(int code, const char *what);
int cuda_fail(cudaError_t e, const char *where);
}  // namespace evxg

using namespace evxg;

// Scratch words: [0, rows) row progress, then 4 counters, then the error word.
// Every GPU that loads this library holds these 16 KiB until the process exits.
static __device__ __align__(256) int g_noalloc_scratch[EVXG_NOALLOC_MAX_MB_ROWS + 5];

namespace {
constexpr int kMaxDevices = 64;
int *g_scratch_ptr[kMaxDevices];   // device address of g_noalloc_scratch, per device
int g_num_sms[kMaxDevices];
int g_setup_rc[kMaxDevices];
std::once_flag g_setup_once[kMaxDevices];   // callers on several threads may meet a device's first call
std::atomic<long long> g_timeout_ns{5000000000LL};

// Once per device, with that device current: translate the array's host-side
// name into its device address and allow the kernel's shared-memory size.
int setup_device(int dev)
{
    int *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
    if (e == cudaSuccess && !p) e = cudaErrorInvalidSymbol;
    if (e != cudaSuccess) return cuda_fail(e, "evxg_mb_pass_noalloc: scratch address (cudaGetSymbolAddress)");
    e = cudaDeviceGetAttribute(&g_num_sms[dev], cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mb_wavefront, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mb_shared_bytes());
    if (e != cudaSuccess) return cuda_fail(e, "evxg_mb_pass_noalloc: device set-up");
    g_scratch_ptr[dev] = p;
    return EVXG_SUCCESS;
}
}  // namespace

extern "C" int evxg_mb_pass_noalloc_set_timeout_ns(int64_t ns)
{
    if (ns <= 0) return fail(EVXG_ERROR_INVALIDARG, "evxg_mb_pass_noalloc_set_timeout_ns: ns must be > 0");
    g_timeout_ns.store(ns);
    return EVXG_SUCCESS;
}

extern "C" int evxg_mb_pass_noalloc(uint32_t aligned_w, uint32_t aligned_h, const evxg_frame *f, const int16_t *src,
                                    int16_t *const dpb[4], int16_t *levels, evxg_block_desc *blocks,
                                    const evxg_block_desc *prev_blocks, void *cuda_stream)
{
    if (!f || !src || !dpb || !levels || !blocks) return fail(EVXG_ERROR_INVALIDARG, "evxg_mb_pass_noalloc: null argument");
    if (!aligned_w || !aligned_h || (aligned_w & 15) || (aligned_h & 15) || aligned_w > 65520)
        return fail(EVXG_ERROR_INVALIDARG, "evxg_mb_pass_noalloc: aligned size must be a multiple of 16, width <= 65520");
    const uint32_t mbw = aligned_w / 16, mbh = aligned_h / 16;
    if (mbh > EVXG_NOALLOC_MAX_MB_ROWS)
        return fail(EVXG_ERROR_CAPACITY_LIMIT, "evxg_mb_pass_noalloc: more macroblock rows than the fixed scratch holds");
    if (f->type < EVXG_FRAME_INTRA || f->type > EVXG_FRAME_BIDIR || f->quality < 1 || f->quality > 63)
        return fail(EVXG_ERROR_INVALIDARG, "evxg_mb_pass_noalloc: bad frame type or quality (QP 1..63)");
    if (f->dpb_slot > 3 || f->ref_slot_fwd > 3 || f->ref_slot_bwd > 3)
        return fail(EVXG_ERROR_INVALID_INDEX, "evxg_mb_pass_noalloc: DPB slot out of range");
    if ((f->type != EVXG_FRAME_INTRA && f->ref_slot_fwd == f->dpb_slot) ||
        (f->type == EVXG_FRAME_BIDIR && f->ref_slot_bwd == f->dpb_slot))
        return fail(EVXG_ERROR_INVALIDARG, "evxg_mb_pass_noalloc: a reference equals the destination slot");
    if (f->type == EVXG_FRAME_INTER && !prev_blocks)
        return fail(EVXG_ERROR_INVALIDARG, "evxg_mb_pass_noalloc: P frames need the previous block table");
    for (int i = 0; i < 4; i++)
        if (!dpb[i]) return fail(EVXG_ERROR_INVALIDARG, "evxg_mb_pass_noalloc: null DPB slot");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return fail(EVXG_ERROR_EXECUTION_FAILURE, "evxg_mb_pass_noalloc: no current device");
    std::call_once(g_setup_once[dev], [&] { g_setup_rc[dev] = setup_device(dev); });
    if (g_setup_rc[dev]) return fail(g_setup_rc[dev], "evxg_mb_pass_noalloc: device set-up failed");
    int *scratch = g_scratch_ptr[dev];
    cudaStream_t st = (cudaStream_t)cuda_stream;

    FrameArgs a{};
    a.W = (int)aligned_w; a.H = (int)aligned_h; a.mbw = (int)mbw; a.mbh = (int)mbh;
    a.vis_w = a.W; a.vis_h = a.H;
    a.type = f->type; a.quality = f->quality; a.dpb = f->dpb_slot;
    a.ref_fwd = f->ref_slot_fwd; a.ref_bwd = f->ref_slot_bwd;
    a.nref = 1; a.ref_slot[0] = f->ref_slot_fwd;   // the default build: P frames search the forward slot
    a.lambda = evxg_lambda(f->quality);
    for (int i = 0; i < 4; i++) a.planes[i] = dpb[i];
    a.src = const_cast<int16_t *>(src);
    a.lev = levels;
    a.bt = blocks;
    a.prev = f->type == EVXG_FRAME_INTER ? prev_blocks : nullptr;
    a.progress = scratch;
    a.counters = scratch + mbh;
    a.error = scratch + mbh + 4;
    a.timeout_ns = g_timeout_ns.load();
    // The array keeps whatever the previous call left: progress words start at
    // -1, the row counter and the error word at 0.
    cudaError_t e = cudaMemsetAsync(scratch, 0xFF, mbh * sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(scratch + mbh, 0, 5 * sizeof(int), st);
    if (e != cudaSuccess) return cuda_fail(e, "evxg_mb_pass_noalloc: scratch initialisation");
    const int grid = (int)(mbh < (uint32_t)g_num_sms[dev] ? mbh : (uint32_t)g_num_sms[dev]);
    k_mb_wavefront<<<grid, mb_threads(), mb_shared_bytes(), st>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "evxg_mb_pass_noalloc: launch");
    int err = 0;
    e = cudaMemcpyAsync(&err, scratch + mbh + 4, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "evxg_mb_pass_noalloc: completion");
    if (err) return fail(err, "evxg_mb_pass_noalloc: the wavefront gave up waiting (timeout)");
    return EVXG_SUCCESS;
}
