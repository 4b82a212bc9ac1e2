// evxg_internal.cuh -- host-side internals shared by the C ABI translation
// units (evxg_api.cu: streams, frames, GOP encoder; evxg_batch.cu: batched
// ticks): the per-stream device state, the kernels they launch, error helpers.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <string>

#include "evxg.h"
#include "evxg_device.cuh"

namespace evxg {
__global__ void k_convert(FrameArgs a);
__global__ void k_mb_wavefront(FrameArgs a);
__global__ void k_mb_cluster(FrameArgs a);
__global__ void k_deblock(FrameArgs a);
__global__ void k_sao_rdo(FrameArgs a);
__global__ void k_sao_merge(FrameArgs a);
__global__ void k_sao_fix(FrameArgs a, int pass);
__global__ void k_sao_restore(FrameArgs a, int last_pass);
__global__ void k_sao_apply(FrameArgs a, int last_pass);
// batched forms (blockIdx.z = stream; the MB kernels take the tick's row queue)
__global__ void k_convert_b(const FrameArgs *args);
__global__ void k_mb_wavefront_b(const FrameArgs *args, const int2 *queue, const int *qlen, int *qctr);
__global__ void k_mb_cluster_b(const FrameArgs *args, const int2 *queue, const int *qlen, int *qctr);
__global__ void k_deblock_b(const FrameArgs *args);
__global__ void k_sao_rdo_b(const FrameArgs *args);
__global__ void k_sao_merge_b(const FrameArgs *args);
__global__ void k_sao_fix_b(const FrameArgs *args, int pass);
__global__ void k_sao_restore_b(const FrameArgs *args, int last_pass);
__global__ void k_sao_apply_b(const FrameArgs *args, int last_pass);
__global__ void k_tick_prep_b(const FrameArgs *args, int sao_passes);
__global__ void k_sao_copy_b(const FrameArgs *args);
__global__ void k_tick_post_b(const FrameArgs *args);
size_t mb_shared_bytes();
int mb_threads();
size_t merge_shared_bytes(int mbw, int mbh);   // dynamic shared memory of k_sao_merge(_b) for an mbw x mbh MB frame
constexpr int kMergeCtas = 8, kMergeThreads = 512;   // the merge kernels: one cluster of 8 CTAs per frame
size_t deblock_shared_bytes(int W);   // dynamic shared memory of k_deblock(_b) for an aligned width W
constexpr int kDeblockCtas = 3 * 8, kDeblockThreads = 256;   // 8 column strips (one cluster) per plane

// Fixed-point passes of the SAO application (evxg_filters.cu); the chains they
// resolve are a few pixels long, the last pass only confirms.
constexpr int kSaoPasses = 8;

int fail(int code, const char *what);
int cuda_fail(cudaError_t e, const char *where);
// Checks a frame descriptor against the stream's configuration and, for
// streams without B frames, derives its DPB slots from the index (out may be
// the same as f).
int check_frame(const evxg_stream *s, const evxg_frame *f, const char *who, evxg_frame *out);
int check_frame_config(const evxg_config &cfg, const evxg_frame *f, const char *who, evxg_frame *out);
// A build configuration the library reproduces (EVXG_ERROR_INVALIDARG otherwise).
int check_config(const evxg_config *c, const char *who);
int max_active_clusters();
// RGB24 of an int16 plane set (EVXG_PEEK_SOURCE / _DESTINATION) or one of the
// block-table maps of the encoder's peek() into device memory out (w x h).
int peek_rgb(const int16_t *planes, const evxg_block_desc *bt, int which, int W, int H, int mbw, int w, int h,
             uint8_t *out, cudaStream_t st);
}  // namespace evxg

#define CK(call)                                                     \
    do {                                                             \
        cudaError_t e_ = (call);                                     \
        if (e_ != cudaSuccess) return evxg::cuda_fail(e_, #call);    \
    } while (0)

struct evxg_stream {
    uint32_t vw, vh, W, H, mbw, mbh;
    size_t plane_elems;                 // elements of one plane set
    int16_t *src, *lev, *dpb[4];
    evxg_block_desc *bt, *prev, *prev_ser;
    evxg_sao_info *sao;
    int2 *sao_stats;                    // per-MB RDO results for the merge (kSaoStatEntries each)
    int16_t *sao_orig;                  // pristine copy for the SAO fixed-point passes
    int *sao_flags;
    unsigned long long *sao_mail;       // SAO merge hand-over words, epoch-tagged
    int epoch;
    uint8_t *rgb;
    int *sync;                          // 3*mbh progress words, 4 counters, 1 error word
    int mb_grid, num_sms;
    int mb_form, mb_clusters;           // macroblock pass shape; clusters launched in the cluster form
    uint32_t launches;
    long long timeout_ns;
    evxg_config cfg;                    // reference build configuration the stream reproduces
    bool profile;
    cudaEvent_t ev[7];
    // deblocking beside the macroblock pass (cluster form): its stream, and
    // events for "sync words reset" and "deblocking done"
    cudaStream_t aux;
    cudaEvent_t ev_aux[2];
    // Pipelined encoding from host memory (evxg_encode_frame_pipelined), set
    // up on first use: an upload and a download stream, two device RGB
    // buffers and two table snapshots, the events that order uploads / frames
    // / downloads across the three streams, and a ring of per-frame
    // completion events with the frames' error words.
    static constexpr int kRing = 16;
    cudaStream_t copy, down;
    uint8_t *prgb[2], *snap[2];
    cudaEvent_t ev_up[2], ev_conv[2], ev_snap[2], ev_free[2], done[kRing];
    int *herr;                          // pinned, one error word per ring entry
    std::atomic<uint64_t> tickets{0};   // frames issued; read by output waits on other threads
};

namespace evxg {
// Kernel parameters of stream s for frame f (advances the stream's SAO epoch).
void fill_args(evxg_stream *s, const evxg_frame *f, const uint8_t *drgb, FrameArgs &a);
// Return a stream to its state at creation: zero planes and tables, epoch 0.
int reset_stream(evxg_stream *s, cudaStream_t st);
// A GOP-level encoder whose frames, once their encode order is known, go to
// sink(ctx, rgb, width, height, frame) instead of its own stream.
typedef int (*FrameSink)(void *ctx, const uint8_t *rgb, uint32_t width, uint32_t height, const evxg_frame *f);
void encoder_set_sink(evxg_encoder *e, FrameSink sink, void *ctx);
}  // namespace evxg
