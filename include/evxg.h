/*
 * evxg.h -- C ABI of the B200 (sm_100a) EVX3 encoder pixel pipeline.
 *
 * The GPU path replaces the reference encoder's per-frame pixel pipeline,
 * engine_encode_frame() minus serialize_slice() (reference
 * src/video/encode.cpp:945-1001): RGB->YUV 4:2:0 conversion, per-macroblock
 * mode decision (intra block copy, inter and bidirectional motion search with
 * 6-tap sub-pel refinement, directional intra, RDO), DCT / adaptive
 * quantisation / trellis, reconstruction, deblocking and SAO.  The outputs are
 * exactly the tables the reference's host entropy coder reads
 * (serialize.cpp:151-314, :564-686): the block table, the previous block
 * table, the SAO table and the quantised level planes, byte-identical to the
 * reference's for the same inputs.
 *
 * Around it, for a drop-in codec: the host entropy coder and decoder
 * (serialize_slice / unserialize_slice), the decoder's pixel half on the GPU
 * (engine_decode_frame after unserialize_slice, decode.cpp:560-612), the GOP
 * level encoder (evx3_encoder), batched and served encoding of many streams,
 * and the packet container (evx_muxer / evx_demuxer, muxer.h:53-160).
 *
 * All entry points return an evx_status-compatible code (reference
 * src/base.h:168-185); no exceptions cross the ABI.  One stream handle is one
 * encoder context (reference evx_context, common.h:209-240); a handle is not
 * thread-safe and needs external synchronisation, like the reference encoder.
 * Pointers are plain host or device pointers; cuda_stream is a cudaStream_t
 * passed as void* (NULL = the legacy default stream).
 */
#ifndef EVXG_H
#define EVXG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: same values as the reference's evx_status (base.h:168-185). */
#define EVXG_SUCCESS              0
#define EVXG_ERROR_INVALIDARG     1
#define EVXG_ERROR_NOTIMPL        2
#define EVXG_ERROR_OUTOFMEMORY    3
#define EVXG_ERROR_INVALID_INDEX  6
#define EVXG_ERROR_CAPACITY_LIMIT 7
#define EVXG_ERROR_INVALID_RESOURCE 8
#define EVXG_ERROR_OPERATION_TIMEDOUT 9
#define EVXG_ERROR_EXECUTION_FAILURE 10
#define EVXG_ERROR_IO_FAILURE     12
#define EVXG_ERROR_NOT_READY      15
#define EVXG_ERROR_OPERATION_COMPLETED 16

/* Frame types (reference types.h:45-53). */
#define EVXG_FRAME_INTRA 0
#define EVXG_FRAME_INTER 1
#define EVXG_FRAME_BIDIR 2

#pragma pack(push, 2)
/* Same byte layout as the reference's evx_frame (common.h:72-87, pack(2), 18 B). */
typedef struct evxg_frame {
    int32_t type;
    uint32_t index;
    uint16_t quality;          /* internal QP, 1..63 (evx3enc.cpp:64-82) */
    uint32_t display_order;
    uint8_t is_reference;
    uint8_t dpb_slot;          /* DPB slot reconstructed into (0..3) */
    uint8_t ref_slot_fwd;
    uint8_t ref_slot_bwd;
} evxg_frame;

/* Same byte layout as the reference's evx_block_desc (common.h:91-115, pack(2), 28 B). */
typedef struct evxg_block_desc {
    int32_t block_type;        /* bit0 intra, bit1 motion, bit2 copy (types.h:63-91) */
    uint8_t prediction_target;
    uint8_t pad0;
    int16_t motion_x;
    int16_t motion_y;
    uint8_t sp_pred;
    uint8_t sp_amount;
    uint8_t sp_index;
    uint8_t q_index;
    uint8_t intra_mode;        /* 0..6 directional, 7 none */
    uint8_t pad1;
    int16_t variance;
    uint8_t prediction_mode;   /* 0 fwd, 1 bwd, 2 bi */
    uint8_t prediction_target_b;
    int16_t motion_x_b;
    int16_t motion_y_b;
    uint8_t sp_pred_b;
    uint8_t sp_amount_b;
    uint8_t sp_index_b;
    uint8_t pad2;
} evxg_block_desc;
#pragma pack(pop)

/* Same byte layout as the reference's evx_sao_params / evx_sao_info (sao.h:66-78, 16 B). */
typedef struct evxg_sao_params {
    uint8_t type;              /* 0 off, 1 edge, 2 band */
    uint8_t eo_class;
    uint8_t band_position;
    int8_t offsets[4];
} evxg_sao_params;
typedef struct evxg_sao_info {
    uint8_t merge_left;
    uint8_t merge_above;
    evxg_sao_params luma;
    evxg_sao_params chroma;
} evxg_sao_info;

typedef struct evxg_stream evxg_stream;

/*
 * The reference's encoder is configured at compile time (src/video/config.h,
 * motion.cpp:29); a stream reproduces one such build, chosen when it is
 * created:
 *   b_frames      EVX_ENABLE_B_FRAMES (config.h:120).  1 (default): the
 *                 hierarchical P / reference-B / B GOP (evx3enc.cpp:167-383),
 *                 frames carry their DPB slots in evxg_frame.  0: an I/P GOP
 *                 encoded in arrival order (evx3enc.cpp:137-160); the slots
 *                 follow from evxg_frame.index (query_prediction_index_by_offset,
 *                 common.cpp:256-259; the slot fields are ignored) and each P
 *                 frame searches the references at offsets 1 .. ref_count-1,
 *                 its descriptors naming the offset (encode.cpp:211-247).  The
 *                 reference's evx_frame / evx_block_desc of such a build are the
 *                 first 10 / 18 bytes of evxg_frame / evxg_block_desc.
 *   ref_count     EVX_REFERENCE_FRAME_COUNT (config.h:39): 4 with B frames;
 *                 2 (one reference) or 4 (three) without.
 *   search_radius EVX_MOTION_SEARCH_RADIUS (motion.cpp:29): 16.
 * Other combinations are refused with EVXG_ERROR_INVALIDARG.
 */
typedef struct evxg_config {
    uint8_t b_frames;
    uint8_t ref_count;
    uint8_t search_radius;
    uint8_t reserved;          /* 0 */
} evxg_config;
/* The default build: b_frames 1, ref_count 4, search_radius 16. */
void evxg_config_default(evxg_config *cfg);

/*
 * Create the device state of one encoding stream for frames of width x height
 * (visible size; the context is 16-aligned like initialize_context,
 * common.cpp:106-202): source, level and 4 DPB plane sets, block / previous
 * block / SAO tables, all zero-initialised.  Replaces evx3_encoder_impl::
 * initialize (evx3enc.cpp:84-103) on the device side.
 */
int evxg_stream_create(uint32_t width, uint32_t height, evxg_stream **out);
/* The same for the build cfg describes (NULL = the default build). */
int evxg_stream_create_config(uint32_t width, uint32_t height, const evxg_config *cfg, evxg_stream **out);
int evxg_stream_config(const evxg_stream *s, evxg_config *out);
int evxg_stream_destroy(evxg_stream *s);

/* Aligned context size and macroblock grid of a stream. */
int evxg_stream_dims(const evxg_stream *s, uint32_t *aligned_w, uint32_t *aligned_h,
                     uint32_t *mb_w, uint32_t *mb_h);

/*
 * engine_encode_frame minus serialize_slice (encode.cpp:945-998): convert the
 * packed RGB24 frame (width*height*3 bytes; rgb_on_device != 0 if it is a
 * device pointer), run the macroblock wavefront (classify, encode, reconstruct
 * into DPB[frame->dpb_slot]), deblock, SAO, and update the previous block
 * table for non-B frames.  Asynchronous on cuda_stream.  frame is the
 * reference's evx_frame as chosen by its GOP logic (evx3enc.cpp:105-414).
 */
int evxg_encode_frame(evxg_stream *s, const uint8_t *rgb, int rgb_on_device,
                      const evxg_frame *frame, void *cuda_stream);

/*
 * Copy the tables the host serializer reads (serialize_slice,
 * serialize.cpp:624-686) to host or device memory (to_device != 0).  Any
 * pointer may be NULL.  Plane sets are int16, Y (aw*ah) then U then V
 * ((aw/2)*(ah/2) each).  The previous block table returned is the one the
 * serializer of the frame just encoded must see, i.e. as it was BEFORE that
 * frame's update (encode.cpp:985-998 serializes before the copy).
 */
int evxg_fetch_tables(evxg_stream *s, evxg_block_desc *blocks, evxg_block_desc *prev_blocks,
                      evxg_sao_info *sao, int16_t *levels, int to_device, void *cuda_stream);

/* Pipelined encoding from host memory (no counterpart in the reference):
 * evxg_encode_frame plus evxg_fetch_tables for one frame, returning at once,
 * with the copies off the frame's critical path -- the RGB upload runs on
 * an upload stream of the stream's own while earlier frames compute, the
 * frame's tables are snapshotted on the device when its kernels end and
 * downloaded on a download stream while the next frame computes.  Frames run in call
 * order on cuda_stream like evxg_encode_frame; results are identical.
 * *ticket names the frame: evxg_stream_output_wait(s, ticket) returns once
 * its tables are in the host buffers (any of which may be NULL), with the
 * frame's error (EVXG_ERROR_OPERATION_TIMEDOUT) if a wait gave up.  rgb and
 * the output buffers must stay valid until then (pinned memory keeps the
 * copies asynchronous); at most the last 16 frames can be waited for, and a
 * 17th call waits for the oldest itself. */
int evxg_encode_frame_pipelined(evxg_stream *s, const uint8_t *rgb, const evxg_frame *frame, evxg_block_desc *blocks,
                                evxg_block_desc *prev_blocks, evxg_sao_info *sao, int16_t *levels, void *cuda_stream,
                                uint64_t *ticket);
int evxg_stream_output_wait(evxg_stream *s, uint64_t ticket);

/* Copy one DPB slot (plane-set layout) or the converted source
 * (slot = 4) out; supports the reference's peek() views (evx3enc.cpp:417-547). */
int evxg_fetch_planes(evxg_stream *s, uint32_t slot, int16_t *out, int to_device, void *cuda_stream);

/* Wait for the stream's work; returns the device error word if a kernel gave
 * up waiting (EVXG_ERROR_OPERATION_TIMEDOUT) or a launch failed. */
int evxg_stream_sync(evxg_stream *s, void *cuda_stream);

/* Failure detection (no counterpart in the reference, whose WPP threads wait
 * for each other without a bound, encode.cpp:866-877).  Every wait of a
 * stream's kernels on other CTAs -- wavefront progress, the cluster form's
 * hand-over, the SAO merge and raster-order application -- gives up after
 * timeout_ns, sets the stream's device error word and lets every CTA of the
 * frame run to its end; evxg_stream_sync (and evxg_fetch_* with host
 * destinations) then return EVXG_ERROR_OPERATION_TIMEDOUT and clear the
 * word.  The frame's results and the stream's reference state are undefined
 * after that: evxg_stream_reset returns the stream to its state at creation
 * (what the reference's clear() does to its context, evx3enc.cpp:35-55), so
 * the next frame should be an intra frame.  The default bound is 5 s;
 * ns must be > 0. */
int evxg_stream_set_timeout_ns(evxg_stream *s, int64_t ns);
int evxg_stream_reset(evxg_stream *s, void *cuda_stream);

/* Checkpoint of a stream (the device half of the reference's evx_context,
 * common.h:209-240; the GOP state lives with the caller or the GOP encoder):
 * evxg_stream_save copies everything later frames read -- the DPB slots, the
 * level planes (copy blocks keep stale levels that later DC prediction
 * reads), the temporal predictor and block tables, the SAO epoch -- into
 * evxg_stream_state_bytes(s) bytes of host memory; evxg_stream_restore loads
 * it into a stream of the same size and build, after which the stream's next
 * frames are bit-identical to those of the stream it was saved from.  Both
 * wait for their copies. */
uint64_t evxg_stream_state_bytes(const evxg_stream *s);
int evxg_stream_save(evxg_stream *s, void *host, uint64_t capacity, void *cuda_stream);
int evxg_stream_restore(evxg_stream *s, const void *host, uint64_t size, void *cuda_stream);

/* Number of kernels launched by the last evxg_encode_frame call. */
uint32_t evxg_last_launch_count(const evxg_stream *s);

/* Shape of the macroblock pass (no counterpart in the reference, whose WPP
 * runs one thread per macroblock row):
 *   EVXG_MB_FORM_CLUSTER  a cluster of three CTAs per macroblock row (intra
 *                         block-copy search and decision / forward search /
 *                         backward search and directional intra on separate
 *                         SMs): the lowest latency per frame; the default
 *                         when the device can co-schedule such clusters.
 *   EVXG_MB_FORM_SINGLE   one CTA per row (the searches share it as warp
 *                         groups): a third of the SMs per row, the higher
 *                         throughput when many streams share the GPU.
 * Both give identical output.  evxg_stream_set_mb_form returns
 * EVXG_ERROR_INVALID_RESOURCE if the cluster form cannot run on this device;
 * evxg_stream_mb_form reports the current form. */
#define EVXG_MB_FORM_SINGLE  0
#define EVXG_MB_FORM_CLUSTER 1
int evxg_stream_set_mb_form(evxg_stream *s, int form);
int evxg_stream_mb_form(const evxg_stream *s);

/* Kernel timing (no counterpart in the reference, which has no device work):
 * when enabled, evxg_encode_frame records a CUDA event around each of its
 * kernels; evxg_stream_kernel_ms waits for the last frame and writes up to n
 * durations in milliseconds, in launch order: convert, macroblock wavefront,
 * deblock, SAO RDO, SAO merge, SAO apply.  Returns the number written. */
int evxg_stream_profile(evxg_stream *s, int enable);
int evxg_stream_kernel_ms(evxg_stream *s, float *out_ms, uint32_t n);

/* ---- Batched encoding ----
 *
 * No counterpart in the reference, which encodes one stream per evx3_encoder
 * (evx3enc.cpp:105-414).  A batch holds n streams of any sizes; each tick
 * advances every stream that has a frame by that one frame, with one kernel
 * launch per pipeline stage for all of them (the macroblock pass claims
 * (stream, row) items from one queue), the tick replayed as a CUDA graph.
 * Every stream's output equals encoding it alone with evxg_encode_frame.
 *
 * Host buffers come in two parities (0, 1), so the host prepares tick t+1
 * while the device runs tick t: write stream i's RGB24 frame into
 * evxg_batch_input(b, i, p), call evxg_batch_encode(b, frames, p, stream),
 * and after evxg_batch_wait(b, p) read stream i's tables (the inputs of the
 * reference serializer, as evxg_fetch_tables returns them) from
 * evxg_batch_output.  Before rewriting parity p's inputs, wait for parity p.
 * frames[i].type < 0 means stream i has no frame in this tick.  The streams
 * stay owned by the caller and must not be used outside the batch while it
 * exists. */
typedef struct evxg_batch evxg_batch;
int evxg_batch_create(evxg_stream *const *streams, uint32_t n, evxg_batch **out);
int evxg_batch_destroy(evxg_batch *b);
uint8_t *evxg_batch_input(evxg_batch *b, uint32_t i, uint32_t parity);
int evxg_batch_encode(evxg_batch *b, const evxg_frame *frames, uint32_t parity, void *cuda_stream);
int evxg_batch_wait(evxg_batch *b, uint32_t parity);
int evxg_batch_output(evxg_batch *b, uint32_t i, uint32_t parity, const evxg_block_desc **blocks,
                      const evxg_block_desc **prev_blocks, const evxg_sao_info **sao, const int16_t **levels);
/* The wait bound of the batch's ticks (see evxg_stream_set_timeout_ns); one
 * wait that gives up fails the whole tick (evxg_batch_wait returns
 * EVXG_ERROR_OPERATION_TIMEDOUT) and leaves every stream of it to be reset. */
int evxg_batch_set_timeout_ns(evxg_batch *b, int64_t ns);
/* Kernels one tick launches (the same for any number of streams). */
uint32_t evxg_batch_launch_count(const evxg_batch *b);
/* Shape of the tick's macroblock pass: form (EVXG_MB_FORM_*), persistent grid
 * (CTAs, or clusters in the cluster form; capped at what is co-resident) and
 * queue order (0: rows interleaved by index; 1: the same, longer remaining
 * critical path first).  A new batch takes the shape a model of the tick
 * favours (the longer of the longest critical path and all MBs over the
 * working units, per form).  evxg_batch_autotune times the candidates on a short
 * synthetic I/P/B sequence at the streams' sizes, keeps the fastest, and
 * returns every stream to its initial state; best_ms (optional) receives the
 * winner's time for the three timed ticks. */
int evxg_batch_set_shape(evxg_batch *b, int form, int grid, int policy);
int evxg_batch_get_shape(const evxg_batch *b, int *form, int *grid, int *policy);
int evxg_batch_autotune(evxg_batch *b, void *cuda_stream, float *best_ms);

/* ---- Serving ----
 *
 * No counterpart in the reference.  A request loop over many live streams:
 * evxg_server_open admits a stream if a slot is free and its device memory
 * fits what is left of the budget (else EVXG_ERROR_CAPACITY_LIMIT: retry once
 * a stream has closed); its state stays on the device until it closes.
 * evxg_server_submit copies one RGB24 frame in (arrival_ns on the
 * evxg_server_now_ns clock; 0 = now).  Each stream follows the reference
 * encoder's GOP (evx3enc.cpp:105-414), so a frame is ready to encode once the
 * frames it depends on have arrived; each lane's worker thread (see
 * evxg_server_create_lanes) batches whatever of its streams' frames is ready
 * (at most one frame per stream per tick, see Batched encoding) while the
 * previous tick runs, and calls cb on that thread, in each stream's bitstream
 * order (streams of different lanes concurrently), with the frame's
 * serializer inputs (valid during the call) and its times.  evxg_server_close flushes a stream (its last frames are encoded);
 * once they are delivered its memory counts as free for admissions and is
 * released when the next admission rebuilds the batch.  evxg_server_drain
 * waits until every frame that can be encoded has been delivered (and the
 * batch covers every admitted stream).  evxg_server_stats' bytes_in_use counts
 * the streams not yet closed and delivered.  Every stream's results equal encoding
 * it alone with evxg_encoder_*. */
typedef struct evxg_server evxg_server;
typedef struct {
    uint64_t arrival_ns;   /* submitted */
    uint64_t ready_ns;     /* its place in encode order known */
    uint64_t launch_ns;    /* its tick launched */
    uint64_t done_ns;      /* its tick's results seen by the host */
} evxg_frame_times;
typedef void (*evxg_result_callback)(void *user, uint32_t stream_id, const evxg_frame *frame,
                                     const evxg_block_desc *blocks, const evxg_block_desc *prev_blocks,
                                     const evxg_sao_info *sao, const int16_t *levels, const evxg_frame_times *times);
int evxg_server_create(uint64_t hbm_budget_bytes, uint32_t max_streams, evxg_result_callback cb, void *user,
                       evxg_server **out);
/* evxg_server_create spreads the streams over min(max_streams, 8) lanes; this
 * form sets the count (1..max_streams).  A lane is a set of streams with its
 * own worker thread, CUDA stream and batched ticks; a new stream joins the
 * lane whose streams are closest to its size (else an empty lane, else the
 * least loaded), lanes tick independently and their ticks share the device,
 * so a small stream's frames do not wait for a large stream's. */
int evxg_server_create_lanes(uint64_t hbm_budget_bytes, uint32_t max_streams, uint32_t lanes, evxg_result_callback cb,
                             void *user, evxg_server **out);
int evxg_server_destroy(evxg_server *srv);
int evxg_server_open(evxg_server *srv, uint32_t width, uint32_t height, uint8_t quality, uint32_t *stream_id);
/* evxg_server_open for a stream of the build cfg describes (NULL = default). */
int evxg_server_open_config(evxg_server *srv, uint32_t width, uint32_t height, uint8_t quality, const evxg_config *cfg,
                            uint32_t *stream_id);
int evxg_server_submit(evxg_server *srv, uint32_t stream_id, const uint8_t *rgb, uint64_t arrival_ns);
int evxg_server_insert_intra(evxg_server *srv, uint32_t stream_id);
int evxg_server_close(evxg_server *srv, uint32_t stream_id);
int evxg_server_drain(evxg_server *srv);
/* Cancel a stream mid-GOP: frames submitted but not yet in a tick (and those
 * still waiting for their anchor) are dropped without being encoded, frames
 * already in a tick are delivered, and the stream's memory is released like a
 * closed stream's.  The other streams' results are not affected. */
int evxg_server_cancel(evxg_server *srv, uint32_t stream_id);
/* Evict a live stream from the device: its frames already submitted are
 * encoded and delivered, its lane stops ticking it, its device state goes to
 * host memory (evxg_stream_save) and its device memory back to the budget;
 * its GOP planner stays.  While evicted, submit / insert_intra / close return
 * EVXG_ERROR_NOT_READY (cancel drops it).  evxg_server_restore re-admits it
 * within the budget (EVXG_ERROR_CAPACITY_LIMIT otherwise; try again later)
 * and it continues bit-identically.  Its id keeps its stream slot. */
int evxg_server_evict(evxg_server *srv, uint32_t stream_id);
int evxg_server_restore(evxg_server *srv, uint32_t stream_id);
int evxg_server_stats(evxg_server *srv, uint64_t *frames, uint64_t *ticks, uint64_t *rebuilds, uint64_t *bytes_in_use);
uint64_t evxg_server_now_ns(void);

/* Host-side fault injection for tests of callers' error paths (no counterpart
 * in the reference): the next n device allocations made when a stream is
 * created fail as if the device were out of memory (the creation returns
 * EVXG_ERROR_OUTOFMEMORY and frees what it had), without allocating. */
int evxg_inject_alloc_failures(uint32_t n);

/* lambda = 0.85 * 2^((q-12)/3) in float, as the reference computes it (common.h:264-266). */
float evxg_lambda(uint16_t quality);

/* ---- Host entropy coder ----
 *
 * The part of engine_encode_frame that stays on the CPU: serialize_slice
 * (serialize.cpp:624-686) -- the block table (block types, intra modes with
 * most-probable-mode prediction, prediction targets, motion-vector
 * differences, sub-pel fields, QP deltas), the SAO table and the residual
 * levels (significance maps in scan order), all through the adaptive binary
 * arithmetic coder (abac.cpp) with exponential-Golomb binarisation
 * (golomb.cpp, stream.cpp:996-1075).  The inputs are exactly what
 * evxg_fetch_tables returns for the frame (host memory), for a stream of the
 * build cfg describes (NULL = default); the output is the frame's slice
 * bytes, identical to the reference's, byte-aligned.  *out_len receives the
 * size even when capacity is too small (EVXG_ERROR_CAPACITY_LIMIT).  Keeps no
 * state: slices of different frames may be coded on different threads at once. */
int evxg_serialize_slice(const evxg_config *cfg, uint32_t aligned_w, uint32_t aligned_h, const evxg_frame *frame,
                         const evxg_block_desc *blocks, const evxg_block_desc *prev_blocks, const evxg_sao_info *sao,
                         const int16_t *levels, uint8_t *out, uint64_t capacity, uint64_t *out_len);
/* The 14-byte stream header (evx_header, common.h:55-64) for visible size
 * width x height: "EVX1", size 14, DPB slot count, version 3.11, width,
 * height; its padding byte (offset 7) is 0 (the reference leaves it
 * uninitialised).  A stream is the header followed, per frame in bitstream
 * order, by -- default build -- a 4-byte little-endian size and that many
 * bytes: the 18-byte evxg_frame and the slice (evx3enc.cpp:249-277), or --
 * without B frames -- the first 10 bytes of evxg_frame and the slice
 * (evx3enc.cpp:141-147). */
int evxg_stream_header(const evxg_config *cfg, uint32_t width, uint32_t height, uint8_t out[14]);

/* ---- Decoder pixel half ----
 *
 * engine_decode_frame (decode.cpp:560-612) after unserialize_slice: per
 * macroblock decode_block (decode.cpp:31-432) into the destination slot,
 * deblock_image_filter, sao_filter_image, and the conversion to RGB24
 * (convert.cpp:162-223).  A decoder holds the DPB of one stream of the build
 * cfg describes (NULL = default), zero-initialised like the reference's
 * context (common.cpp:106-202).  evxg_decode_frame takes one frame in
 * bitstream order: its evxg_frame (the record's descriptor; without B frames
 * the slots follow from the index), block and SAO tables and level planes as
 * the entropy decoder produces them -- the same layouts evxg_fetch_tables
 * returns (host memory, or device memory with tables_on_device != 0) -- and
 * writes the visible width*height*3 bytes of RGB24 to rgb (NULL: none; device
 * memory with rgb_on_device != 0).  Decoding the tables an evxg_stream encoded
 * reproduces its reconstruction exactly.  Asynchronous on cuda_stream;
 * evxg_decoder_sync waits and reports EVXG_ERROR_INVALID_RESOURCE for a block
 * descriptor the reference rejects (an unknown block type, a reference that
 * is not a DPB slot other than the destination) and
 * EVXG_ERROR_OPERATION_TIMEDOUT when the intra wavefront gave up waiting (the
 * bound as in evxg_stream_set_timeout_ns; evxg_decoder_reset then restores the
 * state at creation).  Host tables must stay valid until the call returns;
 * a host rgb buffer until the frame is synchronised. */
typedef struct evxg_decoder evxg_decoder;
int evxg_decoder_create(uint32_t width, uint32_t height, const evxg_config *cfg, evxg_decoder **out);
int evxg_decoder_destroy(evxg_decoder *d);
int evxg_decode_frame(evxg_decoder *d, const evxg_frame *frame, const evxg_block_desc *blocks,
                      const evxg_sao_info *sao, const int16_t *levels, int tables_on_device, uint8_t *rgb,
                      int rgb_on_device, void *cuda_stream);
int evxg_decoder_sync(evxg_decoder *d, void *cuda_stream);
/* Copy one DPB slot (plane-set layout) out. */
int evxg_decoder_fetch_planes(evxg_decoder *d, uint32_t slot, int16_t *out, int to_device, void *cuda_stream);
int evxg_decoder_set_timeout_ns(evxg_decoder *d, int64_t ns);
int evxg_decoder_reset(evxg_decoder *d, void *cuda_stream);

/* The host entropy decoder: unserialize_slice (unserialize.cpp:634-696), the
 * inverse of evxg_serialize_slice.  Decodes one slice (data, len bytes; bytes
 * after the slice may follow) into tables that persist from frame to frame
 * the way the reference decoder's context does: a block descriptor gets only
 * the fields the slice codes (block type; intra mode of intra-default blocks;
 * prediction target of inter blocks; vector and sub-pel fields of motion
 * blocks; the second reference's fields of inter blocks in B frames; QP of
 * blocks that are not copies), the others keep earlier frames' values; every
 * SAO entry is cleared and then decoded; the level planes of blocks that are
 * not copies are rewritten.  prev_blocks is the temporal predictor table (the
 * block table after the last frame that is not a B frame, zero before the
 * first).  *consumed receives the slice's length in bytes, known from the
 * arithmetic decoder itself, so records without a size prefix can be cut.
 * EVXG_ERROR_INVALID_RESOURCE for data that is not such a slice. */
int evxg_unserialize_slice(const evxg_config *cfg, uint32_t aligned_w, uint32_t aligned_h, const evxg_frame *frame,
                           const uint8_t *data, uint64_t len, evxg_block_desc *blocks,
                           const evxg_block_desc *prev_blocks, evxg_sao_info *sao, int16_t *levels,
                           uint64_t *consumed);
/* One frame record of a stream, the reference decoder's decode() without its
 * display reorder (evx3dec.cpp:104-215): default build -- a 4-byte size, the
 * 18-byte evxg_frame, the slice; without B frames -- the first 10 bytes of
 * evxg_frame and the slice.  Entropy-decodes on the host into the decoder's
 * own tables, runs evxg_decode_frame and waits for it, and updates the
 * temporal predictor table after frames that are not B frames.  Frames must
 * come in bitstream order (index 0, 1, ...; EVXG_ERROR_INVALID_RESOURCE
 * otherwise).  rgb (host, may be NULL) receives the frame in decode order;
 * *frame_out its descriptor; *consumed the record's length, so concatenated
 * records of either build can be cut. */
int evxg_decoder_decode_record(evxg_decoder *d, const uint8_t *data, uint64_t len, uint8_t *rgb, evxg_frame *frame_out,
                               uint64_t *consumed, void *cuda_stream);

/* The reference's evx3_decoder (evx3.h:103-127) for a whole stream of the
 * build cfg describes (NULL = default), over evxg_decoder: the first decode
 * call reads the 14-byte stream header (and creates the device state for its
 * size), every call one frame record (records need no size prefix: the
 * entropy decoder finds each slice's end), *consumed the bytes used.  With B
 * frames the frames go through a display buffer of 5 like evx3dec.cpp:137-185
 * and each decode / flush call hands out at most the next frame in display
 * order (*has_output); without them every call outputs its frame.  rgb: host
 * memory of width*height*3 bytes (evxg_stream_decoder_dims after the first
 * call).  clear returns to the state before the header (evx3dec.cpp:25-48). */
typedef struct evxg_stream_decoder evxg_stream_decoder;
int evxg_stream_decoder_create(const evxg_config *cfg, evxg_stream_decoder **out);
int evxg_stream_decoder_destroy(evxg_stream_decoder *d);
int evxg_stream_decoder_clear(evxg_stream_decoder *d);
int evxg_stream_decoder_dims(const evxg_stream_decoder *d, uint32_t *width, uint32_t *height);
int evxg_stream_decoder_decode(evxg_stream_decoder *d, const uint8_t *data, uint64_t len, uint64_t *consumed,
                               uint8_t *rgb, int *has_output);
int evxg_stream_decoder_flush(evxg_stream_decoder *d, uint8_t *rgb, int *has_output);

/* ---- Container ----
 *
 * The reference's packet container (evx_muxer / evx_demuxer, muxer.h:53-160,
 * muxer.cpp), byte for byte: a 10-byte header ("EVX3", u32 header size,
 * version 1, stream count), an 18-byte descriptor per stream (type, id,
 * width, height, f32 frame rate, u32 sample rate, channels, bit depth,
 * quality, a zero pad byte), then packets of a 16-byte header ("EP", stream
 * id, stream type, u64 timestamp in microseconds, u32 payload size) and the
 * payload; all little-endian.  A video stream's packets carry the .evx
 * stream as the reference's encoder tool cuts it (tools/evx_encode.cpp:
 * 185-275): the stream header with the first frame record, then one frame
 * record per packet. */
#define EVXG_STREAM_TYPE_VIDEO 0
#define EVXG_STREAM_TYPE_AUDIO 1
typedef struct evxg_stream_desc {
    uint8_t stream_type;
    uint8_t stream_id;
    uint16_t width, height;    /* video */
    float frame_rate;          /* video */
    uint32_t sample_rate;      /* audio */
    uint8_t channels, bit_depth, quality;   /* audio */
} evxg_stream_desc;
typedef struct evxg_muxer evxg_muxer;
/* Creates (truncates) the file; streams are added before the header is written. */
int evxg_muxer_open(const char *path, evxg_muxer **out);
int evxg_muxer_add_video_stream(evxg_muxer *m, uint16_t width, uint16_t height, float frame_rate, uint8_t *stream_id);
int evxg_muxer_add_audio_stream(evxg_muxer *m, uint32_t sample_rate, uint8_t channels, uint8_t bit_depth,
                                uint8_t quality, uint8_t *stream_id);
int evxg_muxer_write_header(evxg_muxer *m);
int evxg_muxer_write_packet(evxg_muxer *m, uint8_t stream_id, uint8_t stream_type, uint64_t timestamp_us,
                            const void *payload, uint32_t size);
/* Flushes and closes the file and frees m. */
int evxg_muxer_close(evxg_muxer *m);
typedef struct evxg_demuxer evxg_demuxer;
/* Opens the file and reads its header and stream descriptors. */
int evxg_demuxer_open(const char *path, evxg_demuxer **out);
uint32_t evxg_demuxer_stream_count(const evxg_demuxer *d);
int evxg_demuxer_stream(const evxg_demuxer *d, uint32_t index, evxg_stream_desc *out);
/* The next packet: EVXG_ERROR_OPERATION_COMPLETED at the end of the file;
 * EVXG_ERROR_CAPACITY_LIMIT (with *size set, the packet left unread) when
 * capacity is too small. */
int evxg_demuxer_read_packet(evxg_demuxer *d, uint8_t *stream_id, uint8_t *stream_type, uint64_t *timestamp_us,
                             uint8_t *payload, uint32_t capacity, uint32_t *size);
int evxg_demuxer_close(evxg_demuxer *d);

/* Human-readable text of the last error on this thread. */
const char *evxg_last_error(void);

/* ---- Allocation-free macroblock pass ----
 *
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory when they encode (a plugin that must take every buffer from a host
 * application's own arena, code running where an allocation would stall or
 * fail, a process with a device budget fixed at start-up): runs only the
 * macroblock wavefront of one frame -- classify, encode and reconstruct every
 * macroblock into dpb[frame->dpb_slot], writing the block table and the level
 * planes -- on buffers the caller owns, and allocates nothing.
 *
 * Layouts are those of the stream API: src, levels and each dpb[i] are int16
 * plane sets of the 16-aligned size (Y, then U, then V); blocks and
 * prev_blocks hold (aligned_w/16)*(aligned_h/16) descriptors; prev_blocks is
 * read for P frames only.  All pointers are device pointers.
 *
 * Its scratch (a progress word per macroblock row, a row counter and an error
 * word) is a fixed array in the library's device image: at most
 * EVXG_NOALLOC_MAX_MB_ROWS macroblock rows, i.e. aligned_h <= 65408; larger
 * frames are refused with EVXG_ERROR_CAPACITY_LIMIT.  The first call on a
 * device looks up that array's device address; make that first call before
 * any stream capture.  Every call on a device shares the one array and
 * re-initialises it, so calls whose work overlaps on the GPU race: issue them
 * one after another.  The call waits for its work on cuda_stream and returns
 * EVXG_ERROR_OPERATION_TIMEDOUT if the wavefront gave up waiting. */
#define EVXG_NOALLOC_MAX_MB_ROWS 4088
int evxg_mb_pass_noalloc(uint32_t aligned_w, uint32_t aligned_h, const evxg_frame *frame, const int16_t *src,
                         int16_t *const dpb[4], int16_t *levels, evxg_block_desc *blocks,
                         const evxg_block_desc *prev_blocks, void *cuda_stream);
/* The wait bound of evxg_mb_pass_noalloc's wavefront (see
 * evxg_stream_set_timeout_ns), for every later call in the process; 5 s by
 * default, ns > 0. */
int evxg_mb_pass_noalloc_set_timeout_ns(int64_t ns);

/* ---- GOP-level encoder: evx3_encoder (evx3.h:67-100) over the stream API ---- */

typedef struct evxg_encoder evxg_encoder;

/* Called once per encoded frame, in bitstream order, after the frame's GPU
 * work has completed and its tables were copied to host memory. */
typedef void (*evxg_frame_callback)(void *user, const evxg_frame *frame,
                                    const evxg_block_desc *blocks, const evxg_block_desc *prev_blocks,
                                    const evxg_sao_info *sao, const int16_t *levels);

int evxg_encoder_create(evxg_frame_callback cb, void *user, evxg_encoder **out);
/* An encoder of the build cfg describes (NULL = the default build); without B
 * frames every frame is encoded as it arrives and flush has nothing to do. */
int evxg_encoder_create_config(evxg_frame_callback cb, void *user, const evxg_config *cfg, evxg_encoder **out);
int evxg_encoder_destroy(evxg_encoder *e);
int evxg_encoder_clear(evxg_encoder *e);                     /* evx3enc.cpp:35-55 */
int evxg_encoder_insert_intra(evxg_encoder *e);              /* evx3enc.cpp:57-62 */
int evxg_encoder_set_quality(evxg_encoder *e, uint8_t q);    /* evx3enc.cpp:64-82 */
/* evx3enc.cpp:105-234: buffer / encode one RGB24 host frame. */
int evxg_encoder_encode(evxg_encoder *e, const uint8_t *rgb, uint32_t width, uint32_t height);
int evxg_encoder_flush(evxg_encoder *e);                     /* evx3enc.cpp:385-414 */
/* The stream under an encoder (NULL before the first frame). */
evxg_stream *evxg_encoder_stream(evxg_encoder *e);
/* evx3_encoder::peek (evx3enc.cpp:417-547): an RGB24 image of the visible
 * size into host memory -- the converted source, the reference slot the
 * reference's own encoder state names (its running frame's dpb_slot, which
 * its GOP logic never sets in the default build, so slot 0; without B frames
 * the slot one index back from the next frame), or per macroblock of the
 * last encoded frame: block type (R intra, G motion, B copy), QP
 * (255 - 15 q, copies red), variance (variance / 30, copies red), sub-pel
 * (G quarter, B half).  EVXG_PEEK_PREDICTION is EVXG_ERROR_NOTIMPL, as in the
 * reference; before the first frame nothing is written. */
#define EVXG_PEEK_SOURCE         0
#define EVXG_PEEK_PREDICTION     1
#define EVXG_PEEK_BLOCK_TABLE    2
#define EVXG_PEEK_QUANT_TABLE    3
#define EVXG_PEEK_SPMP_TABLE     4
#define EVXG_PEEK_BLOCK_VARIANCE 5
#define EVXG_PEEK_DESTINATION    6
int evxg_encoder_peek(evxg_encoder *e, int which, uint8_t *rgb);
/* Bitstream output: once set, the encoder also codes every frame on the host
 * (evxg_serialize_slice) and hands the stream's bytes to cb in order, on the
 * calling thread -- the 14-byte header before the first frame, then each
 * frame's record (see evxg_stream_header) -- the bytes the reference's
 * encode / flush write into their bit_stream (evx3enc.cpp:105-414).  cb NULL
 * turns it off. */
typedef void (*evxg_bytes_callback)(void *user, const uint8_t *bytes, uint64_t n);
int evxg_encoder_set_output(evxg_encoder *e, evxg_bytes_callback cb, void *user);

#ifdef __cplusplus
}
#endif
#endif
