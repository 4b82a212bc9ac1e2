/*
 * ref_harness.cpp -- test-only C-ABI shim around the UNMODIFIED reference
 * encoder library (ramenhut/chicago, EVX3), compiled from its own sources by
 * oracle/Makefile into oracle/_ref/libevxref.so.
 *
 * This file is test infrastructure: it is the pin for the oracle restatement
 * and the GPU path, and the CPU baseline of the benchmark.  Nothing in the
 * product links it.
 *
 * Two surfaces:
 *   1. evxref_enc_*   : the reference's own public encoder API
 *                       (create_encoder / set_quality / insert_intra / encode /
 *                       flush, src/video/evx3.h:67-100), unchanged, WPP threads.
 *   2. evxref_ctx_*   : a staged per-frame driver that performs the same steps
 *                       as engine_encode_frame (src/video/encode.cpp:945-1001)
 *                       with the reference's external functions, dumping every
 *                       intermediate stage (converted source, block table,
 *                       quantised levels, recon before/after deblock, SAO table,
 *                       recon after SAO, serialized bytes).
 */
#include "evx3.h"
#include "evx3enc.h"
#include "common.h"
#include "convert.h"
#include "image.h"
#include "imageset.h"
#include "sao.h"
#include "bitstream.h"
#include "muxer.h"

#include <cstring>
#include <cstdint>
#include <vector>

using namespace evx;

namespace evx {
evx_status deblock_image_filter(evx_block_desc *block_table, image_set *target_image);
evx_status serialize_slice(const evx_frame &frame, evx_context *context, bit_stream *output);
evx_status encode_slice(const evx_frame &frame, evx_context *context);
evx_status encode_slice_wpp(const evx_frame &frame, evx_context *context);
evx_status unserialize_slice(bit_stream *input, const evx_frame &frame, evx_context *context);
evx_status decode_slice(const evx_frame &frame, evx_context *context);
#if EVX_ENABLE_WPP
evx_status decode_slice_wpp(const evx_frame &frame, evx_context *context);
#endif
}

/*
 * Every table crosses this harness in the layouts of the default build
 * (evx_block_desc 28 B, evx_frame 18 B, pack(2)).  The I/P variants
 * (EVX_ENABLE_B_FRAMES 0, see oracle/variants/) drop the B-frame fields at
 * the end of both structs (common.h:75-81, :105-113): their descriptor is the
 * first 18 bytes of the wide one and their frame the first 10, so the harness
 * converts by truncation and zero extension.
 */
static const size_t WIDE_BLOCK = 28, WIDE_FRAME = 18;
#if EVX_ENABLE_B_FRAMES
static_assert(sizeof(evx_block_desc) == 28, "block desc wire size");
static_assert(sizeof(evx_frame) == 18, "frame header wire size");
#else
static_assert(sizeof(evx_block_desc) == 18, "block desc wire size (no B frames)");
static_assert(sizeof(evx_frame) == 10, "frame header wire size (no B frames)");
#endif
static_assert(sizeof(evx_sao_info) == 16, "sao info wire size");

static evx_frame frame_from_wide(const uint8_t *wide)
{
    evx_frame f;
    memcpy(&f, wide, sizeof(evx_frame));   /* the native struct is a prefix of the wide one */
    return f;
}
static uint32_t dest_slot(const evx_frame &f)
{
#if EVX_ENABLE_B_FRAMES
    return f.dpb_slot;
#else
    return query_prediction_index_by_offset(f, 0);   /* encode.cpp:952-956 */
#endif
}
static void blocks_to_wide(const evx_block_desc *t, uint32_t n, uint8_t *wide)
{
    for (uint32_t i = 0; i < n; i++) {
        memset(wide + i * WIDE_BLOCK, 0, WIDE_BLOCK);
        memcpy(wide + i * WIDE_BLOCK, t + i, sizeof(evx_block_desc));
    }
}
static void blocks_from_wide(const uint8_t *wide, uint32_t n, evx_block_desc *t)
{
    for (uint32_t i = 0; i < n; i++) memcpy(t + i, wide + i * WIDE_BLOCK, sizeof(evx_block_desc));
}

extern "C" {

/* ---------------- 1. stock public API ---------------- */

struct evxref_enc {
    evx3_encoder *enc;
    bit_stream out;
};

void *evxref_enc_create(uint32_t capacity_bytes)
{
    evxref_enc *h = new evxref_enc;
    if (create_encoder(&h->enc) != EVX_SUCCESS) { delete h; return nullptr; }
    h->out.resize_capacity(capacity_bytes * 8u);   /* capacity is given in bits */
    return h;
}

void evxref_enc_destroy(void *p)
{
    evxref_enc *h = (evxref_enc *)p;
    if (!h) return;
    destroy_encoder(h->enc);
    delete h;
}

int evxref_enc_set_quality(void *p, uint8_t q) { return ((evxref_enc *)p)->enc->set_quality(q); }
int evxref_enc_insert_intra(void *p) { return ((evxref_enc *)p)->enc->insert_intra(); }

/* Encode one RGB24 frame; the bytes produced by this call are appended to out. */
int evxref_enc_encode(void *p, const uint8_t *rgb, uint32_t w, uint32_t h,
                      uint8_t *out, uint32_t cap, uint32_t *out_len)
{
    evxref_enc *e = (evxref_enc *)p;
    e->out.empty();
    evx_status s = e->enc->encode((void *)rgb, w, h, &e->out);
    uint32_t n = e->out.query_byte_occupancy();
    *out_len = n;
    if (s != EVX_SUCCESS) return s;
    if (n > cap) return EVX_ERROR_CAPACITY_LIMIT;
    if (n) memcpy(out, e->out.query_data(), n);
    return 0;
}

/* evx3_encoder::peek (evx3enc.cpp:417-547) into out (visible size RGB24). */
int evxref_enc_peek(void *p, int state, uint8_t *out)
{
    return ((evxref_enc *)p)->enc->peek((EVX_PEEK_STATE)state, out);
}

int evxref_enc_flush(void *p, uint8_t *out, uint32_t cap, uint32_t *out_len)
{
    evxref_enc *e = (evxref_enc *)p;
    e->out.empty();
#if EVX_ENABLE_B_FRAMES
    evx_status s = e->enc->flush(&e->out);
#else
    evx_status s = EVX_SUCCESS;   /* no reorder buffer, nothing pending (evx3.h:92-95) */
#endif
    uint32_t n = e->out.query_byte_occupancy();
    *out_len = n;
    if (s != EVX_SUCCESS) return s;
    if (n > cap) return EVX_ERROR_CAPACITY_LIMIT;
    if (n) memcpy(out, e->out.query_data(), n);
    return 0;
}

/* Decode a whole .evx stream with the reference's public decoder
 * (create_decoder / decode / has_output / flush, src/video/evx3.h:103-127),
 * the way its own round-trip test drives it (tests/test_codec_roundtrip.cpp:
 * 211-231): frames come out in display order, w*h*3 bytes each; at most
 * max_frames are stored, *n_out counts all of them. */
int evxref_decode_stream(const uint8_t *data, uint32_t len, uint32_t w, uint32_t h, uint8_t *out,
                         uint32_t max_frames, uint32_t *n_out)
{
    evx3_decoder *dec = nullptr;
    if (create_decoder(&dec) != EVX_SUCCESS) return EVX_ERROR_EXECUTION_FAILURE;
    bit_stream bs;
    bs.resize_capacity((len + 64) * 8u);
    bs.write_bytes((void *)data, len);
    const size_t fb = (size_t)w * h * 3;
    std::vector<uint8_t> buf(fb);
    uint32_t n = 0;
    int rc = 0;
    auto keep = [&]() {
        if (n < max_frames) memcpy(out + n * fb, buf.data(), fb);
        n++;
    };
    while (bs.query_byte_occupancy() > 0) {
        const evx_status s = dec->decode(&bs, buf.data());
        if (s != EVX_SUCCESS) { rc = s; break; }
#if EVX_ENABLE_B_FRAMES
        if (!dec->has_output()) continue;
#endif
        keep();
    }
#if EVX_ENABLE_B_FRAMES
    while (rc == 0) {
        dec->flush(buf.data());
        if (!dec->has_output()) break;
        keep();
    }
#endif
    destroy_decoder(dec);
    *n_out = n;
    return rc;
}

/* The same decoder fed one frame record per decode() call, each in a bit
 * stream of its own (record k = data[offsets[k] .. offsets[k+1]), the first
 * one with the stream header in front), as a container delivers packets.
 * Builds without B frames need this: their records carry no size prefix and
 * the arithmetic decoder reads past a frame's end (decode.cpp's reason for
 * the prefix, evx3dec.cpp:116-135), so a concatenated stream decodes only its
 * first frame. */
int evxref_decode_records(const uint8_t *data, const uint32_t *offsets, uint32_t n_records, uint32_t w, uint32_t h,
                          uint8_t *out, uint32_t max_frames, uint32_t *n_out)
{
    evx3_decoder *dec = nullptr;
    if (create_decoder(&dec) != EVX_SUCCESS) return EVX_ERROR_EXECUTION_FAILURE;
    const size_t fb = (size_t)w * h * 3;
    std::vector<uint8_t> buf(fb);
    uint32_t n = 0;
    int rc = 0;
    auto keep = [&]() {
        if (n < max_frames) memcpy(out + n * fb, buf.data(), fb);
        n++;
    };
    for (uint32_t k = 0; k < n_records && rc == 0; k++) {
        const uint32_t len = offsets[k + 1] - offsets[k];
        bit_stream bs;
        bs.resize_capacity((len + 64) * 8u);
        bs.write_bytes((void *)(data + offsets[k]), len);
        const evx_status s = dec->decode(&bs, buf.data());
        if (s != EVX_SUCCESS) { rc = s; break; }
#if EVX_ENABLE_B_FRAMES
        if (!dec->has_output()) continue;
#endif
        keep();
    }
#if EVX_ENABLE_B_FRAMES
    while (rc == 0) {
        dec->flush(buf.data());
        if (!dec->has_output()) break;
        keep();
    }
#endif
    destroy_decoder(dec);
    *n_out = n;
    return rc;
}

static void copy_set(const image_set &s, int16_t *dst, uint32_t w, uint32_t h)
{
    if (!dst) return;
    memcpy(dst, s.query_y_image()->query_data(), (size_t)w * h * 2);
    memcpy(dst + (size_t)w * h, s.query_u_image()->query_data(), (size_t)(w / 2) * (h / 2) * 2);
    memcpy(dst + (size_t)w * h + (size_t)(w / 2) * (h / 2), s.query_v_image()->query_data(),
           (size_t)(w / 2) * (h / 2) * 2);
}

/* ---------------- container (src/muxer.cpp) ---------------- */

/* A container written by the reference's evx_muxer: a video stream (w x h at
 * fps; and an audio stream after it when with_audio), then n packets of the
 * video stream, packet k = data[offsets[k] .. offsets[k+1]) at timestamp ts[k]. */
int evxref_mux_file(const char *path, uint16_t w, uint16_t h, float fps, int with_audio, uint32_t n,
                    const uint8_t *data, const uint32_t *offsets, const uint64_t *ts)
{
    evx_muxer mux;
    uint8 vid = 0, aud = 0;
    if (mux.open(path) != EVX_SUCCESS) return EVX_ERROR_IO_FAILURE;
    mux.add_video_stream(w, h, fps, &vid);
    if (with_audio) mux.add_audio_stream(48000, 2, 16, 5, &aud);
    if (mux.write_header() != EVX_SUCCESS) return EVX_ERROR_IO_FAILURE;
    for (uint32_t k = 0; k < n; k++)
        if (mux.write_packet(vid, EVX_STREAM_TYPE_VIDEO, ts[k], data + offsets[k], offsets[k + 1] - offsets[k]) !=
            EVX_SUCCESS)
            return EVX_ERROR_IO_FAILURE;
    mux.close();
    return 0;
}

/* The reference encoder tool's video path (tools/evx_encode.cpp:143-275) on n
 * raw RGB24 frames instead of FFmpeg's decoder: set_quality, encode() every
 * frame into one bit stream, cut each call's output into packets as the tool
 * does (with B frames: the first output whole -- stream header and the first
 * record -- then one size-prefixed record per packet, flush() included;
 * without: one packet per call), timestamps count * 10^6 / fps. */
int evxref_encode_container(const char *path, const uint8_t *frames, uint32_t n, uint32_t w, uint32_t h, double fps,
                            uint8_t quality)
{
    evx_muxer mux;
    uint8 vid = 0;
    if (mux.open(path) != EVX_SUCCESS) return EVX_ERROR_IO_FAILURE;
    mux.add_video_stream((uint16)w, (uint16)h, (float32)fps, &vid);
    mux.write_header();
    evx3_encoder *enc = nullptr;
    if (create_encoder(&enc) != EVX_SUCCESS) return EVX_ERROR_EXECUTION_FAILURE;
    enc->set_quality(quality);
    bit_stream coded;
    coded.resize_capacity((w * h * 3 * 4 + (1u << 20)) * 8u);
    uint64_t count = 0;
    bool header_written = false;
    auto packet = [&](const uint8_t *p, uint32_t len) {
        mux.write_packet(vid, EVX_STREAM_TYPE_VIDEO, (uint64)(count * 1000000.0 / fps), p, len);
        count++;
    };
    auto records = [&]() {   /* size-prefixed records of one output */
        const uint8_t *base = coded.query_data();
        uint32_t pos = 0, total = coded.query_byte_occupancy();
        while (pos + 4 <= total) {
            uint32_t size;
            memcpy(&size, base + pos, 4);
            if (pos + 4 + size > total) break;
            packet(base + pos, 4 + size);
            pos += 4 + size;
        }
    };
    int rc = 0;
    for (uint32_t i = 0; i < n && rc == 0; i++) {
        coded.empty();
        rc = enc->encode((void *)(frames + (size_t)i * w * h * 3), w, h, &coded);
        if (rc) break;
#if EVX_ENABLE_B_FRAMES && (EVX_B_FRAME_COUNT > 0)
        if (coded.query_byte_occupancy() > 0) {
            if (!header_written) {
                packet(coded.query_data(), coded.query_byte_occupancy());
                header_written = true;
            } else {
                records();
            }
        }
#else
        (void)header_written;
        packet(coded.query_data(), coded.query_byte_occupancy());
#endif
    }
#if EVX_ENABLE_B_FRAMES
    if (rc == 0) {
        coded.empty();
        rc = enc->flush(&coded);
        records();
    }
#else
    (void)records;
#endif
    destroy_encoder(enc);
    mux.close();
    return rc;
}

/* A container read by the reference's evx_demuxer: the stream count and every
 * packet's stream id, timestamp and payload (payloads concatenated into data,
 * at most max packets). */
int evxref_demux_file(const char *path, uint32_t *n_streams, uint8_t *data, uint64_t cap, uint32_t *sizes,
                      uint8_t *ids, uint64_t *ts, uint32_t max, uint32_t *n)
{
    evx_demuxer dmx;
    if (dmx.open(path) != EVX_SUCCESS || dmx.read_header() != EVX_SUCCESS) return EVX_ERROR_IO_FAILURE;
    *n_streams = dmx.query_stream_count();
    evx_demux_packet pkt;
    uint64_t used = 0;
    uint32_t k = 0;
    evx_status s;
    while ((s = dmx.read_packet(&pkt)) == EVX_SUCCESS) {
        if (k < max && used + pkt.payload.size() <= cap) {
            memcpy(data + used, pkt.payload.data(), pkt.payload.size());
            used += pkt.payload.size();
            sizes[k] = (uint32_t)pkt.payload.size();
            ids[k] = pkt.stream_id;
            ts[k] = pkt.timestamp;
        }
        k++;
    }
    dmx.close();
    *n = k;
    return s == EVX_ERROR_OPERATION_COMPLETED ? 0 : s;
}

/* ---------------- staged decoder ----------------
 * engine_decode_frame (src/video/decode.cpp:560-612) step by step with the
 * reference's own functions, dumping what unserialize_slice produced (block
 * table, SAO table, level planes) and the final reconstruction: the tables a
 * GPU decoder is given and the pixels it must reach. */
struct evxref_dctx {
    evx_context ctx;
    uint32_t w, h;       /* aligned (context) dimensions */
};

void *evxref_dctx_create(uint32_t aligned_w, uint32_t aligned_h)
{
    evxref_dctx *c = new evxref_dctx;
    if (initialize_context(aligned_w, aligned_h, &c->ctx) != EVX_SUCCESS) { delete c; return nullptr; }
    c->w = aligned_w; c->h = aligned_h;
    return c;
}

void evxref_dctx_destroy(void *p)
{
    evxref_dctx *c = (evxref_dctx *)p;
    if (!c) return;
    clear_context(&c->ctx);
    delete c;
}

/* record = the frame's evx_frame (native size) followed by its slice; the
 * descriptor is returned in the default build's 18-byte layout. */
int evxref_dctx_decode_frame(void *p, const uint8_t *record, uint32_t len, uint32_t vis_w, uint32_t vis_h,
                             uint8_t *frame18_out, uint8_t *dump_blocks, uint8_t *dump_sao, int16_t *dump_levels,
                             int16_t *dump_final, uint8_t *rgb_out)
{
    evxref_dctx *c = (evxref_dctx *)p;
    const uint32_t nblk = c->ctx.width_in_blocks * c->ctx.height_in_blocks;
    bit_stream bs;
    bs.resize_capacity((len + 64) * 8u);
    bs.write_bytes((void *)record, len);
    evx_frame frame;
    if (bs.read_bytes(&frame, sizeof(evx_frame)) != EVX_SUCCESS) return 110;
    if (frame18_out) {
        memset(frame18_out, 0, WIDE_FRAME);
        memcpy(frame18_out, &frame, sizeof(evx_frame));
    }
    if (unserialize_slice(&bs, frame, &c->ctx) != EVX_SUCCESS) return 111;
    if (dump_blocks) blocks_to_wide(c->ctx.block_table, nblk, dump_blocks);
    if (dump_sao) memcpy(dump_sao, c->ctx.sao_table, (size_t)nblk * 16);
    copy_set(c->ctx.cache_bank.input_cache, dump_levels, c->w, c->h);
#if EVX_ENABLE_WPP
    if (decode_slice_wpp(frame, &c->ctx) != EVX_SUCCESS) return 112;
#else
    if (decode_slice(frame, &c->ctx) != EVX_SUCCESS) return 112;
#endif
    image_set &dest = c->ctx.cache_bank.prediction_cache[dest_slot(frame)];
    if (deblock_image_filter(c->ctx.block_table, &dest) != EVX_SUCCESS) return 113;
    if (sao_filter_image(c->ctx.sao_table, c->ctx.width_in_blocks, c->ctx.height_in_blocks, &dest) != EVX_SUCCESS)
        return 114;
    copy_set(dest, dump_final, c->w, c->h);
    if (rgb_out) {
        image out;
        if (create_image(EVX_IMAGE_FORMAT_R8G8B8, rgb_out, vis_w, vis_h, &out) != EVX_SUCCESS) return 115;
        if (convert_image(dest, &out) != EVX_SUCCESS) return 116;
    }
#if EVX_ENABLE_B_FRAMES
    if (frame.type != EVX_FRAME_BIDIR)   /* decode.cpp:601-609 */
#endif
        memcpy(c->ctx.prev_block_table, c->ctx.block_table, (size_t)nblk * sizeof(evx_block_desc));
    return 0;
}

#ifndef EVXREF_STOCK_ONLY   /* the staged driver needs encode.cpp; builds without it keep the stock API */
/* ---------------- 2. staged per-frame driver ---------------- */

struct evxref_ctx {
    evx_context ctx;
    uint32_t w, h;       /* aligned (context) dimensions */
    bit_stream stream;
};

void *evxref_ctx_create(uint32_t aligned_w, uint32_t aligned_h)
{
    evxref_ctx *c = new evxref_ctx;
    if (initialize_context(aligned_w, aligned_h, &c->ctx) != EVX_SUCCESS) { delete c; return nullptr; }
    c->w = aligned_w; c->h = aligned_h;
    c->stream.resize_capacity((aligned_w * aligned_h * 8 + (1u << 20)) * 8u);   /* bits */
    return c;
}

void evxref_ctx_destroy(void *p)
{
    evxref_ctx *c = (evxref_ctx *)p;
    if (!c) return;
    clear_context(&c->ctx);
    delete c;
}


static void load_set(image_set *s, const int16_t *src, uint32_t w, uint32_t h)
{
    memcpy(s->query_y_image()->query_data(), src, (size_t)w * h * 2);
    memcpy(s->query_u_image()->query_data(), src + (size_t)w * h, (size_t)(w / 2) * (h / 2) * 2);
    memcpy(s->query_v_image()->query_data(), src + (size_t)w * h + (size_t)(w / 2) * (h / 2),
           (size_t)(w / 2) * (h / 2) * 2);
}

/*
 * Plane-set buffers are laid out Y (w*h) then U then V ((w/2)*(h/2) each), int16.
 * Any dump pointer may be NULL.  frame18 is the 18-byte packed evx_frame of the
 * default build (variants read its prefix); dump_blocks receives 28-byte
 * descriptors.  use_wpp selects encode_slice_wpp (the stock schedule) instead
 * of encode_slice where the build has it.  The destination slot is the
 * frame's dpb_slot, or, without B frames, the one its index selects
 * (query_prediction_index_by_offset(frame, 0), common.cpp:256-259).
 */
int evxref_ctx_encode_frame(void *p, const uint8_t *rgb, uint32_t w, uint32_t h,
                            const uint8_t *frame18, int use_wpp,
                            int16_t *dump_src, uint8_t *dump_blocks, int16_t *dump_levels,
                            int16_t *dump_recon, int16_t *dump_deblock,
                            uint8_t *dump_sao, int16_t *dump_final,
                            uint8_t *bytes, uint32_t cap, uint32_t *nbytes)
{
    evxref_ctx *c = (evxref_ctx *)p;
    evx_frame frame = frame_from_wide(frame18);
    uint32_t nblk = c->ctx.width_in_blocks * c->ctx.height_in_blocks;

    image input;
    if (create_image(EVX_IMAGE_FORMAT_R8G8B8, (void *)rgb, w, h, &input) != EVX_SUCCESS) return 100;
    if (convert_image(input, &c->ctx.cache_bank.input_cache) != EVX_SUCCESS) return 101;
    copy_set(c->ctx.cache_bank.input_cache, dump_src, c->w, c->h);

#if EVX_ENABLE_WPP
    evx_status s = use_wpp ? encode_slice_wpp(frame, &c->ctx) : encode_slice(frame, &c->ctx);
#else
    (void)use_wpp;
    evx_status s = encode_slice(frame, &c->ctx);
#endif
    if (s != EVX_SUCCESS) return 102;
    image_set &dest = c->ctx.cache_bank.prediction_cache[dest_slot(frame)];
    if (dump_blocks) blocks_to_wide(c->ctx.block_table, nblk, dump_blocks);
    copy_set(c->ctx.cache_bank.output_cache, dump_levels, c->w, c->h);
    copy_set(dest, dump_recon, c->w, c->h);

    if (deblock_image_filter(c->ctx.block_table, &dest) != EVX_SUCCESS) return 103;
    copy_set(dest, dump_deblock, c->w, c->h);

    if (sao_encode_frame(c->ctx.cache_bank.input_cache, &dest, c->ctx.sao_table,
                         c->ctx.width_in_blocks, c->ctx.height_in_blocks,
                         compute_lambda(frame.quality)) != EVX_SUCCESS) return 104;
    if (dump_sao) memcpy(dump_sao, c->ctx.sao_table, (size_t)nblk * 16);
    copy_set(dest, dump_final, c->w, c->h);

    c->stream.empty();
    if (serialize_slice(frame, &c->ctx, &c->stream) != EVX_SUCCESS) return 105;
    uint32_t n = c->stream.query_byte_occupancy();
    if (nbytes) *nbytes = n;
    if (bytes) {
        if (n > cap) return EVX_ERROR_CAPACITY_LIMIT;
        memcpy(bytes, c->stream.query_data(), n);
    }

#if EVX_ENABLE_B_FRAMES
    if (frame.type != EVX_FRAME_BIDIR)   /* encode.cpp:990-998 */
#endif
        memcpy(c->ctx.prev_block_table, c->ctx.block_table, (size_t)nblk * sizeof(evx_block_desc));
    return 0;
}

/*
 * Serialize externally produced tables with the reference's own entropy coder
 * (serialize_slice, src/video/serialize.cpp:624-686).  Loads block table,
 * SAO table, level planes and prev_block_table into the context first.
 * Used to turn GPU outputs into .evx bytes in tests.
 */
int evxref_ctx_serialize(void *p, const uint8_t *frame18, const uint8_t *blocks,
                         const uint8_t *prev_blocks, const uint8_t *sao,
                         const int16_t *levels, uint8_t *bytes, uint32_t cap, uint32_t *nbytes)
{
    evxref_ctx *c = (evxref_ctx *)p;
    evx_frame frame = frame_from_wide(frame18);
    uint32_t nblk = c->ctx.width_in_blocks * c->ctx.height_in_blocks;
    blocks_from_wide(blocks, nblk, c->ctx.block_table);
    blocks_from_wide(prev_blocks, nblk, c->ctx.prev_block_table);
    memcpy(c->ctx.sao_table, sao, (size_t)nblk * 16);
    load_set(&c->ctx.cache_bank.output_cache, levels, c->w, c->h);
    c->stream.empty();
    if (serialize_slice(frame, &c->ctx, &c->stream) != EVX_SUCCESS) return 105;
    uint32_t n = c->stream.query_byte_occupancy();
    *nbytes = n;
    if (n > cap) return EVX_ERROR_CAPACITY_LIMIT;
    memcpy(bytes, c->stream.query_data(), n);
    return 0;
}

/* Read back one DPB slot (plane-set layout). */
int evxref_ctx_get_slot(void *p, uint32_t slot, int16_t *out)
{
    evxref_ctx *c = (evxref_ctx *)p;
    if (slot >= EVX_REFERENCE_FRAME_COUNT) return EVX_ERROR_INVALIDARG;
    copy_set(c->ctx.cache_bank.prediction_cache[slot], out, c->w, c->h);
    return 0;
}

#endif /* EVXREF_STOCK_ONLY */

float evxref_lambda(uint16_t q) { return compute_lambda(q); }

/* The compile-time configuration of this build: B frames on/off
 * (EVX_ENABLE_B_FRAMES), DPB slots (EVX_REFERENCE_FRAME_COUNT), WPP threads
 * on/off (EVX_ENABLE_WPP) and the native sizes of evx_frame / evx_block_desc. */
void evxref_config(int *b_frames, int *ref_count, int *wpp, int *frame_bytes, int *block_bytes)
{
    *b_frames = EVX_ENABLE_B_FRAMES;
    *ref_count = EVX_REFERENCE_FRAME_COUNT;
    *wpp = EVX_ENABLE_WPP;
    *frame_bytes = (int)sizeof(evx_frame);
    *block_bytes = (int)sizeof(evx_block_desc);
}

uint32_t evxref_sizeof_block_desc(void) { return sizeof(evx_block_desc); }

} /* extern "C" */
