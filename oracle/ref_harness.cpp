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

#include <cstring>
#include <cstdint>
#include <vector>

using namespace evx;

namespace evx {
evx_status deblock_image_filter(evx_block_desc *block_table, image_set *target_image);
evx_status serialize_slice(const evx_frame &frame, evx_context *context, bit_stream *output);
evx_status encode_slice(const evx_frame &frame, evx_context *context);
evx_status encode_slice_wpp(const evx_frame &frame, evx_context *context);
}

static_assert(sizeof(evx_block_desc) == 28, "block desc wire size");
static_assert(sizeof(evx_sao_info) == 16, "sao info wire size");
static_assert(sizeof(evx_frame) == 18, "frame header wire size");

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

int evxref_enc_flush(void *p, uint8_t *out, uint32_t cap, uint32_t *out_len)
{
    evxref_enc *e = (evxref_enc *)p;
    e->out.empty();
    evx_status s = e->enc->flush(&e->out);
    uint32_t n = e->out.query_byte_occupancy();
    *out_len = n;
    if (s != EVX_SUCCESS) return s;
    if (n > cap) return EVX_ERROR_CAPACITY_LIMIT;
    if (n) memcpy(out, e->out.query_data(), n);
    return 0;
}

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

static void copy_set(const image_set &s, int16_t *dst, uint32_t w, uint32_t h)
{
    if (!dst) return;
    memcpy(dst, s.query_y_image()->query_data(), (size_t)w * h * 2);
    memcpy(dst + (size_t)w * h, s.query_u_image()->query_data(), (size_t)(w / 2) * (h / 2) * 2);
    memcpy(dst + (size_t)w * h + (size_t)(w / 2) * (h / 2), s.query_v_image()->query_data(),
           (size_t)(w / 2) * (h / 2) * 2);
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
 * Any dump pointer may be NULL.  frame18 is the 18-byte packed evx_frame.
 * use_wpp selects encode_slice_wpp (the stock schedule) instead of encode_slice.
 */
int evxref_ctx_encode_frame(void *p, const uint8_t *rgb, uint32_t w, uint32_t h,
                            const uint8_t *frame18, int use_wpp,
                            int16_t *dump_src, uint8_t *dump_blocks, int16_t *dump_levels,
                            int16_t *dump_recon, int16_t *dump_deblock,
                            uint8_t *dump_sao, int16_t *dump_final,
                            uint8_t *bytes, uint32_t cap, uint32_t *nbytes)
{
    evxref_ctx *c = (evxref_ctx *)p;
    evx_frame frame;
    memcpy(&frame, frame18, sizeof(evx_frame));
    uint32_t nblk = c->ctx.width_in_blocks * c->ctx.height_in_blocks;

    image input;
    if (create_image(EVX_IMAGE_FORMAT_R8G8B8, (void *)rgb, w, h, &input) != EVX_SUCCESS) return 100;
    if (convert_image(input, &c->ctx.cache_bank.input_cache) != EVX_SUCCESS) return 101;
    copy_set(c->ctx.cache_bank.input_cache, dump_src, c->w, c->h);

    evx_status s = use_wpp ? encode_slice_wpp(frame, &c->ctx) : encode_slice(frame, &c->ctx);
    if (s != EVX_SUCCESS) return 102;
    image_set &dest = c->ctx.cache_bank.prediction_cache[frame.dpb_slot];
    if (dump_blocks) memcpy(dump_blocks, c->ctx.block_table, (size_t)nblk * 28);
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

    if (frame.type != EVX_FRAME_BIDIR)
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
    evx_frame frame;
    memcpy(&frame, frame18, sizeof(evx_frame));
    uint32_t nblk = c->ctx.width_in_blocks * c->ctx.height_in_blocks;
    memcpy(c->ctx.block_table, blocks, (size_t)nblk * 28);
    memcpy(c->ctx.prev_block_table, prev_blocks, (size_t)nblk * 28);
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

float evxref_lambda(uint16_t q) { return compute_lambda(q); }

uint32_t evxref_sizeof_block_desc(void) { return sizeof(evx_block_desc); }

} /* extern "C" */
