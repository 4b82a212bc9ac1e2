/*
 * evxg_binding.cpp -- the reference-side binding of this library, as a
 * maintainer of the reference would add it: engine_encode_frame
 * (src/video/encode.cpp:945-1001, declared in src/video/evx3enc.cpp:11)
 * reimplemented over include/evxg.h.  The pixel pipeline runs on the GPU
 * (evxg_encode_frame), the tables come back (evxg_fetch_tables) and the
 * library's host entropy coder writes the slice (evxg_serialize_slice) into
 * the reference's bit_stream.
 *
 * TEST INFRASTRUCTURE: compiled against the reference's own headers, so the
 * layout checks below compare the real structs, and linked by oracle/Makefile
 * into a copy of the reference library from which encode.cpp is left out;
 * the reference's unmodified evx3_encoder (evx3enc.cpp) then drives the GPU
 * through this function, and tests/test_gpu_binding.py requires its stream
 * to equal the unmodified reference's.  Nothing in the product links it.
 */
#include "evx3enc.h"
#include "common.h"
#include "image.h"
#include "bitstream.h"
#include "sao.h"

#include <cstddef>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "evxg.h"

using namespace evx;

// The wire structs: the library's are the default build's; a build without
// B frames uses their prefix (common.h:72-115).
static_assert(offsetof(evx_block_desc, prediction_target) == offsetof(evxg_block_desc, prediction_target), "layout");
static_assert(offsetof(evx_block_desc, motion_x) == offsetof(evxg_block_desc, motion_x), "layout");
static_assert(offsetof(evx_block_desc, q_index) == offsetof(evxg_block_desc, q_index), "layout");
static_assert(offsetof(evx_block_desc, variance) == offsetof(evxg_block_desc, variance), "layout");
static_assert(offsetof(evx_frame, quality) == offsetof(evxg_frame, quality), "layout");
#if EVX_ENABLE_B_FRAMES
static_assert(sizeof(evx_block_desc) == sizeof(evxg_block_desc) && sizeof(evx_frame) == sizeof(evxg_frame), "layout");
static_assert(offsetof(evx_block_desc, sp_index_b) == offsetof(evxg_block_desc, sp_index_b), "layout");
static_assert(offsetof(evx_frame, ref_slot_bwd) == offsetof(evxg_frame, ref_slot_bwd), "layout");
#else
static_assert(sizeof(evx_block_desc) == 18 && sizeof(evx_frame) == 10, "layout");
#endif
static_assert(sizeof(evx_sao_info) == sizeof(evxg_sao_info), "layout");

namespace {

// One GPU stream per encoder context and its host copies of the tables.
struct Gpu {
    evxg_stream *st = nullptr;
    uint32_t w = 0, h = 0, aw = 0, ah = 0;
    std::vector<evxg_block_desc> bt, prev;
    std::vector<evxg_sao_info> sao;
    std::vector<int16_t> lev;
    std::vector<uint8_t> bytes;
};
std::mutex g_mu;
std::map<const evx_context *, Gpu> g_gpu;

evxg_config build_config()
{
    evxg_config c;
    c.b_frames = EVX_ENABLE_B_FRAMES;
    c.ref_count = EVX_REFERENCE_FRAME_COUNT;
    c.search_radius = 16;   // EVX_MOTION_SEARCH_RADIUS (motion.cpp:29)
    c.reserved = 0;
    return c;
}

}  // namespace

namespace evx {

evx_status engine_encode_frame(const image &input, const evx_frame &frame, evx_context *context, bit_stream *output)
{
    const evxg_config cfg = build_config();
    Gpu *g;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g = &g_gpu[context];
    }
    const uint32_t w = input.query_width(), h = input.query_height();
    if (!g->st || frame.index == 0 || w != g->w || h != g->h) {   // a new coding session on this context
        if (g->st) evxg_stream_destroy(g->st);
        g->st = nullptr;
        if (evxg_stream_create_config(w, h, &cfg, &g->st)) return EVX_ERROR_EXECUTION_FAILURE;
        uint32_t mbw = 0, mbh = 0;
        evxg_stream_dims(g->st, &g->aw, &g->ah, &mbw, &mbh);
        g->w = w; g->h = h;
        g->bt.resize((size_t)mbw * mbh);
        g->prev.resize((size_t)mbw * mbh);
        g->sao.resize((size_t)mbw * mbh);
        g->lev.resize((size_t)g->aw * g->ah * 3 / 2);
        g->bytes.resize((size_t)g->aw * g->ah * 4);
    }
    evxg_frame f;
    std::memset(&f, 0, sizeof f);
    std::memcpy(&f, &frame, sizeof(evx_frame));   // the build's evx_frame is a prefix of evxg_frame
    uint64_t n = 0;
    if (evxg_encode_frame(g->st, input.query_data(), 0, &f, nullptr) ||
        evxg_fetch_tables(g->st, g->bt.data(), g->prev.data(), g->sao.data(), g->lev.data(), 0, nullptr) ||
        evxg_serialize_slice(&cfg, g->aw, g->ah, &f, g->bt.data(), g->prev.data(), g->sao.data(), g->lev.data(),
                             g->bytes.data(), g->bytes.size(), &n))
        return EVX_ERROR_EXECUTION_FAILURE;
    return output->write_bytes(g->bytes.data(), (uint32)n);
}

}  // namespace evx
