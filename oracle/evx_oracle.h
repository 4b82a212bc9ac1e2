/*
 * evx_oracle.h -- CPU restatement (plain C) of the EVX3 encoder's per-frame
 * pixel pipeline, used ONLY as test infrastructure: the parity checker for the
 * CUDA path and the "port" CPU baseline.  The product never links it.
 *
 * Parity is pinned: tests/test_oracle_pin.py compares every stage of this
 * restatement byte for byte with the unmodified reference library built by
 * oracle/Makefile (oracle/_ref/libevxref.so) on seeded inputs, and with the
 * committed fixtures in tests/golden/.
 *
 * Plane sets are int16, laid out Y (w*h) then U then V ((w/2)*(h/2) each),
 * pitch = width, exactly like the reference's image_set (imageset.cpp:33-53).
 */
#ifndef EVX_ORACLE_H
#define EVX_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

orc_ctx *orc_create(uint32_t aligned_w, uint32_t aligned_h);
void orc_destroy(orc_ctx *c);

/* The reference build being restated (compile-time switches there):
 * b_frames = EVX_ENABLE_B_FRAMES (1 default; 0 = I/P GOP whose P frames search
 * the slots at offsets 1 .. ref_count-1 from the frame index), ref_count =
 * EVX_REFERENCE_FRAME_COUNT (4 default; 2 or 4 without B frames), radius =
 * EVX_MOTION_SEARCH_RADIUS (16 default, or 32).  Non-zero for an unsupported
 * combination.  Call before the first frame. */
int orc_set_config(orc_ctx *c, int b_frames, int ref_count, int radius);

/* One frame of engine_encode_frame minus serialization (encode.cpp:945-998).
 * frame18: 18-byte packed evx_frame.  Dumps may be NULL; same layouts as the
 * reference harness (blocks: 28 B per MB, sao: 16 B per MB). */
int orc_encode_frame(orc_ctx *c, const uint8_t *rgb, uint32_t w, uint32_t h,
                     const uint8_t *frame18,
                     int16_t *dump_src, uint8_t *dump_blocks, int16_t *dump_levels,
                     int16_t *dump_recon, int16_t *dump_deblock,
                     uint8_t *dump_sao, int16_t *dump_final);

/* Accessors for the persistent per-stream state. */
int orc_get_slot(orc_ctx *c, uint32_t slot, int16_t *out);
int orc_get_prev_blocks(orc_ctx *c, uint8_t *out);
int orc_get_levels(orc_ctx *c, int16_t *out);

/* Unit entry points (known-answer tests restated from the reference suite). */
float orc_lambda(uint16_t quality);
void orc_hadamard_4x4(const int16_t *src, int32_t stride, int32_t *out);
int32_t orc_satd_16x16(const int16_t *a, int32_t as, const int16_t *b, int32_t bs);
void orc_interpolate(const int16_t *planes, int32_t w, int32_t h, int32_t base_x, int32_t base_y,
                     int16_t dir_x, int16_t dir_y, int32_t quarter, int16_t *out /* 16x16 + 2x8x8 */);
void orc_fdct_8x8(const int16_t *src, int32_t sp, int16_t *dst, int32_t dp);
void orc_idct_8x8(const int16_t *src, int32_t sp, int16_t *dst, int32_t dp);
void orc_intra_predict(uint8_t mode, const int16_t *planes, int32_t w, int32_t h,
                       int32_t px, int32_t py, int16_t *out /* 16x16 + 2x8x8 */);
void orc_mv_predictor(const uint8_t *blocks, const uint8_t *prev_blocks, uint32_t mbw,
                      uint32_t index, int16_t *px, int16_t *py);
uint8_t orc_deblock_strength(int32_t mb_boundary, const uint8_t *left_desc, const uint8_t *right_desc);
void orc_convert(const uint8_t *rgb, uint32_t w, uint32_t h, int16_t *planes, uint32_t aw, uint32_t ah);
void orc_yuv_to_rgb(const int16_t *planes, uint32_t aw, uint32_t ah, uint32_t w, uint32_t h, uint8_t *rgb);

#ifdef __cplusplus
}
#endif
#endif
