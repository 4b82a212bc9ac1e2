/*
 * evx_oracle.c -- plain-C restatement of the EVX3 encoder per-frame pixel
 * pipeline (ramenhut/chicago, src/video).  TEST INFRASTRUCTURE ONLY: it is the
 * parity checker for the CUDA kernels and the scalar CPU baseline; nothing in
 * the product links or calls it.
 *
 * Every function names the reference lines it restates.  Paths are relative
 * to the reference project root.  The restatement runs the sequential raster
 * schedule (encode.cpp:752-813), which the reference's WPP schedule
 * reproduces byte for byte.  Integer semantics of C are kept on purpose:
 * truncating division, int16 stores that wrap, int32 products that wrap.
 */
#include "evx_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef int16_t i16;
typedef int32_t i32;
typedef uint8_t u8;
typedef uint16_t u16;
typedef uint32_t u32;

/* ---------- wire structs (common.h:52-119 pack(2); sao.h:66-78) ---------- */
#pragma pack(push, 2)
typedef struct blk {
    i32 block_type;
    u8 prediction_target;
    u8 pad0;
    i16 motion_x, motion_y;
    u8 sp_pred, sp_amount, sp_index, q_index, intra_mode, pad1;
    i16 variance;
    u8 prediction_mode, prediction_target_b;
    i16 motion_x_b, motion_y_b;
    u8 sp_pred_b, sp_amount_b, sp_index_b, pad2;
} blk;
typedef struct frm {
    i32 type;
    u32 index;
    u16 quality;
    u32 display_order;
    u8 is_reference, dpb_slot, ref_slot_fwd, ref_slot_bwd;
} frm;
#pragma pack(pop)
typedef struct saop { u8 type, eo_class, band_position; int8_t off[4]; } saop;
typedef struct saoi { u8 merge_left, merge_above; saop luma, chroma; } saoi;

_Static_assert(sizeof(blk) == 28, "blk");
_Static_assert(sizeof(frm) == 18, "frm");
_Static_assert(sizeof(saoi) == 16, "saoi");

/* block type bits (types.h:63-91) */
#define BT_INTRA 1
#define BT_MOTION 2
#define BT_COPY 4
#define IS_INTRA(t) (!!((t)&1))
#define IS_MOTION(t) (!!((t)&2))
#define IS_COPY(t) (!!((t)&4))
enum { INTRA_DEFAULT = 1, INTRA_MOTION_COPY = 7, INTRA_MOTION_DELTA = 3, INTER_COPY = 4,
       INTER_DELTA = 0, INTER_MOTION_COPY = 6, INTER_MOTION_DELTA = 2 };
enum { F_INTRA = 0, F_INTER = 1, F_BIDIR = 2 };
#define MODE_NONE 7
#define SAD_THRESHOLD 8192   /* motion.cpp:24 */
/* EVX_MOTION_SEARCH_RADIUS (motion.cpp:29) is 16 in the default build; the
 * context carries it (orc_set_config) so that build variants can be restated. */
#define MAXQ 63              /* quantize.h:42 (levels - 1) */

/* ---------- integer helpers (evx_math.h) ---------- */
static inline u8 lg2(u32 v) /* evx_math.h:69-113: floor(log2), log2(0)=0 */
{
    u8 r = 0;
    while (v >>= 1) r++;
    return r;
}
static inline i32 req_bits8(i32 x) { return lg2((u8)x) + 1; } /* evx_required_bits on a uint8 cast */
static inline i32 rdiv(i32 n, i32 d)                            /* rounded_div, evx_math.h:228-236 */
{
    if ((n < 0) != (d < 0)) return (n - d / 2) / d;
    return (n + d / 2) / d;
}
static inline i32 iabs32(i32 v) { return v == INT32_MIN ? INT32_MAX : (v < 0 ? -v : v); }
static inline i16 iabs16(i16 v) { return v == INT16_MIN ? INT16_MAX : (i16)(v < 0 ? -v : v); }
static inline i16 sgn16(i16 v) { return (i16)((v > 0) - (v < 0)); }
static inline i32 imin(i32 a, i32 b) { return a < b ? a : b; }
static inline i32 imax(i32 a, i32 b) { return a > b ? a : b; }
static inline i32 wmul(i32 a, i32 b) { return (i32)((u32)a * (u32)b); }  /* wrapping int32 product */

float orc_lambda(u16 q) { return 0.85f * powf(2.0f, ((float)q - 12.0f) / 3.0f); } /* common.h:264-266 */

/* ---------- plane sets and macroblock views ---------- */
typedef struct pset { i16 *y, *u, *v; i32 w, h; } pset;  /* chroma planes are (w/2)x(h/2) */
typedef struct mbv { i16 *y, *u, *v; i32 s; } mbv;        /* luma stride s, chroma stride s/2 */

static pset pset_wrap(i16 *base, i32 w, i32 h)
{
    pset p; p.w = w; p.h = h; p.y = base; p.u = base + (size_t)w * h;
    p.v = p.u + (size_t)(w / 2) * (h / 2); return p;
}
static mbv mb_at(const pset *p, i32 x, i32 y) /* macroblock.h:81-87, chroma at (x>>1, y>>1) */
{
    mbv m; m.s = p->w;
    m.y = p->y + (size_t)y * p->w + x;
    m.u = p->u + (size_t)(y >> 1) * (p->w / 2) + (x >> 1);
    m.v = p->v + (size_t)(y >> 1) * (p->w / 2) + (x >> 1);
    return m;
}
typedef struct mbbuf { i16 y[256], u[64], v[64]; } mbbuf;  /* a standalone 16x16+2x8x8 block */
static mbv mb_buf(mbbuf *b) { mbv m; m.y = b->y; m.u = b->u; m.v = b->v; m.s = 16; return m; }

static void mb_copy(mbv s, mbv d) /* macroblock.h:168-180 */
{
    for (int j = 0; j < 16; j++) for (int i = 0; i < 16; i++) d.y[j * d.s + i] = s.y[j * s.s + i];
    for (int j = 0; j < 8; j++) for (int i = 0; i < 8; i++) {
        d.u[j * (d.s / 2) + i] = s.u[j * (s.s / 2) + i];
        d.v[j * (d.s / 2) + i] = s.v[j * (s.s / 2) + i];
    }
}

/* ---------- block metrics (analysis.h) ---------- */
void orc_hadamard_4x4(const i16 *src, i32 stride, i32 *out) /* analysis.h:44-85 */
{
    i32 t[16];
    for (int r = 0; r < 4; r++) {
        i32 a = src[r * stride], b = src[r * stride + 1], c = src[r * stride + 2], d = src[r * stride + 3];
        t[r * 4 + 0] = (a + b) + (c + d); t[r * 4 + 1] = (a - b) + (c - d);
        t[r * 4 + 2] = (a + b) - (c + d); t[r * 4 + 3] = (a - b) - (c - d);
    }
    for (int c = 0; c < 4; c++) {
        i32 a = t[c], b = t[4 + c], cc = t[8 + c], d = t[12 + c];
        out[c] = (a + b) + (cc + d); out[4 + c] = (a - b) + (cc - d);
        out[8 + c] = (a + b) - (cc + d); out[12 + c] = (a - b) - (cc - d);
    }
}
static i32 satd16(const i16 *a, i32 as, const i16 *b, i32 bs) /* analysis.h:89-116 */
{
    i32 acc = 0; i16 d[16]; i32 h[16];
    for (int by = 0; by < 16; by += 4) for (int bx = 0; bx < 16; bx += 4) {
        for (int r = 0; r < 4; r++) for (int c = 0; c < 4; c++)
            d[r * 4 + c] = (i16)(a[(by + r) * as + bx + c] - b[(by + r) * bs + bx + c]);
        orc_hadamard_4x4(d, 4, h);
        for (int k = 0; k < 16; k++) acc += iabs32(h[k]);
    }
    return (acc + 1) >> 1;
}
i32 orc_satd_16x16(const i16 *a, i32 as, const i16 *b, i32 bs) { return satd16(a, as, b, bs); }
static i32 sad_y(mbv a, mbv b) /* analysis.h:119-131 */
{
    i32 s = 0;
    for (int j = 0; j < 16; j++) for (int i = 0; i < 16; i++) s += iabs32(a.y[j * a.s + i] - b.y[j * b.s + i]);
    return s;
}
static i32 sad_self(mbv a) /* analysis.h:133-145 */
{
    i32 s = 0;
    for (int j = 0; j < 16; j++) for (int i = 0; i < 16; i++) s += iabs16(a.y[j * a.s + i]);
    return s;
}
static i32 mad3(mbv a, mbv b) /* analysis.h:180-202: max abs diff over Y, U and V */
{
    i32 m = 0;
    for (int j = 0; j < 16; j++) for (int i = 0; i < 16; i++) m = imax(m, iabs32(a.y[j * a.s + i] - b.y[j * b.s + i]));
    for (int j = 0; j < 8; j++) for (int i = 0; i < 8; i++) {
        m = imax(m, iabs32(a.u[j * (a.s / 2) + i] - b.u[j * (b.s / 2) + i]));
        m = imax(m, iabs32(a.v[j * (a.s / 2) + i] - b.v[j * (b.s / 2) + i]));
    }
    return m;
}
static i32 variance2(mbv a) /* analysis.h:251-275, int32 wrapping kept */
{
    i32 sum = 0, sq = 0, cnt = 0;
    for (int j = 0; j < 16; j++) for (int i = 0; i < 16; i++) {
        if (i == 0 && j == 0) continue;
        i32 t = a.y[j * a.s + i];
        if (t) { sum = (i32)((u32)sum + (u32)t); sq = (i32)((u32)sq + (u32)wmul(t, t)); cnt++; }
    }
    return cnt > 0 ? (i32)((u32)sq - (u32)rdiv(wmul(sum, sum), cnt)) : 0;
}

/* ---------- YUV 4:2:0 -> RGB24 (convert.cpp:15-18, :75-93, :162-223) ----------
 * Each chroma sample colours a 2x2 quad; (256(Y-16) + k(C-128) + 128) >> 8
 * saturated to 0..255; the frame is cropped to w x h (the visible size). */
static u8 sat8(i32 v) { return (u8)(v < 0 ? 0 : (v > 255 ? 255 : v)); }
void orc_yuv_to_rgb(const i16 *planes, u32 aw, u32 ah, u32 w, u32 h, u8 *rgb)
{
    pset p = pset_wrap((i16 *)planes, (i32)aw, (i32)ah);
    u32 cw = w < aw ? w : aw, ch = h < ah ? h : ah;
    for (u32 y = 0; y < ch; y++) for (u32 x = 0; x < cw; x++) {
        i32 l = 256 * ((i32)p.y[(size_t)y * aw + x] - 16);
        i32 u = (i32)p.u[(size_t)(y / 2) * (aw / 2) + x / 2] - 128;
        i32 v = (i32)p.v[(size_t)(y / 2) * (aw / 2) + x / 2] - 128;
        u8 *o = rgb + ((size_t)y * w + x) * 3;
        o[0] = sat8((l + 358 * v + 128) >> 8);
        o[1] = sat8((l - 88 * u - 182 * v + 128) >> 8);
        o[2] = sat8((l + 452 * u + 128) >> 8);
    }
}

/* ---------- colour conversion (convert.cpp:11-14, :30-73, :95-160) ---------- */
void orc_convert(const u8 *rgb, u32 w, u32 h, i16 *planes, u32 aw, u32 ah)
{
    pset p = pset_wrap(planes, (i32)aw, (i32)ah);
    u32 cw = w < aw ? w : aw, ch = h < ah ? h : ah;
    for (u32 y = 0; y < ch; y += 2) {
        for (u32 x = 0; x < cw; x += 2) {
            i32 u = 0, v = 0;
            for (int dy = 0; dy < 2; dy++) for (int dx = 0; dx < 2; dx++) {
                const u8 *px = rgb + ((size_t)(y + dy) * w + x + dx) * 3;
                i32 r = px[0], g = px[1], b = px[2];
                p.y[(size_t)(y + dy) * aw + x + dx] = (i16)(((77 * r + 150 * g + 29 * b + 128) >> 8) + 16);
                u = (i16)(u + ((-43 * r - 85 * g + 128 * b + 128) / 256) + 128);
                v = (i16)(v + ((128 * r - 107 * g - 21 * b + 128) / 256) + 128);
            }
            p.u[(size_t)(y / 2) * (aw / 2) + x / 2] = (i16)((u + 2) >> 2);
            p.v[(size_t)(y / 2) * (aw / 2) + x / 2] = (i16)((v + 2) >> 2);
        }
    }
}

/* ---------- 6-tap sub-pel interpolation (interp.cpp:8-202) ---------- */
static inline i16 smp(const i16 *d, i32 s, i32 x, i32 y, i32 w, i32 h)
{
    x = imax(0, imin(x, w - 1)); y = imax(0, imin(y, h - 1));
    return d[y * s + x];
}
static inline i16 tap6(i32 a, i32 b, i32 c, i32 d, i32 e, i32 f)
{
    return (i16)((a - 5 * b + 20 * c + 20 * d - 5 * e + f + 16) >> 5);
}
static void interp_plane(const i16 *d, i32 s, i32 w, i32 h, i32 bx, i32 by, int n,
                         i16 dx, i16 dy, int quarter, i16 *o, i32 os)
{
    i32 xo = dx > 0 ? 0 : -1, yo = dy > 0 ? 0 : -1;
    for (int r = 0; r < n; r++) for (int c = 0; c < n; c++) {
        i16 half;
        if (dx && !dy) {
            i32 x = bx + c + xo, y = by + r;
            half = tap6(smp(d, s, x - 2, y, w, h), smp(d, s, x - 1, y, w, h), smp(d, s, x, y, w, h),
                        smp(d, s, x + 1, y, w, h), smp(d, s, x + 2, y, w, h), smp(d, s, x + 3, y, w, h));
        } else if (!dx && dy) {
            i32 x = bx + c, y = by + r + yo;
            half = tap6(smp(d, s, x, y - 2, w, h), smp(d, s, x, y - 1, w, h), smp(d, s, x, y, w, h),
                        smp(d, s, x, y + 1, w, h), smp(d, s, x, y + 2, w, h), smp(d, s, x, y + 3, w, h));
        } else {
            /* diagonal: horizontal half-pel rows (rounded to int16) then vertical */
            i16 t[6];
            for (int k = 0; k < 6; k++) {
                i32 x = bx + c + xo, y = by + r + yo + k - 2;
                t[k] = tap6(smp(d, s, x - 2, y, w, h), smp(d, s, x - 1, y, w, h), smp(d, s, x, y, w, h),
                            smp(d, s, x + 1, y, w, h), smp(d, s, x + 2, y, w, h), smp(d, s, x + 3, y, w, h));
            }
            half = tap6(t[0], t[1], t[2], t[3], t[4], t[5]);
        }
        if (quarter) {
            i16 full = smp(d, s, bx + c, by + r, w, h);
            o[r * os + c] = (i16)((full + half + 1) >> 1);
        } else {
            o[r * os + c] = half;
        }
    }
}
static void interp_mb(const pset *p, i32 bx, i32 by, i16 dx, i16 dy, int quarter, mbv o)
{
    interp_plane(p->y, p->w, p->w, p->h, bx, by, 16, dx, dy, quarter, o.y, o.s);
    interp_plane(p->u, p->w / 2, p->w / 2, p->h / 2, bx >> 1, by >> 1, 8, dx, dy, quarter, o.u, o.s / 2);
    interp_plane(p->v, p->w / 2, p->w / 2, p->h / 2, bx >> 1, by >> 1, 8, dx, dy, quarter, o.v, o.s / 2);
}
void orc_interpolate(const i16 *planes, i32 w, i32 h, i32 bx, i32 by, i16 dx, i16 dy, i32 quarter, i16 *out)
{
    pset p = pset_wrap((i16 *)planes, w, h);
    mbv o; o.y = out; o.u = out + 256; o.v = out + 320; o.s = 16;
    interp_mb(&p, bx, by, dx, dy, quarter, o);
}

/* frac index <-> direction (motion.cpp:68-116) */
static i16 frac_from_dir(i16 i, i16 j)
{
    i++; j++;
    if (j == 0) return i;
    if (j == 1) return i == 0 ? 3 : 4;
    return (i16)(i + 5);
}
static void dir_from_frac(i16 f, i16 *dx, i16 *dy)
{
    if (f <= 2) { *dy = -1; *dx = (i16)(f - 1); }
    else if (f == 3) { *dx = -1; *dy = 0; }
    else if (f == 4) { *dx = 1; *dy = 0; }
    else { *dy = 1; *dx = (i16)(f - 6); }
}

/* ---------- intra prediction (intra_pred.cpp:13-324) ---------- */
typedef struct nbr { i16 top[16], left[16], corner; int ht, hl; } nbr;
static void neighbours(const i16 *d, i32 s, i32 cx, i32 cy, int n, nbr *o)
{
    o->ht = cy > 0; o->hl = cx > 0;
    for (int i = 0; i < n; i++) {
        o->top[i] = o->ht ? d[(cy - 1) * s + cx + i] : 128;
        o->left[i] = o->hl ? d[(cy + i) * s + cx - 1] : 128;
    }
    if (o->ht && o->hl) o->corner = d[(cy - 1) * s + cx - 1];
    else if (o->ht) o->corner = o->top[0];
    else if (o->hl) o->corner = o->left[0];
    else o->corner = 128;
}
static void predict(u8 mode, const nbr *nb, int n, i16 *o, i32 os)
{
    i16 ref[33];
    for (int i = 0; i < n; i++) ref[i] = nb->left[n - 1 - i];
    ref[n] = nb->corner;
    for (int i = 0; i < n; i++) ref[n + 1 + i] = nb->top[i];
    for (int y = 0; y < n; y++) for (int x = 0; x < n; x++) {
        i32 v;
        switch (mode) {
        case 0: { /* DC */
            i32 sum = 0, cnt = 0;
            if (nb->ht) { for (int i = 0; i < n; i++) sum += nb->top[i]; cnt += n; }
            if (nb->hl) { for (int i = 0; i < n; i++) sum += nb->left[i]; cnt += n; }
            v = cnt > 0 ? (i16)((sum + cnt / 2) / cnt) : 128;
        } break;
        case 1: v = nb->top[x]; break;
        case 2: v = nb->left[y]; break;
        case 3: {
            i32 k = x + y;
            v = (i16)((nb->top[imin(k, n - 1)] + 2 * nb->top[imin(k + 1, n - 1)] + nb->top[imin(k + 2, n - 1)] + 2) >> 2);
        } break;
        case 4: { i32 d = x - y + n; v = (i16)((ref[d - 1] + 2 * ref[d] + ref[d + 1] + 2) >> 2); } break;
        case 5: {
            i32 d = imin(imax(x - (y >> 1) + n, 1), 2 * n - 1);
            v = (y & 1) ? (i16)((ref[d - 1] + 2 * ref[d] + ref[d + 1] + 2) >> 2) : (i16)((ref[d] + ref[d + 1] + 1) >> 1);
        } break;
        case 6: {
            i32 d = imin(imax((x >> 1) - y + n, 1), 2 * n - 1);
            v = (x & 1) ? (i16)((ref[d - 1] + 2 * ref[d] + ref[d + 1] + 2) >> 2) : (i16)((ref[d] + ref[d + 1] + 1) >> 1);
        } break;
        default: v = 128;
        }
        o[y * os + x] = (i16)v;
    }
}
static void intra_pred_mb(u8 mode, const pset *rec, i32 px, i32 py, mbv o) /* intra_pred.cpp:180-217 */
{
    nbr ny, nu, nv;
    neighbours(rec->y, rec->w, px, py, 16, &ny);
    neighbours(rec->u, rec->w / 2, px >> 1, py >> 1, 8, &nu);
    neighbours(rec->v, rec->w / 2, px >> 1, py >> 1, 8, &nv);
    predict(mode, &ny, 16, o.y, o.s);
    predict(mode, &nu, 8, o.u, o.s / 2);
    predict(mode, &nv, 8, o.v, o.s / 2);
}
void orc_intra_predict(u8 mode, const i16 *planes, i32 w, i32 h, i32 px, i32 py, i16 *out)
{
    pset p = pset_wrap((i16 *)planes, w, h);
    mbv o; o.y = out; o.u = out + 256; o.v = out + 320; o.s = 16;
    intra_pred_mb(mode, &p, px, py, o);
}
static void intra_candidates(const pset *rec, i32 px, i32 py, u8 c[3]) /* intra_pred.cpp:225-260, :291-324 */
{
    nbr nb; neighbours(rec->y, rec->w, px, py, 16, &nb);
    i32 gh = 0, gv = 0;
    if (nb.ht) for (int i = 1; i < 16; i++) gh += iabs32(nb.top[i] - nb.top[i - 1]);
    if (nb.hl) for (int i = 1; i < 16; i++) gv += iabs32(nb.left[i] - nb.left[i - 1]);
    c[0] = 0;
    if (gv > gh * 3 / 2) { c[1] = 2; c[2] = 6; }
    else if (gh > gv * 3 / 2) { c[1] = 1; c[2] = 5; }
    else { c[1] = 3; c[2] = 4; }
}
static u8 best_intra_mode(mbv src, const pset *rec, i32 px, i32 py, i32 *out_sad) /* intra_pred.cpp:219-289 */
{
    u8 c[3]; intra_candidates(rec, px, py, c);
    i32 best = INT32_MAX; u8 bm = 0; mbbuf b;
    for (int k = 0; k < 3; k++) {
        intra_pred_mb(c[k], rec, px, py, mb_buf(&b));
        i32 s = sad_y(src, mb_buf(&b));
        if (s < best) { best = s; bm = c[k]; }
    }
    *out_sad = best;
    return bm;
}

/* ---------- 8x8 integer DCT (transform.cpp:264-452; xftables.h:57-67) ---------- */
static const i16 LUT8[64] = {
    128, 128, 128, 128, 128, 128, 128, 128, 126, 106, 71, 25, -25, -71, -106, -126,
    118, 49, -49, -118, -118, -49, 49, 118, 106, -25, -126, -71, 71, 126, 25, -106,
    91, -91, -91, 91, 91, -91, -91, 91, 71, -126, 25, 106, -106, -25, 126, -71,
    49, -118, 118, -49, -49, 118, -118, 49, 25, -71, 106, -126, 126, -106, 71, -25};
static void fdct_line(const i16 *s, i32 sp, i16 *d, i32 dp)
{
    for (int i = 0; i < 8; i++) {
        i32 t = 0;
        for (int k = 0; k < 8; k++) t += s[k * sp] * LUT8[i * 8 + k];
        t = i == 0 ? (t * 45) / 128 : t / 2;
        d[i * dp] = (i16)rdiv(t, 128);
    }
}
static void idct_line(const i16 *s, i32 sp, i16 *d, i32 dp, const i16 *add, i32 ap)
{
    for (int i = 0; i < 8; i++) {
        i32 t = ((s[0] * LUT8[i]) * 45) / 128;
        for (int k = 1; k < 8; k++) t += (s[k * sp] * LUT8[k * 8 + i]) / 2;
        t = rdiv(t, 128);
        d[i * dp] = (i16)(add ? t + add[i * ap] : t);
    }
}
/* forward: rows then columns, int16 between the passes; sub may be NULL */
static void fdct8(const i16 *s, i32 sp, const i16 *sub, i32 subp, i16 *d, i32 dp)
{
    i16 diff[64], tmp[64];
    for (int j = 0; j < 8; j++) {
        for (int i = 0; i < 8; i++) diff[j * 8 + i] = (i16)(sub ? s[j * sp + i] - sub[j * subp + i] : s[j * sp + i]);
        fdct_line(diff + j * 8, 1, tmp + j * 8, 1);
    }
    for (int j = 0; j < 8; j++) fdct_line(tmp + j, 8, d + j, dp);
}
/* inverse: columns then rows; add may be NULL */
static void idct8(const i16 *s, i32 sp, const i16 *add, i32 ap, i16 *d, i32 dp)
{
    i16 tmp[64];
    for (int j = 0; j < 8; j++) idct_line(s + j, sp, tmp + j, 8, NULL, 0);
    for (int j = 0; j < 8; j++) idct_line(tmp + j * 8, 1, d + j * dp, 1, add ? add + j * ap : NULL, 1);
}
void orc_fdct_8x8(const i16 *src, i32 sp, i16 *dst, i32 dp) { fdct8(src, sp, NULL, 0, dst, dp); }
void orc_idct_8x8(const i16 *src, i32 sp, i16 *dst, i32 dp) { idct8(src, sp, NULL, 0, dst, dp); }

/* 16x16 luma = four independent 8x8 quadrants (transform.cpp:485-494, :572-594) */
static void fdct_mb(mbv s, const mbv *sub, mbv d)
{
    for (int q = 0; q < 4; q++) {
        i32 ox = (q & 1) * 8, oy = (q >> 1) * 8;
        fdct8(s.y + oy * s.s + ox, s.s, sub ? sub->y + oy * sub->s + ox : NULL, sub ? sub->s : 0,
              d.y + oy * d.s + ox, d.s);
    }
    fdct8(s.u, s.s / 2, sub ? sub->u : NULL, sub ? sub->s / 2 : 0, d.u, d.s / 2);
    fdct8(s.v, s.s / 2, sub ? sub->v : NULL, sub ? sub->s / 2 : 0, d.v, d.s / 2);
}
static void idct_mb(mbv s, const mbv *add, mbv d)
{
    for (int q = 0; q < 4; q++) {
        i32 ox = (q & 1) * 8, oy = (q >> 1) * 8;
        idct8(s.y + oy * s.s + ox, s.s, add ? add->y + oy * add->s + ox : NULL, add ? add->s : 0,
              d.y + oy * d.s + ox, d.s);
    }
    idct8(s.u, s.s / 2, add ? add->u : NULL, add ? add->s / 2 : 0, d.u, d.s / 2);
    idct8(s.v, s.s / 2, add ? add->v : NULL, add ? add->s / 2 : 0, d.v, d.s / 2);
}

/* ---------- quantisation (quantize.cpp) ---------- */
static const i16 QM_INTRA[64] = {
    8, 10, 12, 15, 19, 23, 25, 27, 10, 12, 14, 17, 21, 25, 27, 28, 12, 14, 18, 21, 24, 26, 28, 30,
    15, 17, 21, 24, 26, 28, 30, 32, 19, 21, 24, 26, 28, 30, 32, 35, 23, 25, 26, 28, 30, 32, 35, 38,
    25, 27, 28, 30, 32, 35, 38, 41, 27, 28, 30, 32, 35, 38, 41, 45};
static const i16 QM_INTER[64] = {
    16, 17, 18, 19, 20, 21, 22, 23, 17, 18, 19, 20, 21, 22, 23, 24, 18, 19, 20, 21, 22, 23, 24, 25,
    19, 20, 21, 22, 23, 24, 26, 27, 20, 21, 22, 23, 25, 26, 27, 28, 21, 22, 23, 24, 26, 27, 28, 30,
    22, 23, 24, 26, 27, 28, 30, 31, 23, 24, 25, 27, 28, 30, 31, 33};
static const u8 DZ_INTRA[64] = {
    0, 1, 1, 1, 1, 1, 2, 2, 1, 1, 1, 1, 1, 2, 2, 2, 1, 1, 1, 1, 2, 2, 2, 2, 1, 1, 1, 2, 2, 2, 2, 3,
    1, 1, 2, 2, 2, 2, 3, 3, 1, 2, 2, 2, 2, 3, 3, 3, 2, 2, 2, 2, 3, 3, 3, 3, 2, 2, 2, 3, 3, 3, 3, 3};
static const u8 DZ_INTER[64] = {
    2, 2, 2, 3, 3, 3, 4, 4, 2, 2, 3, 3, 3, 4, 4, 4, 2, 3, 3, 3, 4, 4, 4, 4, 3, 3, 3, 4, 4, 4, 4, 4,
    3, 3, 4, 4, 4, 4, 4, 4, 3, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4};
static i16 luma_dc_scale(i16 qp) /* quantize.cpp:74-83 */
{
    if (qp < 5) return (i16)imax(qp << 1, 2);
    if (qp < 9) return (i16)(qp << 1);
    if (qp < 25) return (i16)(qp + 8);
    return (i16)((qp << 1) - 16);
}
static i16 chroma_dc_scale(i16 qp) /* quantize.cpp:85-92 */
{
    if (qp < 5) return (i16)imax(qp << 1, 2);
    if (qp < 25) return (i16)((qp + 13) >> 1);
    return (i16)(qp - 6);
}
static u8 aq_qp(u8 quality, mbv coeffs) /* quantize.cpp:97-118 */
{
    u32 var = (u32)variance2(coeffs);
    i32 idx = imin(imax(lg2(var) >> 1, 1), MAXQ);
    i16 delta = (i16)(((i16)idx - (i16)quality) >> 1);
    if (delta > 6) delta = 6;
    if (delta < -6) delta = -6;
    return (u8)imin(imax(quality + delta, 1), MAXQ);
}
static void quant8(u8 qp, int intra, int chroma, const i16 *s, i32 sp, i16 *d, i32 dp) /* quantize.cpp:120-252 */
{
    for (int j = 0; j < 8; j++) for (int k = 0; k < 8; k++) {
        i32 o = j * 8 + k; i16 sv = s[j * sp + k];
        if (intra) {
            i16 qf = (i16)rdiv(sv * 16, QM_INTRA[o]);
            if (qp >= 16 && o != 0) {
                i16 dz = (i16)((sgn16(qf) * qp * DZ_INTRA[o]) >> 1);
                qf = (i16)(qf - dz);
            }
            d[j * dp + k] = (i16)rdiv(qf, qp << 1);
        } else {
            i16 qf = (i16)rdiv(sv * 16, QM_INTER[o]);
            i16 wgt = DZ_INTER[o];
            if (qp >= 16) wgt = (i16)imin(wgt + 1, 6);
            i16 dz = (i16)((sgn16(qf) * qp * wgt) >> 1);
            d[j * dp + k] = (i16)rdiv(qf - dz, qp << 1);
        }
    }
    if (intra) d[0] = (i16)rdiv(s[0], chroma ? chroma_dc_scale(qp) : luma_dc_scale(qp));
}
static i16 dq_coeff(i16 lv, u8 qp, int o, int intra, int chroma) /* quantize.cpp:271-332, :481-514 */
{
    if (intra && o == 0) return (i16)(lv * (chroma ? chroma_dc_scale(qp) : luma_dc_scale(qp)));
    return (i16)((2 * lv * (intra ? QM_INTRA[o] : QM_INTER[o]) * qp) / 16);
}
static void dequant8(u8 qp, int intra, int chroma, const i16 *s, i32 sp, i16 *d, i32 dp)
{
    for (int j = 0; j < 8; j++) for (int k = 0; k < 8; k++) d[j * dp + k] = dq_coeff(s[j * sp + k], qp, j * 8 + k, intra, chroma);
}

/* scans (scan.h:60-70, :125-159) */
static const u8 ZIGZAG[64] = {
    0, 1, 8, 16, 9, 2, 3, 10, 17, 24, 32, 25, 18, 11, 4, 5, 12, 19, 26, 33, 40, 48, 41, 34,
    27, 20, 13, 6, 7, 14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
    58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};
static u8 scan_pos(u8 mode, int pos)
{
    if (mode == 1 || mode == 5) return (u8)pos;                           /* row-first */
    if (mode == 2 || mode == 6) return (u8)((pos & 7) * 8 + (pos >> 3));  /* column-first */
    return ZIGZAG[pos];
}
static u32 coeff_bits(i16 lv) /* quantize.cpp:517-532 (sig-map estimate) */
{
    if (lv == 0) return 1;
    u16 a = (u16)imin(iabs16(lv), 255);
    u32 b = 2;
    if (a > 1) b += 1;
    if (a > 2) b += 1 + 2 * req_bits8(a - 3 + 1);
    else b += 1;
    return b;
}
static void trellis8(u8 qp, int intra, int chroma, const i16 *tc, u8 mode, float lambda, i16 *lv)
{ /* quantize.cpp:536-613; tc and lv are contiguous 8x8 */
    int last = -1;
    for (int p = 63; p >= 0; p--) if (lv[scan_pos(mode, p)]) { last = p; break; }
    if (last < 0) return;
    for (int p = last; p >= 1; p--) {
        int o = scan_pos(mode, p); i16 l = lv[o];
        if (!l) continue;
        i32 dk = (i32)tc[o] - (i32)dq_coeff(l, qp, o, intra, chroma), dz = tc[o];
        float ck = (float)wmul(dk, dk) + lambda * (float)coeff_bits(l);
        float cz = (float)wmul(dz, dz) + lambda * (float)coeff_bits(0);
        if (cz <= ck) lv[o] = 0; else break;
    }
    last = -1;
    for (int p = 63; p >= 0; p--) if (lv[scan_pos(mode, p)]) { last = p; break; }
    if (last < 0) return;
    for (int p = 1; p <= last; p++) {
        int o = scan_pos(mode, p); i16 l = lv[o];
        if (!l) continue;
        i16 r = (i16)(l - sgn16(l));
        i32 dk = (i32)tc[o] - (i32)dq_coeff(l, qp, o, intra, chroma);
        i32 dr = (i32)tc[o] - (i32)dq_coeff(r, qp, o, intra, chroma);
        float ck = (float)wmul(dk, dk) + lambda * (float)coeff_bits(l);
        float cr = (float)wmul(dr, dr) + lambda * (float)coeff_bits(r);
        if (cr < ck) lv[o] = r;
    }
}
static u8 chroma_qp(u8 qp) { return (u8)imin(qp + 2, MAXQ); }
static int is_intra_q(i32 bt) { return IS_INTRA(bt) && !IS_MOTION(bt); } /* quantize.cpp:457 */
static void quant_mb(u8 qp, i32 bt, mbv tc, mbv d)
{
    int in = is_intra_q(bt);
    for (int q = 0; q < 4; q++) {
        i32 ox = (q & 1) * 8, oy = (q >> 1) * 8;
        quant8(qp, in, 0, tc.y + oy * tc.s + ox, tc.s, d.y + oy * d.s + ox, d.s);
    }
    quant8(chroma_qp(qp), in, 1, tc.u, tc.s / 2, d.u, d.s / 2);
    quant8(chroma_qp(qp), in, 1, tc.v, tc.s / 2, d.v, d.s / 2);
}
static void dequant_mb(u8 qp, i32 bt, mbv lv, mbv d)
{
    int in = is_intra_q(bt);
    for (int q = 0; q < 4; q++) {
        i32 ox = (q & 1) * 8, oy = (q >> 1) * 8;
        dequant8(qp, in, 0, lv.y + oy * lv.s + ox, lv.s, d.y + oy * d.s + ox, d.s);
    }
    dequant8(chroma_qp(qp), in, 1, lv.u, lv.s / 2, d.u, d.s / 2);
    dequant8(chroma_qp(qp), in, 1, lv.v, lv.s / 2, d.v, d.s / 2);
}
static void trellis_mb(u8 qp, i32 bt, mbv tc, u8 mode, float lambda, mbv lv) /* quantize.cpp:615-679 */
{
    int in = is_intra_q(bt); i16 t[64], l[64];
    for (int b = 0; b < 6; b++) {
        const i16 *ts; i16 *ls; i32 s1, s2; u8 q = b < 4 ? qp : chroma_qp(qp);
        if (b < 4) {
            i32 ox = (b & 1) * 8, oy = (b >> 1) * 8;
            ts = tc.y + oy * tc.s + ox; ls = lv.y + oy * lv.s + ox; s1 = tc.s; s2 = lv.s;
        } else {
            ts = b == 4 ? tc.u : tc.v; ls = b == 4 ? lv.u : lv.v; s1 = tc.s / 2; s2 = lv.s / 2;
        }
        for (int j = 0; j < 8; j++) for (int k = 0; k < 8; k++) { t[j * 8 + k] = ts[j * s1 + k]; l[j * 8 + k] = ls[j * s2 + k]; }
        trellis8(q, in, b >= 4, t, mode, lambda, l);
        for (int j = 0; j < 8; j++) for (int k = 0; k < 8; k++) ls[j * s2 + k] = l[j * 8 + k];
    }
}

/* ---------- encoder context ---------- */
struct orc_ctx {
    i32 w, h, mbw, mbh;
    /* compile-time switches of the reference build being restated:
     * EVX_ENABLE_B_FRAMES (config.h:120), EVX_REFERENCE_FRAME_COUNT (:39),
     * EVX_MOTION_SEARCH_RADIUS (motion.cpp:29) */
    int b_frames, ref_count, radius;
    i16 *src_mem, *lev_mem, *dpb_mem[4];
    pset src, lev, dpb[4];
    blk *bt, *prev;
    saoi *sao;
};

orc_ctx *orc_create(u32 aw, u32 ah)
{
    orc_ctx *c = (orc_ctx *)calloc(1, sizeof(orc_ctx));
    size_t n = (size_t)aw * ah + 2 * (size_t)(aw / 2) * (ah / 2);
    c->w = (i32)aw; c->h = (i32)ah; c->mbw = (i32)aw / 16; c->mbh = (i32)ah / 16;
    c->b_frames = 1; c->ref_count = 4; c->radius = 16;
    c->src_mem = (i16 *)calloc(n, 2); c->lev_mem = (i16 *)calloc(n, 2);
    c->src = pset_wrap(c->src_mem, c->w, c->h); c->lev = pset_wrap(c->lev_mem, c->w, c->h);
    for (int i = 0; i < 4; i++) { c->dpb_mem[i] = (i16 *)calloc(n, 2); c->dpb[i] = pset_wrap(c->dpb_mem[i], c->w, c->h); }
    c->bt = (blk *)calloc((size_t)c->mbw * c->mbh, sizeof(blk));
    c->prev = (blk *)calloc((size_t)c->mbw * c->mbh, sizeof(blk));
    c->sao = (saoi *)calloc((size_t)c->mbw * c->mbh, sizeof(saoi));
    return c;
}
void orc_destroy(orc_ctx *c)
{
    if (!c) return;
    free(c->src_mem); free(c->lev_mem);
    for (int i = 0; i < 4; i++) free(c->dpb_mem[i]);
    free(c->bt); free(c->prev); free(c->sao); free(c);
}
int orc_set_config(orc_ctx *c, int b_frames, int ref_count, int radius)
{
    if (b_frames ? ref_count != 4 : (ref_count != 2 && ref_count != 4)) return 1;
    if (radius != 16 && radius != 32) return 1;
    c->b_frames = b_frames; c->ref_count = ref_count; c->radius = radius;
    return 0;
}
/* Without B frames every slot follows from the frame index:
 * query_prediction_index_by_offset (common.cpp:256-259). */
static u32 slot_by_offset(const orc_ctx *c, const frm *f, u32 offset)
{
    return (f->index + (u32)c->ref_count - offset) % (u32)c->ref_count;
}
static size_t pset_n(const orc_ctx *c) { return (size_t)c->w * c->h + 2 * (size_t)(c->w / 2) * (c->h / 2); }
int orc_get_slot(orc_ctx *c, u32 slot, i16 *out) { if (slot > 3) return 1; memcpy(out, c->dpb_mem[slot], pset_n(c) * 2); return 0; }
int orc_get_prev_blocks(orc_ctx *c, u8 *out) { memcpy(out, c->prev, (size_t)c->mbw * c->mbh * 28); return 0; }
int orc_get_levels(orc_ctx *c, i16 *out) { memcpy(out, c->lev_mem, pset_n(c) * 2); return 0; }

static void clear_blk(blk *b) /* common.cpp:76-94 */
{
    memset(b, 0, sizeof(*b));
    b->block_type = INTRA_DEFAULT;
    b->intra_mode = MODE_NONE;
}

/* ---------- motion search (motion.cpp) ---------- */
typedef struct sel {
    i32 bx, by, sad, mad, ssd; float cost; i16 sp_index; u8 sp_amount, sp_enabled;
} sel;
typedef struct sparams { const pset *pred; i16 thr; i32 px, py; float lambda; } sparams;

static void eval_cand(i32 x, i32 y, const sparams *pp, mbv src, sel *s) /* motion.cpp:125-178 */
{
    mbv t = mb_at(pp->pred, x, y);
    i32 sad = sad_y(src, t);
    i32 ssd = (x - pp->px) * (x - pp->px) + (y - pp->py) * (y - pp->py);
    i32 mad = mad3(src, t);
    float cost = (float)sad;
    if (pp->lambda > 0.0f) {
        i16 mx = (i16)(x - pp->px), my = (i16)(y - pp->py);
        i32 satd = satd16(src.y, src.s, t.y, t.s);
        cost = (float)satd + pp->lambda * (float)(iabs16(mx) + iabs16(my) + 1);
    }
    if (s->mad < pp->thr) {
        if (mad < s->mad || (mad == s->mad && ssd < s->ssd)) {
            s->bx = x; s->by = y; s->sad = sad; s->ssd = ssd; s->mad = mad; s->cost = cost;
        }
    } else if ((cost < s->cost || ((cost == s->cost && ssd < s->ssd) && sad < SAD_THRESHOLD)) || mad < pp->thr) {
        s->bx = x; s->by = y; s->sad = sad; s->ssd = ssd; s->mad = mad; s->cost = cost;
    }
}
static int out_of_frame(const sparams *pp, i32 x, i32 y)
{
    return x < 0 || x > pp->pred->w - 16 || y < 0 || y > pp->pred->h - 16;
}
static int in_unstable(const sparams *pp, i32 x, i32 y) /* motion.cpp:361-365: not yet coded region */
{
    return y > pp->py - 16 && x > pp->px - 16;
}
static void step_search(int intra, i16 l, i16 t, i16 r, i16 b, i16 st, const sparams *pp, mbv src, sel *s)
{ /* motion.cpp:348-406 */
    i32 bx = s->bx, by = s->by;
    for (i16 j = t; j <= b; j += st) for (i16 i = l; i <= r; i += st) {
        i32 x = bx + i, y = by + j;
        if (intra && in_unstable(pp, x, y)) continue;
        if (out_of_frame(pp, x, y)) continue;
        eval_cand(x, y, pp, src, s);
        if (s->mad < pp->thr) return;
    }
}
static void subpel_eval(i16 i, i16 j, const sparams *pp, mbv src, sel *s) /* motion.cpp:180-261 */
{
    mbbuf cb; mbv c = mb_buf(&cb);
    for (int quarter = 0; quarter < 2; quarter++) {
        interp_mb(pp->pred, s->bx, s->by, i, j, quarter, c);
        i32 sad = sad_y(src, c), mad = mad3(src, c);
        int take = s->mad < pp->thr ? (mad < s->mad)
                                    : ((sad < s->sad && sad < SAD_THRESHOLD) || mad < pp->thr);
        if (take) {
            s->sp_enabled = 1; s->sp_amount = (u8)quarter; s->sp_index = frac_from_dir(i, j);
            s->sad = sad; s->mad = mad;
        }
    }
}
static void subpel_search(int intra, const sparams *pp, mbv src, sel *s) /* motion.cpp:408-483 */
{
    s->sp_index = 0; s->sp_amount = 0; s->sp_enabled = 0;
    for (i16 j = -1; j <= 1; j++) for (i16 i = -1; i <= 1; i++) {
        if (!i && !j) continue;
        i32 x = s->bx + i, y = s->by + j;
        if (intra && in_unstable(pp, x, y)) continue;
        if (out_of_frame(pp, x, y)) continue;
        subpel_eval(i, j, pp, src, s);
    }
}
static void fill_desc(const sel *s, i32 px, i32 py, int intra, i16 thr, blk *o)
{
    clear_blk(o);
    o->block_type = intra ? BT_INTRA : 0;
    if (s->bx != px || s->by != py || s->sp_enabled) o->block_type |= BT_MOTION;
    if (s->mad < thr) o->block_type |= BT_COPY;
    o->motion_x = (i16)(s->bx - px); o->motion_y = (i16)(s->by - py);
    o->sp_pred = s->sp_enabled; o->sp_amount = s->sp_amount; o->sp_index = (u8)s->sp_index;
}
static i32 intra_bc_search(const frm *f, orc_ctx *c, mbv src, i32 px, i32 py, blk *o) /* motion.cpp:485-565 */
{
    sel s = {px, py, sad_self(src), INT32_MAX, INT32_MAX, 0.0f, 0, 0, 0};
    s.cost = (float)s.sad;
    sparams pp = {&c->dpb[f->dpb_slot], (i16)((f->quality >> 2) + 1), px, py, orc_lambda(f->quality)};
    const i16 R = (i16)c->radius;
    step_search(1, -R, -(R << 1), R, 0, R, &pp, src, &s);
    if (s.mad >= pp.thr)
        for (i16 st = R >> 1; st > 0; st >>= 1) {
            step_search(1, -st, -st, st, st, st, &pp, src, &s);
            if (s.mad < pp.thr) break;
        }
    subpel_search(1, &pp, src, &s);
    fill_desc(&s, px, py, 1, pp.thr, o);
    o->prediction_target = 0;
    return s.sad;
}
static void mv_predictor(const blk *bt, const blk *prev, u32 mbw, u32 idx, i16 *ox, i16 *oy) /* motion.cpp:271-346 */
{
    u32 bx = idx % mbw, by = idx / mbw; i16 mx[3], my[3]; int n = 0;
    if (bx > 0 && IS_MOTION(bt[idx - 1].block_type)) { mx[n] = bt[idx - 1].motion_x; my[n++] = bt[idx - 1].motion_y; }
    if (by > 0 && IS_MOTION(bt[idx - mbw].block_type)) { mx[n] = bt[idx - mbw].motion_x; my[n++] = bt[idx - mbw].motion_y; }
    if (by > 0 && bx + 1 < mbw && IS_MOTION(bt[idx - mbw + 1].block_type)) {
        mx[n] = bt[idx - mbw + 1].motion_x; my[n++] = bt[idx - mbw + 1].motion_y;
    } else if (by > 0 && bx > 0 && IS_MOTION(bt[idx - mbw - 1].block_type)) {
        mx[n] = bt[idx - mbw - 1].motion_x; my[n++] = bt[idx - mbw - 1].motion_y;
    }
    if (n < 3 && prev && IS_MOTION(prev[idx].block_type)) { mx[n] = prev[idx].motion_x; my[n++] = prev[idx].motion_y; }
    if (n == 0) { *ox = 0; *oy = 0; }
    else if (n == 1) { *ox = mx[0]; *oy = my[0]; }
    else if (n == 2) { *ox = (i16)((mx[0] + mx[1]) / 2); *oy = (i16)((my[0] + my[1]) / 2); }
    else {
        for (int k = 0; k < 2; k++) {
            i16 *v = k ? my : mx; i16 a = v[0], b = v[1], cc = v[2], t;
            if (a > b) { t = a; a = b; b = t; }
            if (b > cc) b = cc;
            if (a > b) b = a;
            if (k) *oy = b; else *ox = b;
        }
    }
}
void orc_mv_predictor(const u8 *blocks, const u8 *prev_blocks, u32 mbw, u32 idx, i16 *px, i16 *py)
{
    mv_predictor((const blk *)blocks, (const blk *)prev_blocks, mbw, idx, px, py);
}
static i32 inter_search(const frm *f, orc_ctx *c, mbv src, i32 px, i32 py, u32 slot, u32 idx,
                        const blk *prev, blk *o) /* motion.cpp:567-679 */
{
    sparams pp = {&c->dpb[slot], (i16)((f->quality >> 2) + 1), px, py, orc_lambda(f->quality)};
    mbv t = mb_at(pp.pred, px, py);
    sel s = {px, py, sad_y(src, t), mad3(src, t), INT32_MAX, 0.0f, 0, 0, 0};
    s.cost = (float)s.sad;
    if (pp.lambda > 0.0f) s.cost = (float)satd16(src.y, src.s, t.y, t.s) + pp.lambda * 1.0f;
    i16 pmx, pmy;
    mv_predictor(c->bt, prev, (u32)c->mbw, idx, &pmx, &pmy);
    if (pmx || pmy) {
        i32 x = px + pmx, y = py + pmy;
        x = imin(imax(x, 0), c->w - 16); y = imin(imax(y, 0), c->h - 16);
        eval_cand(x, y, &pp, src, &s);
    }
    if (s.mad >= pp.thr) {
        i16 r = (i16)c->radius;
        if (s.sad < SAD_THRESHOLD / 4) r = (i16)(c->radius / 4);
        else if (s.sad < SAD_THRESHOLD / 2) r = (i16)(c->radius / 2);
        for (i16 st = r; st > 0; st >>= 1) {
            step_search(0, -st, -st, st, st, st, &pp, src, &s);
            if (s.mad < pp.thr) break;
        }
        subpel_search(0, &pp, src, &s);
    }
    fill_desc(&s, px, py, 0, pp.thr, o);
    return s.sad;
}

/* Prediction block for a motion descriptor (encode.cpp:523-724, decode.cpp:59-426). */
static void motion_pred(const pset *ref, i32 x, i32 y, u8 spp, u8 spa, u8 spi, mbbuf *tmp, mbv *out)
{
    if (spp) {
        i16 dx, dy; dir_from_frac(spi, &dx, &dy);
        interp_mb(ref, x, y, dx, dy, spa, mb_buf(tmp));
        *out = mb_buf(tmp);
    } else {
        *out = mb_at(ref, x, y);
    }
}
static void bi_average(mbv f, mbv b, mbv d)
{
    for (int j = 0; j < 16; j++) for (int i = 0; i < 16; i++)
        d.y[j * d.s + i] = (i16)((f.y[j * f.s + i] + b.y[j * b.s + i] + 1) >> 1);
    for (int j = 0; j < 8; j++) for (int i = 0; i < 8; i++) {
        d.u[j * (d.s / 2) + i] = (i16)((f.u[j * (f.s / 2) + i] + b.u[j * (b.s / 2) + i] + 1) >> 1);
        d.v[j * (d.s / 2) + i] = (i16)((f.v[j * (f.s / 2) + i] + b.v[j * (b.s / 2) + i] + 1) >> 1);
    }
}
/* The prediction a descriptor implies (NULL-equivalent flag for intra-none). */
static int build_pred(const frm *f, orc_ctx *c, const blk *d, i32 i, i32 j, mbbuf *b0, mbbuf *b1, mbbuf *b2, mbv *out)
{
    i32 bt = d->block_type;
    if (bt == INTRA_DEFAULT) {
        if (d->intra_mode == MODE_NONE) return 0;
        intra_pred_mb(d->intra_mode, &c->dpb[f->dpb_slot], i, j, mb_buf(b0));
        *out = mb_buf(b0); return 1;
    }
    if (IS_INTRA(bt)) { /* intra motion copy / delta: current frame */
        motion_pred(&c->dpb[f->dpb_slot], i + d->motion_x, j + d->motion_y, d->sp_pred, d->sp_amount, d->sp_index, b0, out);
        return 1;
    }
    if (f->type == F_BIDIR && d->prediction_mode == 2) {
        mbv fw, bw;
        if (IS_MOTION(bt)) {
            motion_pred(&c->dpb[d->prediction_target], i + d->motion_x, j + d->motion_y, d->sp_pred, d->sp_amount, d->sp_index, b0, &fw);
            motion_pred(&c->dpb[d->prediction_target_b], i + d->motion_x_b, j + d->motion_y_b, d->sp_pred_b, d->sp_amount_b, d->sp_index_b, b1, &bw);
        } else {
            fw = mb_at(&c->dpb[d->prediction_target], i, j);
            bw = mb_at(&c->dpb[d->prediction_target_b], i, j);
        }
        bi_average(fw, bw, mb_buf(b2));
        *out = mb_buf(b2); return 1;
    }
    /* with B frames the target is a DPB slot, without them an offset from the
     * frame index (encode.cpp:597-608, decode.cpp:196-203) */
    const u32 ref = c->b_frames ? d->prediction_target : slot_by_offset(c, f, d->prediction_target);
    if (IS_MOTION(bt)) motion_pred(&c->dpb[ref], i + d->motion_x, j + d->motion_y, d->sp_pred, d->sp_amount, d->sp_index, b0, out);
    else *out = mb_at(&c->dpb[ref], i, j);
    return 1;
}

/* encode_block (encode.cpp:481-750): levels into lv, sets q_index/variance. */
static void encode_block(const frm *f, orc_ctx *c, mbv src, i32 i, i32 j, blk *d, mbv lv, mbbuf *coef)
{
    if (IS_COPY(d->block_type)) return;
    mbbuf b0, b1, b2; mbv pred;
    int has = build_pred(f, c, d, i, j, &b0, &b1, &b2, &pred);
    mbv tc = mb_buf(coef);
    fdct_mb(src, has ? &pred : NULL, tc);
    d->q_index = aq_qp((u8)f->quality, tc);
    d->variance = (i16)variance2(tc);
    quant_mb(d->q_index, d->block_type, tc, lv);
    trellis_mb(d->q_index, d->block_type, tc, d->intra_mode, orc_lambda(f->quality), lv);
}
/* decode_block (decode.cpp:31-432): reconstruction into dst. */
static void decode_block(const frm *f, orc_ctx *c, const blk *d, mbv lv, i32 i, i32 j, mbv dst)
{
    mbbuf b0, b1, b2, dq; mbv pred;
    int has = build_pred(f, c, d, i, j, &b0, &b1, &b2, &pred);
    if (IS_COPY(d->block_type)) { mb_copy(pred, dst); return; }
    dequant_mb(d->q_index, d->block_type, lv, mb_buf(&dq));
    idct_mb(mb_buf(&dq), has ? &pred : NULL, dst);
}

/* ---------- RDO (encode.cpp:39-164) ---------- */
static u32 est_bits(const blk *d, mbv q)
{
    u32 bits = 3; i32 bt = d->block_type;
    if (!IS_INTRA(bt)) bits += 2;
    if (IS_MOTION(bt)) {
        bits += 2 * req_bits8(iabs16(d->motion_x) + 1) + 2 * req_bits8(iabs16(d->motion_y) + 1);
        bits += d->sp_pred ? 5 : 1;
    }
    if (IS_COPY(bt)) return bits;
    if (bt == INTRA_DEFAULT) bits += 3;
    bits += 2 * req_bits8(iabs32(d->q_index) + 1);
    for (int bj = 0; bj < 16; bj += 8) for (int bi = 0; bi < 16; bi += 8) {
        u32 nz = 0, cb = 0;
        for (int y = 0; y < 8; y++) for (int x = 0; x < 8; x++) {
            i16 v = q.y[(bj + y) * q.s + bi + x];
            if (v) {
                nz++;
                u16 a = (u16)imin(iabs16(v), 255);
                cb += 2;
                if (a > 1) cb += 1;
                if (a > 2) cb += 1 + 2 * req_bits8(a - 3 + 1);
                else cb += 1;
            }
        }
        bits += req_bits8(nz + 1) * 2 + 1 + cb;
    }
    return bits;
}
static i32 ssd_y(mbv a, mbv b)
{
    i32 s = 0;
    for (int j = 0; j < 16; j++) for (int i = 0; i < 16; i++) {
        i32 d = a.y[j * a.s + i] - b.y[j * b.s + i];
        s = (i32)((u32)s + (u32)wmul(d, d));
    }
    return s;
}
static float rdo_cost(const frm *f, orc_ctx *c, mbv src, i32 i, i32 j, blk *d, float lambda)
{
    /* The reference builds both the quantised block and the reconstruction in
     * the same staging buffer (encode.cpp:151 and :158), so decode_block
     * overwrites the levels and the rate estimate reads the reconstruction. */
    mbbuf q, r, coef; memset(&q, 0, sizeof q);
    encode_block(f, c, src, i, j, d, mb_buf(&q), &coef);
    decode_block(f, c, d, mb_buf(&q), i, j, mb_buf(&r));
    return (float)ssd_y(src, mb_buf(&r)) + lambda * (float)est_bits(d, mb_buf(&r));
}

/* ---------- per-MB classification (encode.cpp:168-477) ---------- */
static void classify(const frm *f, orc_ctx *c, mbv src, i32 i, i32 j, u32 idx, blk *out)
{
    blk best; i32 best_sad = intra_bc_search(f, c, src, i, j, &best);
    float lambda = orc_lambda(f->quality);
    if (f->type == F_BIDIR) {
        blk fw, bw; /* the bi-pred search repeats these exact searches (motion.cpp:710-726) */
        i32 fs = inter_search(f, c, src, i, j, f->ref_slot_fwd, idx, NULL, &fw);
        fw.prediction_mode = 0; fw.prediction_target = f->ref_slot_fwd;
        if (fs < best_sad) { best = fw; best_sad = fs; }
        i32 bs = inter_search(f, c, src, i, j, f->ref_slot_bwd, idx, NULL, &bw);
        bw.prediction_mode = 1; bw.prediction_target = f->ref_slot_bwd;
        if (bs < best_sad) { best = bw; best_sad = bs; }
        /* bi-prediction (motion.cpp:702-840) */
        mbbuf b0, b1; mbv fp, bp;
        motion_pred(&c->dpb[f->ref_slot_fwd], i + fw.motion_x, j + fw.motion_y, fw.sp_pred, fw.sp_amount, fw.sp_index, &b0, &fp);
        motion_pred(&c->dpb[f->ref_slot_bwd], i + bw.motion_x, j + bw.motion_y, bw.sp_pred, bw.sp_amount, bw.sp_index, &b1, &bp);
        i32 bi = 0;
        for (int y = 0; y < 16; y++) for (int x = 0; x < 16; x++) {
            i32 av = (fp.y[y * fp.s + x] + bp.y[y * bp.s + x] + 1) >> 1;
            bi += iabs32(src.y[y * src.s + x] - av);
        }
        for (int y = 0; y < 8; y++) for (int x = 0; x < 8; x++) {
            i32 au = (fp.u[y * (fp.s / 2) + x] + bp.u[y * (bp.s / 2) + x] + 1) >> 1;
            bi += iabs32(src.u[y * (src.s / 2) + x] - au);
            i32 av = (fp.v[y * (fp.s / 2) + x] + bp.v[y * (bp.s / 2) + x] + 1) >> 1;
            bi += iabs32(src.v[y * (src.s / 2) + x] - av);
        }
        if (bi + (i32)(lambda * 8.0f) < best_sad) {
            clear_blk(&best);
            best.block_type = INTER_MOTION_DELTA; best.prediction_mode = 2;
            best.prediction_target = f->ref_slot_fwd;
            best.motion_x = fw.motion_x; best.motion_y = fw.motion_y;
            best.sp_pred = fw.sp_pred; best.sp_amount = fw.sp_amount; best.sp_index = fw.sp_index;
            best.prediction_target_b = f->ref_slot_bwd;
            best.motion_x_b = bw.motion_x; best.motion_y_b = bw.motion_y;
            best.sp_pred_b = bw.sp_pred; best.sp_amount_b = bw.sp_amount; best.sp_index_b = bw.sp_index;
            best_sad = bi;
        }
        i32 ds; u8 m = best_intra_mode(src, &c->dpb[f->dpb_slot], i, j, &ds);
        if (ds < best_sad) { clear_blk(&best); best.intra_mode = m; best_sad = ds; }
        *out = best;
        return;
    }
    if (f->type == F_INTER && c->b_frames) {   /* one reference, the frame's forward slot (encode.cpp:182-209) */
        blk in; i32 is = inter_search(f, c, src, i, j, f->ref_slot_fwd, idx, c->prev, &in);
        in.prediction_target = f->ref_slot_fwd;
        if (IS_COPY(in.block_type) ^ IS_COPY(best.block_type)) {
            if (IS_COPY(in.block_type)) { best = in; best_sad = is; }
        } else if (is < best_sad) { best = in; best_sad = is; }
    } else if (f->type == F_INTER) {
        /* without B frames: every offset 1 .. EVX_REFERENCE_FRAME_COUNT-1, the
         * nearer references favoured by a distance bias (encode.cpp:211-247,
         * calculate_inter_prediction motion.cpp:681-698) */
        for (u32 off = 1; off < (u32)c->ref_count; off++) {
            blk in; i32 is = inter_search(f, c, src, i, j, slot_by_offset(c, f, off), idx, c->prev, &in);
            in.prediction_target = (u8)off;
            const i32 bias = (i32)(lambda * (float)(off * 2));
            if (IS_COPY(in.block_type) ^ IS_COPY(best.block_type)) {
                if (IS_COPY(in.block_type)) { best = in; best_sad = is; }
            } else if (is + bias < best_sad) { best = in; best_sad = is; }
        }
    }
    i32 ds; u8 m = best_intra_mode(src, &c->dpb[f->dpb_slot], i, j, &ds);
    if (ds < best_sad) { clear_blk(&best); best.intra_mode = m; best_sad = ds; }
    if (f->type == F_INTER) {
        blk cand = best; float bc = rdo_cost(f, c, src, i, j, &cand, lambda);
        best = cand;
        if (best.block_type != INTRA_DEFAULT) {
            blk id; clear_blk(&id);
            float ic = rdo_cost(f, c, src, i, j, &id, lambda);
            if (ic < bc) { best = id; bc = ic; }
        }
        u8 cm[3]; intra_candidates(&c->dpb[f->dpb_slot], i, j, cm);
        for (int k = 0; k < 3; k++) {
            blk dd; clear_blk(&dd); dd.intra_mode = cm[k];
            float dc = rdo_cost(f, c, src, i, j, &dd, lambda);
            if (dc < bc) { best = dd; bc = dc; }
        }
    }
    *out = best;
}

/* ---------- deblocking (deblock.cpp) ---------- */
static const i16 ALPHA[64] = {
    0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 2, 2, 3, 3, 4, 5, 6, 7, 8, 9, 10, 12, 14, 16, 18, 20, 22, 24, 26, 29, 32, 35,
    38, 42, 46, 50, 54, 59, 64, 70, 76, 82, 89, 96, 104, 112, 120, 128, 138, 148, 158, 170, 182, 196, 210, 224,
    240, 255, 255, 255, 255, 255, 255, 255};
static const i16 BETA[64] = {
    0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 3, 3, 3, 4, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8, 9, 10, 11,
    12, 13, 14, 15, 16, 17, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18,
    18, 18, 18, 18, 18, 18, 18, 18};
static u8 avg_qp(const blk *l, const blk *r) /* deblock.cpp:58-74 */
{
    if (!IS_COPY(l->block_type) && !IS_COPY(r->block_type)) return (u8)((l->q_index + r->q_index) >> 1);
    if (!IS_COPY(l->block_type)) return l->q_index;
    if (!IS_COPY(r->block_type)) return r->q_index;
    return 0;
}
static u8 strength(int mb_boundary, const blk *l, const blk *r) /* deblock.cpp:76-89 */
{
    int lc = IS_COPY(l->block_type), rc = IS_COPY(r->block_type);
    if (lc && rc) return 0;
    if (lc ^ rc) return 1;
    return mb_boundary ? 2 : 1;
}
uint8_t orc_deblock_strength(int32_t mbb, const uint8_t *l, const uint8_t *r)
{
    return strength(mbb, (const blk *)l, (const blk *)r);
}
/* one filtered line: p[k] = sample at -1-k from the edge, q[k] at +k; stride between samples */
static void filter_line(i16 *e, i32 step, u8 qp_eff, u8 st, int luma) /* deblock.cpp:91-146 */
{
    i16 p0 = e[-step], p1 = e[-2 * step], p2 = e[-3 * step], p3 = e[-4 * step];
    i16 q0 = e[0], q1 = e[step], q2 = e[2 * step], q3 = e[3 * step];
    u8 qi = qp_eff;
    if (st == 2 && qp_eff > 0) qi = (u8)imin(qp_eff + 2, MAXQ);
    /* abs() of the int difference, then stored to int16 (deblock.cpp:105-107) */
    if ((i16)iabs32(p0 - q0) >= ALPHA[qi] || (i16)iabs32(p1 - p0) >= BETA[qi] || (i16)iabs32(q1 - q0) >= BETA[qi]) return;
    if (st == 2) {
        e[-step] = (i16)rdiv(p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1, 8);
        e[-2 * step] = (i16)rdiv(p2 + p1 + p0 + q0, 4);
        e[0] = (i16)rdiv(p1 + 2 * p0 + 2 * q0 + 2 * q1 + q2, 8);
        e[step] = (i16)rdiv(p0 + q0 + q1 + q2, 4);
        if (luma) {
            e[-3 * step] = (i16)rdiv(2 * p3 + 3 * p2 + p1 + p0 + q0, 8);
            e[2 * step] = (i16)rdiv(2 * q3 + 3 * q2 + q1 + q0 + p0, 8);
        }
    } else if (st == 1) {
        e[-step] = (i16)rdiv(((q0 + p0) * 4) + p1 - q1, 8);
        e[0] = (i16)rdiv(((q0 + p0) * 4) + q1 - p1, 8);
        if (luma) {
            e[-2 * step] = (i16)rdiv((p2 * 4) + (p0 * 2) + (q0 * 2), 8);
            e[step] = (i16)rdiv((q2 * 4) + (q0 * 2) + (p0 * 2), 8);
        }
    }
}
static void edge(i16 *d, i32 w, const blk *bt, i32 mbs, i32 mbw, i32 x, i32 y, int vertical, int luma, i32 qoff)
{ /* deblock.cpp:148-220: vertical edge at column x (rows y..y+7) or horizontal at row y (cols x..x+7) */
    i32 li = vertical ? (x - 1) / mbs + (y / mbs) * mbw : x / mbs + ((y - 1) / mbs) * mbw;
    i32 ri = x / mbs + (y / mbs) * mbw;
    u8 aq = avg_qp(&bt[li], &bt[ri]);
    u8 st = strength(li != ri, &bt[li], &bt[ri]);
    if (!st) return;
    u8 qe = (u8)imin((i16)aq + qoff, MAXQ);
    for (int k = 0; k < 8; k++) {
        if (vertical) filter_line(d + (size_t)(y + k) * w + x, 1, qe, st, luma);
        else filter_line(d + (size_t)y * w + x + k, w, qe, st, luma);
    }
}
static void deblock_plane(i16 *d, i32 w, i32 h, const blk *bt, i32 mbs, i32 mbw, int luma, i32 qoff)
{ /* deblock.cpp:222-275 */
    for (i32 x = 8; x < w; x += 8) edge(d, w, bt, mbs, mbw, x, 0, 1, luma, qoff);
    for (i32 y = 8; y < h; y += 8) {
        edge(d, w, bt, mbs, mbw, 0, y, 0, luma, qoff);
        for (i32 x = 8; x < w; x += 8) {
            edge(d, w, bt, mbs, mbw, x, y, 0, luma, qoff);
            edge(d, w, bt, mbs, mbw, x, y, 1, luma, qoff);
        }
    }
}

/* ---------- SAO (sao.cpp) ---------- */
static const int8_t EO[4][4] = {{-1, 0, 1, 0}, {0, -1, 0, 1}, {-1, -1, 1, 1}, {1, -1, -1, 1}};
static inline i16 sclamp(i32 v) { return (i16)(v < 0 ? 0 : v > 255 ? 255 : v); }
static u8 eo_cat(i16 p, i16 a, i16 b)
{
    int s = ((a > p) - (a < p)) + ((b > p) - (b < p));
    return s == 2 ? 0 : s == 1 ? 1 : s == -1 ? 2 : s == -2 ? 3 : 4;
}
static u32 sao_bits(const saop *p)
{
    if (p->type == 0) return 2;
    u32 b = 2 + (p->type == 1 ? 2 : 5);
    for (int i = 0; i < 4; i++) b += p->off[i] ? 4 : 1;
    return b;
}
/* corrected value of pixel (x,y) under params p, reading neighbours from img */
static i16 sao_px(const i16 *img, i32 w, i32 h, i32 x, i32 y, const saop *p)
{
    i16 v = img[y * w + x];
    if (p->type == 2) {
        i32 idx = (sclamp(v) >> 3) - p->band_position;
        return (idx >= 0 && idx < 4) ? sclamp(v + p->off[idx]) : v;
    }
    if (p->type == 1) {
        i32 ax = x + EO[p->eo_class][0], ay = y + EO[p->eo_class][1];
        i32 bx = x + EO[p->eo_class][2], by = y + EO[p->eo_class][3];
        if (ax < 0 || ax >= w || ay < 0 || ay >= h || bx < 0 || bx >= w || by < 0 || by >= h) return v;
        u8 ct = eo_cat(v, img[ay * w + ax], img[by * w + bx]);
        return ct < 4 ? sclamp(v + p->off[ct]) : v;
    }
    return v;
}
static int64_t sao_ssd(const i16 *s, const i16 *r, i32 w, i32 h, i32 x0, i32 y0, i32 n, const saop *p)
{
    int64_t acc = 0;
    for (i32 y = y0; y < y0 + n; y++) for (i32 x = x0; x < x0 + n; x++) {
        i32 d = (i32)s[y * w + x] - (i32)(p ? sao_px(r, w, h, x, y, p) : r[y * w + x]);
        acc += d * d;
    }
    return acc;
}
static i32 avg_off(i32 sum, i32 cnt) /* sao.cpp:205-207 */
{
    i32 a = (sum + (sum >= 0 ? cnt / 2 : -cnt / 2)) / cnt;
    return a > 7 ? 7 : a < -7 ? -7 : a;
}
static void sao_rdo(const i16 *s, const i16 *r, i32 w, i32 h, i32 x0, i32 y0, i32 n, float lambda, saop *out)
{ /* sao.cpp:150-343 */
    memset(out, 0, sizeof *out);
    float best = (float)sao_ssd(s, r, w, h, x0, y0, n, NULL) + lambda * (float)sao_bits(out);
    i32 bs[32] = {0}, bc[32] = {0};
    for (i32 y = y0; y < y0 + n; y++) for (i32 x = x0; x < x0 + n; x++) {
        i32 b = sclamp(r[y * w + x]) >> 3;
        bs[b] += (i32)s[y * w + x] - (i32)r[y * w + x]; bc[b]++;
    }
    for (int bp = 0; bp <= 28; bp++) {
        saop c; memset(&c, 0, sizeof c); c.type = 2; c.band_position = (u8)bp;
        int nz = 0;
        for (int k = 0; k < 4; k++) { c.off[k] = bc[bp + k] > 0 ? (int8_t)avg_off(bs[bp + k], bc[bp + k]) : 0; nz |= c.off[k] != 0; }
        if (!nz) continue;
        float cost = (float)sao_ssd(s, r, w, h, x0, y0, n, &c) + lambda * (float)sao_bits(&c);
        if (cost < best) { best = cost; *out = c; }
    }
    for (int ec = 0; ec < 4; ec++) {
        i32 cs[4] = {0}, cc[4] = {0};
        for (i32 y = y0; y < y0 + n; y++) for (i32 x = x0; x < x0 + n; x++) {
            i32 ax = x + EO[ec][0], ay = y + EO[ec][1], bx = x + EO[ec][2], by = y + EO[ec][3];
            if (ax < 0 || ax >= w || ay < 0 || ay >= h || bx < 0 || bx >= w || by < 0 || by >= h) continue;
            u8 ct = eo_cat(r[y * w + x], r[ay * w + ax], r[by * w + bx]);
            if (ct < 4) { cs[ct] += (i32)s[y * w + x] - (i32)r[y * w + x]; cc[ct]++; }
        }
        saop c; memset(&c, 0, sizeof c); c.type = 1; c.eo_class = (u8)ec;
        int nz = 0;
        for (int k = 0; k < 4; k++) { c.off[k] = cc[k] > 0 ? (int8_t)avg_off(cs[k], cc[k]) : 0; nz |= c.off[k] != 0; }
        if (!nz) continue;
        float cost = (float)sao_ssd(s, r, w, h, x0, y0, n, &c) + lambda * (float)sao_bits(&c);
        if (cost < best) { best = cost; *out = c; }
    }
}
static void sao_apply_mb(i16 *img, i32 w, i32 h, i32 x0, i32 y0, i32 n, const saop *p) /* sao.cpp:40-97 */
{
    i16 v[256];
    for (i32 y = 0; y < n; y++) for (i32 x = 0; x < n; x++) v[y * n + x] = sao_px(img, w, h, x0 + x, y0 + y, p);
    for (i32 y = 0; y < n; y++) for (i32 x = 0; x < n; x++) img[(y0 + y) * w + x0 + x] = v[y * n + x];
}
static void sao_frame(orc_ctx *c, pset *rec, float lambda) /* sao.cpp:389-594 (luma-only merge branch) */
{
    i32 cw = c->w / 2, ch = c->h / 2;
    for (i32 by = 0; by < c->mbh; by++) for (i32 bx = 0; bx < c->mbw; bx++) {
        i32 m = by * c->mbw + bx; saoi *in = &c->sao[m];
        memset(in, 0, sizeof *in);
        sao_rdo(c->src.y, rec->y, c->w, c->h, bx * 16, by * 16, 16, lambda, &in->luma);
        sao_rdo(c->src.u, rec->u, cw, ch, bx * 8, by * 8, 8, lambda, &in->chroma);
        float cur;
        if (in->luma.type == 0) cur = (float)sao_ssd(c->src.y, rec->y, c->w, c->h, bx * 16, by * 16, 16, NULL) + lambda * 2.0f;
        else cur = ((float)sao_ssd(c->src.y, rec->y, c->w, c->h, bx * 16, by * 16, 16, &in->luma) + lambda * 1.0f)
                   - lambda * 1.0f + lambda * (float)sao_bits(&in->luma);
        if (bx > 0 && c->sao[m - 1].luma.type != 0) {
            float mc = (float)sao_ssd(c->src.y, rec->y, c->w, c->h, bx * 16, by * 16, 16, &c->sao[m - 1].luma) + lambda * 1.0f;
            if (mc < cur) { in->merge_left = 1; in->luma = c->sao[m - 1].luma; in->chroma = c->sao[m - 1].chroma; cur = mc; }
        }
        if (!in->merge_left && by > 0 && c->sao[m - c->mbw].luma.type != 0) {
            float mc = (float)sao_ssd(c->src.y, rec->y, c->w, c->h, bx * 16, by * 16, 16, &c->sao[m - c->mbw].luma) + lambda * 1.0f;
            if (mc < cur) { in->merge_above = 1; in->luma = c->sao[m - c->mbw].luma; in->chroma = c->sao[m - c->mbw].chroma; }
        }
    }
    /* raster in-place application, Y then U then V (sao.cpp:99-146) */
    for (int pl = 0; pl < 3; pl++) {
        i16 *img = pl == 0 ? rec->y : pl == 1 ? rec->u : rec->v;
        i32 w = pl ? cw : c->w, h = pl ? ch : c->h, n = pl ? 8 : 16;
        for (i32 by = 0; by < c->mbh; by++) for (i32 bx = 0; bx < c->mbw; bx++) {
            const saop *p = pl ? &c->sao[by * c->mbw + bx].chroma : &c->sao[by * c->mbw + bx].luma;
            if (p->type) sao_apply_mb(img, w, h, bx * n, by * n, n, p);
        }
    }
}

/* ---------- frame driver (encode.cpp:945-998 minus serialize_slice) ---------- */
static void dump_pset(const orc_ctx *c, const i16 *mem, i16 *out) { if (out) memcpy(out, mem, pset_n(c) * 2); }

int orc_encode_frame(orc_ctx *c, const u8 *rgb, u32 w, u32 h, const u8 *frame18,
                     i16 *dump_src, u8 *dump_blocks, i16 *dump_levels, i16 *dump_recon,
                     i16 *dump_deblock, u8 *dump_sao, i16 *dump_final)
{
    frm f; memcpy(&f, frame18, sizeof f);
    if ((w | h) & 1) return 1;
    if (!c->b_frames) {   /* the destination follows from the index (encode.cpp:952-956) */
        if (f.type == F_BIDIR) return 1;
        f.dpb_slot = (u8)slot_by_offset(c, &f, 0);
        f.ref_slot_fwd = (u8)slot_by_offset(c, &f, 1);
        f.ref_slot_bwd = 0;
    }
    if (f.dpb_slot > 3 || f.ref_slot_fwd > 3 || f.ref_slot_bwd > 3) return 1;
    orc_convert(rgb, w, h, c->src_mem, (u32)c->w, (u32)c->h);
    dump_pset(c, c->src_mem, dump_src);
    pset *dst = &c->dpb[f.dpb_slot];
    u32 idx = 0;
    for (i32 j = 0; j < c->h; j += 16) for (i32 i = 0; i < c->w; i += 16, idx++) {
        mbv src = mb_at(&c->src, i, j), lv = mb_at(&c->lev, i, j), rc = mb_at(dst, i, j);
        blk *d = &c->bt[idx];
        classify(&f, c, src, i, j, idx, d);
        mbbuf coef;
        encode_block(&f, c, src, i, j, d, lv, &coef);
        decode_block(&f, c, d, lv, i, j, rc);
    }
    if (dump_blocks) memcpy(dump_blocks, c->bt, (size_t)c->mbw * c->mbh * 28);
    dump_pset(c, c->lev_mem, dump_levels);
    dump_pset(c, dst->y, dump_recon);
    deblock_plane(dst->y, c->w, c->h, c->bt, 16, c->mbw, 1, 0);
    deblock_plane(dst->u, c->w / 2, c->h / 2, c->bt, 8, c->mbw, 0, 2);
    deblock_plane(dst->v, c->w / 2, c->h / 2, c->bt, 8, c->mbw, 0, 2);
    dump_pset(c, dst->y, dump_deblock);
    sao_frame(c, dst, orc_lambda(f.quality));
    if (dump_sao) memcpy(dump_sao, c->sao, (size_t)c->mbw * c->mbh * 16);
    dump_pset(c, dst->y, dump_final);
    if (f.type != F_BIDIR) memcpy(c->prev, c->bt, (size_t)c->mbw * c->mbh * sizeof(blk));   /* encode.cpp:988-998 */
    return 0;
}
