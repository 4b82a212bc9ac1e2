// evxg_decode.cu -- the decoder's pixel half on the GPU: engine_decode_frame
// (src/video/decode.cpp:560-612) after unserialize_slice.  For one frame
// whose block table, SAO table and quantised levels are given:
//   decode_slice_wpp (decode.cpp:466-556; per-MB decode_block, :31-432),
//   deblock_image_filter, sao_filter_image (the encoder's filter kernels,
//   evxg_filters.cu), and the YUV -> RGB24 conversion (convert.cpp:162-223).
//
// Macroblock reconstruction runs in two launches.  Inter macroblocks read
// only other DPB slots, so k_dec_inter decodes all of them at once, one warp
// per macroblock.  Intra macroblocks read the frame being decoded -- the
// directional predictors their left / top neighbours, the intra block copy a
// block up to 49 rows above and 50 columns right of the macroblock, plus the
// 6-tap overshoot -- so k_dec_intra walks the rows as a wavefront, row r
// trailing row r-1 by four macroblocks like decode.cpp:509-521, one CTA per
// row.  The reference's sequential order (decode.cpp:434-462) defines what
// those reads see: macroblocks earlier in raster order are decoded, later
// ones still hold the slot's previous frame; the block copy search admits
// blocks reaching below the current row (motion.cpp:361-365), so its 6-tap
// reads can touch raster-later macroblocks, which k_dec_inter may already
// have rewritten.  Such samples come from a copy of the slot taken before
// the frame (DecArgs::snap).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "evxg_internal.cuh"

namespace evxg {

namespace {

__constant__ int16_t d_lut8[64] = {  // xftables.h:57-67 (cos table x128)
    128, 128, 128, 128, 128, 128, 128, 128, 126, 106, 71, 25, -25, -71, -106, -126,
    118, 49, -49, -118, -118, -49, 49, 118, 106, -25, -126, -71, 71, 126, 25, -106,
    91, -91, -91, 91, 91, -91, -91, 91, 71, -126, 25, 106, -106, -25, 126, -71,
    49, -118, 118, -49, -49, 118, -118, 49, 25, -71, 106, -126, 126, -106, 71, -25};
__constant__ int16_t d_qm[2][64] = {
    {8, 10, 12, 15, 19, 23, 25, 27, 10, 12, 14, 17, 21, 25, 27, 28, 12, 14, 18, 21, 24, 26, 28, 30,   // intra, quantize.cpp:14-24
     15, 17, 21, 24, 26, 28, 30, 32, 19, 21, 24, 26, 28, 30, 32, 35, 23, 25, 26, 28, 30, 32, 35, 38,
     25, 27, 28, 30, 32, 35, 38, 41, 27, 28, 30, 32, 35, 38, 41, 45},
    {16, 17, 18, 19, 20, 21, 22, 23, 17, 18, 19, 20, 21, 22, 23, 24, 18, 19, 20, 21, 22, 23, 24, 25,  // inter, quantize.cpp:26-36
     19, 20, 21, 22, 23, 24, 26, 27, 20, 21, 22, 23, 25, 26, 27, 28, 21, 22, 23, 24, 26, 27, 28, 30,
     22, 23, 24, 26, 27, 28, 30, 31, 23, 24, 25, 27, 28, 30, 31, 33}};

constexpr int MB_N = 384;            // 16x16 luma + 2 x 8x8 chroma; MB buffers are Y | U | V
constexpr int INTER_WARPS = 8;       // k_dec_inter: warps per CTA, one macroblock each
constexpr int INTRA_THREADS = 256;   // k_dec_intra: one CTA per macroblock row
// Block-copy source staged in shared memory by k_dec_intra: the 16x16 luma
// block with the 6-tap margin (-3 .. +18) and the two 8x8 chroma blocks with
// theirs (-3 .. +10).
constexpr int WIN_L = 22, WIN_C = 14, WIN_N = WIN_L * WIN_L + 2 * WIN_C * WIN_C;

// Kernel parameters of one decoded frame.
struct DecArgs {
    int W, H, mbw, mbh;
    int type, dest;                  // frame type, destination slot
    int b_frames, R, index;          // build; without B frames the slots follow from the index
    int16_t *planes[4];
    const int16_t *snap;             // the destination slot as it was before this frame
    const int16_t *lev;              // quantised levels, plane-set layout
    const evxg_block_desc *bt;
    int *progress, *counters, *error;
    long long timeout_ns;
};

struct PlaneView {                   // one plane of a plane set
    const int16_t *p;
    int w, h;                        // size = row stride
};
__device__ __forceinline__ PlaneView plane_of(const int16_t *set, int W, int H, int pl)
{
    const size_t ny = (size_t)W * H, nc = (size_t)(W / 2) * (H / 2);
    return pl == 0 ? PlaneView{set, W, H} : PlaneView{set + ny + (pl - 1) * nc, W / 2, H / 2};
}
// Sample e of an MB buffer: plane, row, column.
__device__ __forceinline__ void mb_pos(int e, int &pl, int &r, int &c)
{
    if (e < 256) { pl = 0; r = e >> 4; c = e & 15; }
    else { pl = 1 + ((e - 256) >> 6); const int k = (e - 256) & 63; r = k >> 3; c = k & 7; }
}

__device__ __forceinline__ void dir_of_frac(int f, int &dx, int &dy)   // motion.cpp:93-116
{
    if (f <= 2) { dy = -1; dx = f - 1; }
    else if (f == 3) { dx = -1; dy = 0; }
    else if (f == 4) { dx = 1; dy = 0; }
    else { dy = 1; dx = f - 6; }
}

// Reads of a reference plane: any slot but the destination, clamped to the
// plane like interp.cpp:8-14.
struct RefReader {
    PlaneView v;
    __device__ __forceinline__ int operator()(int x, int y) const
    {
        x = max(0, min(x, v.w - 1)); y = max(0, min(y, v.h - 1));
        return __ldg(v.p + (size_t)y * v.w + x);
    }
};
// Reads of the frame being decoded by macroblock m: samples of macroblocks
// before m in raster order from the slot, the others from its copy.
struct CurReader {
    PlaneView v, old;
    int sh, mbw, m;                  // sh: log2 of the MB size in this plane
    __device__ __forceinline__ int operator()(int x, int y) const
    {
        x = max(0, min(x, v.w - 1)); y = max(0, min(y, v.h - 1));
        const size_t k = (size_t)y * v.w + x;
        return (y >> sh) * mbw + (x >> sh) < m ? __ldcg(v.p + k) : __ldg(old.p + k);
    }
};

// Reads of a staged window whose cell (i, j) holds the sample the frame
// reader gives at (x0 + j, y0 + i); every read of a prediction stays inside.
struct WinReader {
    const int16_t *p;
    int n, x0, y0;
    __device__ __forceinline__ int operator()(int x, int y) const { return p[(y - y0) * n + (x - x0)]; }
};

// One predicted sample at (c, r) of an n x n block whose integer position is
// (bx, by), optionally at the half / quarter position in direction (dx, dy)
// (interp.cpp:52-164: horizontal, vertical, or horizontal rows rounded to
// int16 and then vertical; quarter = (full + half + 1) >> 1).
template <class Rd>
__device__ __forceinline__ int16_t mc_sample(const Rd &rd, int bx, int by, int r, int c, bool sp, int dx, int dy,
                                             bool quarter)
{
    const int fx = bx + c, fy = by + r;
    if (!sp) return (int16_t)rd(fx, fy);
    int half;
    if (dx && !dy) {
        const int x = fx + (dx > 0 ? 0 : -1);
        half = tap6(rd(x - 2, fy), rd(x - 1, fy), rd(x, fy), rd(x + 1, fy), rd(x + 2, fy), rd(x + 3, fy));
    } else if (!dx && dy) {
        const int y = fy + (dy > 0 ? 0 : -1);
        half = tap6(rd(fx, y - 2), rd(fx, y - 1), rd(fx, y), rd(fx, y + 1), rd(fx, y + 2), rd(fx, y + 3));
    } else {
        const int x = fx + (dx > 0 ? 0 : -1), y0 = fy + (dy > 0 ? 0 : -1);
        int t[6];
#pragma unroll
        for (int k = 0; k < 6; k++) {
            const int y = y0 + k - 2;
            t[k] = tap6(rd(x - 2, y), rd(x - 1, y), rd(x, y), rd(x + 1, y), rd(x + 2, y), rd(x + 3, y));
        }
        half = tap6(t[0], t[1], t[2], t[3], t[4], t[5]);
    }
    if (!quarter) return (int16_t)half;
    return (int16_t)((rd(fx, fy) + half + 1) >> 1);
}

__device__ __forceinline__ int16_t luma_dc(int qp)   // quantize.cpp:74-83
{
    if (qp < 5) return (int16_t)max(qp << 1, 2);
    if (qp < 9) return (int16_t)(qp << 1);
    if (qp < 25) return (int16_t)(qp + 8);
    return (int16_t)((qp << 1) - 16);
}
__device__ __forceinline__ int16_t chroma_dc(int qp)   // quantize.cpp:85-92
{
    if (qp < 5) return (int16_t)max(qp << 1, 2);
    if (qp < 25) return (int16_t)((qp + 13) >> 1);
    return (int16_t)(qp - 6);
}
// inverse_quantize_macroblock, one coefficient (quantize.cpp:271-343, :399-476):
// intra matrices for intra blocks without motion, chroma at min(qp + 2, 63).
__device__ __forceinline__ int16_t dequant(int16_t lv, int qp, int o, bool intra, bool chroma)
{
    if (intra && o == 0) return (int16_t)(lv * (chroma ? chroma_dc(qp) : luma_dc(qp)));
    return (int16_t)((2 * lv * d_qm[intra ? 0 : 1][o] * qp) / 16);
}
// Output i of an inverse 8-point line with per-term truncation
// (transform.cpp:330-349); in[k] = input k.
__device__ __forceinline__ int idct_out(const int in[8], int i)
{
    int t = ((in[0] * d_lut8[i]) * 45) / 128;
#pragma unroll
    for (int k = 1; k < 8; k++) t += (in[k] * d_lut8[k * 8 + i]) / 2;
    return rdiv(t, 128);
}

// Neighbours of a directional intra prediction (intra_pred.cpp:13-54): the
// row above and the column left of the block, 128 where the frame ends.
struct Nbrs {
    int16_t top[3][16], left[3][16], corner[3], dc[3];
};
__device__ __forceinline__ int16_t intra_sample(int mode, const Nbrs &nb, int pl, int n, int x, int y)   // intra_pred.cpp:60-174
{
    auto ref = [&](int i) -> int {
        return i < n ? nb.left[pl][n - 1 - i] : (i == n ? nb.corner[pl] : nb.top[pl][i - n - 1]);
    };
    switch (mode) {
    case 0: return nb.dc[pl];
    case 1: return nb.top[pl][x];
    case 2: return nb.left[pl][y];
    case 3: {
        const int k = x + y;
        return (int16_t)((nb.top[pl][min(k, n - 1)] + 2 * nb.top[pl][min(k + 1, n - 1)] + nb.top[pl][min(k + 2, n - 1)] + 2) >> 2);
    }
    case 4: { const int d = x - y + n; return (int16_t)((ref(d - 1) + 2 * ref(d) + ref(d + 1) + 2) >> 2); }
    case 5: {
        const int d = min(max(x - (y >> 1) + n, 1), 2 * n - 1);
        return (y & 1) ? (int16_t)((ref(d - 1) + 2 * ref(d) + ref(d + 1) + 2) >> 2) : (int16_t)((ref(d) + ref(d + 1) + 1) >> 1);
    }
    case 6: {
        const int d = min(max((x >> 1) - y + n, 1), 2 * n - 1);
        return (x & 1) ? (int16_t)((ref(d - 1) + 2 * ref(d) + ref(d + 1) + 2) >> 2) : (int16_t)((ref(d) + ref(d + 1) + 1) >> 1);
    }
    default: return 128;
    }
}

__device__ __forceinline__ int blk_elem(int b, int r, int c)   // element (r, c) of 8x8 block b of an MB buffer
{
    return b < 4 ? ((b >> 1) * 8 + r) * 16 + (b & 1) * 8 + c : 256 + (b - 4) * 64 + r * 8 + c;
}
__device__ __forceinline__ void set_error(const DecArgs &a, int code) { atomicCAS(a.error, 0, code); }

// A reference slot of the descriptor's prediction (decode.cpp:196-203): the
// slot itself with B frames, else the offset from the frame index
// (query_prediction_index_by_offset, common.cpp:256-259).  -1 if invalid.
__device__ __forceinline__ int ref_slot(const DecArgs &a, int target)
{
    int s;
    if (a.b_frames) s = target;
    else s = (target >= 1 && target < a.R) ? (a.index + a.R - target) % a.R : -1;
    return (s >= 0 && s < 4 && s != a.dest) ? s : -1;
}

// decode_block (decode.cpp:31-432) of macroblock (row, col) by the nth
// threads of a group (t = thread index in it; sync() = the group's barrier):
// prediction into pred, inverse quantisation and the inverse transform in
// buf (2 x 384 samples), the sum written into the destination slot.
template <int NTH, bool STAGE, class Sync>
__device__ void decode_mb(const DecArgs &a, int row, int col, int t, int16_t *pred, int16_t *buf, Nbrs &nb,
                          int16_t *win, Sync sync)
{
    const int m = row * a.mbw + col, px = col * 16, py = row * 16;
    const evxg_block_desc d = a.bt[m];
    const int bt = d.block_type;
    const bool intra = bt & 1, motion = bt & 2, copy = bt & 4;
    if (bt > 7 || bt == 5) { if (t == 0) set_error(a, EVXG_ERROR_INVALID_RESOURCE); return; }   // decode.cpp:429
    // this thread's levels, loaded now so that they arrive while the prediction is built
    constexpr int PER = (MB_N + NTH - 1) / NTH;
    int16_t lv[PER];
    if (!copy) {
#pragma unroll
        for (int k = 0; k < PER; k++) {
            const int e = t + k * NTH;
            if (e < MB_N) {
                int pl, r, c;
                mb_pos(e, pl, r, c);
                const size_t ny = (size_t)a.W * a.H, nc = (size_t)(a.W / 2) * (a.H / 2);
                lv[k] = __ldg(pl == 0 ? a.lev + (size_t)(py + r) * a.W + px + c
                                      : a.lev + ny + (pl - 1) * nc + (size_t)((py >> 1) + r) * (a.W / 2) + (px >> 1) + c);
            }
        }
    }
    bool has_pred = true;
    if (bt == 1) {   // intra default: directional prediction, or none
        has_pred = d.intra_mode != 7;
        if (has_pred) {
            for (int k = t; k < 3 * 33; k += NTH) {   // per plane: n top, n left, corner
                const int pl = k / 33, j = k % 33, n = pl ? 8 : 16;
                if (j > 2 * n) continue;
                const PlaneView v = plane_of(a.planes[a.dest], a.W, a.H, pl);
                const int cx = pl ? px >> 1 : px, cy = pl ? py >> 1 : py;
                const bool ht = cy > 0, hl = cx > 0;
                if (j < n) nb.top[pl][j] = ht ? __ldcg(v.p + (size_t)(cy - 1) * v.w + cx + j) : (int16_t)128;
                else if (j < 2 * n) nb.left[pl][j - n] = hl ? __ldcg(v.p + (size_t)(cy + j - n) * v.w + cx - 1) : (int16_t)128;
                else nb.corner[pl] = ht && hl ? __ldcg(v.p + (size_t)(cy - 1) * v.w + cx - 1) : (int16_t)-1;
            }
            sync();
            if (t < 3) {
                const int n = t ? 8 : 16, cx = t ? px >> 1 : px, cy = t ? py >> 1 : py;
                const bool ht = cy > 0, hl = cx > 0;
                int sum = 0, cnt = 0;
                if (ht) { for (int i = 0; i < n; i++) sum += nb.top[t][i]; cnt += n; }
                if (hl) { for (int i = 0; i < n; i++) sum += nb.left[t][i]; cnt += n; }
                nb.dc[t] = cnt > 0 ? (int16_t)((sum + cnt / 2) / cnt) : (int16_t)128;
                if (!(ht && hl)) nb.corner[t] = ht ? nb.top[t][0] : (hl ? nb.left[t][0] : (int16_t)128);
            }
            sync();
            for (int e = t; e < MB_N; e += NTH) {
                int pl, r, c;
                mb_pos(e, pl, r, c);
                pred[e] = intra_sample(d.intra_mode, nb, pl, pl ? 8 : 16, c, r);
            }
        }
    } else if (intra) {   // intra block copy from the frame itself
        int dx = 0, dy = 0;
        if (d.sp_pred) dir_of_frac(d.sp_index, dx, dy);
        const int bx = px + d.motion_x, by = py + d.motion_y;
        if constexpr (STAGE) {   // the source with its taps, once, then the prediction from shared memory
            for (int k = t; k < WIN_N; k += NTH) {
                int pl, r, c, x0, y0;
                if (k < WIN_L * WIN_L) { pl = 0; r = k / WIN_L; c = k % WIN_L; x0 = bx - 3; y0 = by - 3; }
                else {
                    const int q = k - WIN_L * WIN_L;
                    pl = 1 + q / (WIN_C * WIN_C); r = (q % (WIN_C * WIN_C)) / WIN_C; c = q % WIN_C;
                    x0 = (bx >> 1) - 3; y0 = (by >> 1) - 3;
                }
                const CurReader rd{plane_of(a.planes[a.dest], a.W, a.H, pl), plane_of(a.snap, a.W, a.H, pl),
                                   pl ? 3 : 4, a.mbw, m};
                win[k] = (int16_t)rd(x0 + c, y0 + r);
            }
            sync();
            for (int e = t; e < MB_N; e += NTH) {
                int pl, r, c;
                mb_pos(e, pl, r, c);
                const WinReader wr = pl == 0 ? WinReader{win, WIN_L, bx - 3, by - 3}
                                             : WinReader{win + WIN_L * WIN_L + (pl - 1) * WIN_C * WIN_C, WIN_C,
                                                         (bx >> 1) - 3, (by >> 1) - 3};
                pred[e] = mc_sample(wr, pl ? bx >> 1 : bx, pl ? by >> 1 : by, r, c, d.sp_pred, dx, dy, d.sp_amount);
            }
        } else {
            for (int e = t; e < MB_N; e += NTH) {
                int pl, r, c;
                mb_pos(e, pl, r, c);
                const CurReader rd{plane_of(a.planes[a.dest], a.W, a.H, pl), plane_of(a.snap, a.W, a.H, pl),
                                   pl ? 3 : 4, a.mbw, m};
                pred[e] = mc_sample(rd, pl ? bx >> 1 : bx, pl ? by >> 1 : by, r, c, d.sp_pred, dx, dy, d.sp_amount);
            }
        }
    } else if (a.type == EVXG_FRAME_BIDIR && d.prediction_mode == 2) {   // bi-prediction: (fwd + bwd + 1) >> 1
        const int sf = ref_slot(a, d.prediction_target), sb = ref_slot(a, d.prediction_target_b);
        if (sf < 0 || sb < 0) { if (t == 0) set_error(a, EVXG_ERROR_INVALID_RESOURCE); return; }
        int fdx = 0, fdy = 0, bdx = 0, bdy = 0;
        if (motion && d.sp_pred) dir_of_frac(d.sp_index, fdx, fdy);
        if (motion && d.sp_pred_b) dir_of_frac(d.sp_index_b, bdx, bdy);
        const int fx = motion ? px + d.motion_x : px, fy = motion ? py + d.motion_y : py;
        const int bx = motion ? px + d.motion_x_b : px, by = motion ? py + d.motion_y_b : py;
        for (int e = t; e < MB_N; e += NTH) {
            int pl, r, c;
            mb_pos(e, pl, r, c);
            const RefReader rf{plane_of(a.planes[sf], a.W, a.H, pl)}, rb{plane_of(a.planes[sb], a.W, a.H, pl)};
            const int f = mc_sample(rf, pl ? fx >> 1 : fx, pl ? fy >> 1 : fy, r, c, motion && d.sp_pred, fdx, fdy, d.sp_amount);
            const int b = mc_sample(rb, pl ? bx >> 1 : bx, pl ? by >> 1 : by, r, c, motion && d.sp_pred_b, bdx, bdy,
                                    d.sp_amount_b);
            pred[e] = (int16_t)((f + b + 1) >> 1);
        }
    } else {   // one reference
        const int s = ref_slot(a, d.prediction_target);
        if (s < 0) { if (t == 0) set_error(a, EVXG_ERROR_INVALID_RESOURCE); return; }
        int dx = 0, dy = 0;
        if (motion && d.sp_pred) dir_of_frac(d.sp_index, dx, dy);
        const int x0 = motion ? px + d.motion_x : px, y0 = motion ? py + d.motion_y : py;
        for (int e = t; e < MB_N; e += NTH) {
            int pl, r, c;
            mb_pos(e, pl, r, c);
            const RefReader rd{plane_of(a.planes[s], a.W, a.H, pl)};
            pred[e] = mc_sample(rd, pl ? x0 >> 1 : x0, pl ? y0 >> 1 : y0, r, c, motion && d.sp_pred, dx, dy, d.sp_amount);
        }
    }
    sync();
    int16_t *Y = a.planes[a.dest];
    auto out_at = [&](int e) -> int16_t * {   // destination sample of MB buffer element e
        int pl, r, c;
        mb_pos(e, pl, r, c);
        const size_t ny = (size_t)a.W * a.H, nc = (size_t)(a.W / 2) * (a.H / 2);
        return pl == 0 ? Y + (size_t)(py + r) * a.W + px + c
                       : Y + ny + (pl - 1) * nc + (size_t)((py >> 1) + r) * (a.W / 2) + (px >> 1) + c;
    };
    if (copy) {   // copy blocks: the prediction itself
        for (int e = t; e < MB_N; e += NTH) *out_at(e) = pred[e];
        return;
    }
    int16_t *coef = buf, *tmp = buf + MB_N;
    const bool iq = intra && !motion;   // quantize.cpp:457
    const int qy = d.q_index, qc = min(d.q_index + 2, 63);
#pragma unroll
    for (int k = 0; k < PER; k++) {   // the levels loaded at the start
        const int e = t + k * NTH;
        if (e >= MB_N) break;
        int pl, r, c;
        mb_pos(e, pl, r, c);
        const int o = (r & 7) * 8 + (c & 7);
        coef[e] = dequant(lv[k], pl ? qc : qy, o, iq, pl != 0);
    }
    sync();
    for (int q = t; q < MB_N; q += NTH) {   // columns: coef -> tmp (int16)
        const int b = q >> 6, j = (q >> 3) & 7, i = q & 7;
        int in[8];
#pragma unroll
        for (int k = 0; k < 8; k++) in[k] = coef[blk_elem(b, k, j)];
        tmp[blk_elem(b, i, j)] = (int16_t)idct_out(in, i);
    }
    sync();
    for (int q = t; q < MB_N; q += NTH) {   // rows, plus the prediction: tmp -> slot
        const int b = q >> 6, j = (q >> 3) & 7, i = q & 7;
        int in[8];
#pragma unroll
        for (int k = 0; k < 8; k++) in[k] = tmp[blk_elem(b, j, k)];
        const int e = blk_elem(b, j, i), v = idct_out(in, i);
        *out_at(e) = (int16_t)(has_pred ? v + pred[e] : v);
    }
}

// Inter macroblocks, one warp each, all at once.
__global__ void __launch_bounds__(32 * INTER_WARPS) k_dec_inter(DecArgs a)
{
    __shared__ int16_t s_pred[INTER_WARPS][MB_N];
    __shared__ int16_t s_buf[INTER_WARPS][2 * MB_N];
    __shared__ Nbrs s_nb[INTER_WARPS];   // intra only; decode_mb's signature
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nmb = a.mbw * a.mbh;
    for (int m = blockIdx.x * INTER_WARPS + w; m < nmb; m += gridDim.x * INTER_WARPS) {
        if (a.bt[m].block_type & 1) continue;
        decode_mb<32, false>(a, m / a.mbw, m % a.mbw, lane, s_pred[w], s_buf[w], s_nb[w], nullptr, [] { __syncwarp(); });
        __syncwarp();
    }
}

// Thread 0: wait until rows lo .. hi have decoded their intra macroblocks up
// to column col; false (and the error word set) when the bound ran out.
// seen[k] caches the last progress read of row hi - k (progress only grows),
// so rows already known to be far enough are not read again.
constexpr int kSeenRows = 8;
__device__ bool wait_rows(const DecArgs &a, int lo, int hi, int col, int *seen)
{
    unsigned long long t0 = 0;
    for (int r = max(lo, 0); r <= hi; r++) {
        const int k = hi - r;
        if (k < kSeenRows && seen[k] >= col) continue;
        int v;
        while ((v = ld_acquire(&a.progress[r])) < col) {
            if (!t0) t0 = globaltimer_ns();
            else if ((long long)(globaltimer_ns() - t0) > a.timeout_ns) {
                set_error(a, EVXG_ERROR_OPERATION_TIMEDOUT);
                return false;
            }
            __nanosleep(200);
        }
        if (k < kSeenRows) seen[k] = v;
    }
    return true;
}

// Rows of earlier macroblocks an intra macroblock reads, and the last column
// it reads in them: its directional neighbours, or the block it copies with
// the 6-tap taps (-3 .. +18 luma, -3 .. +10 chroma samples), clamped to the
// frame like the reads themselves.
__device__ void intra_reach(const DecArgs &a, const evxg_block_desc &d, int row, int col, int &lo, int &c_need)
{
    lo = row; c_need = -1;
    if (d.block_type == 1) {
        if (d.intra_mode != 7) { lo = row - 1; c_need = col; }
        return;
    }
    const int bx = col * 16 + d.motion_x, by = row * 16 + d.motion_y, pad = d.sp_pred ? 3 : 0;
    const int ly0 = max(by - pad, 0), lx1 = min(bx + 15 + pad, a.W - 1);
    const int cy0 = max((by >> 1) - pad, 0), cx1 = min((bx >> 1) + 7 + pad, a.W / 2 - 1);
    lo = min(ly0 >> 4, cy0 >> 3);
    c_need = min(max(max(lx1, 0) >> 4, max(cx1, 0) >> 3), a.mbw - 1);
}

// Intra macroblocks: one CTA per row, rows claimed in order.  progress[r] is
// the column up to which row r's intra macroblocks are decoded.
__global__ void __launch_bounds__(INTRA_THREADS) k_dec_intra(DecArgs a)
{
    __shared__ int16_t s_pred[MB_N];
    __shared__ int16_t s_buf[2 * MB_N];
    __shared__ Nbrs s_nb;
    __shared__ int16_t s_win[WIN_N];
    __shared__ unsigned s_mask[128];   // intra columns of the row (mbw <= 4096)
    __shared__ int s_row, s_ok;
    const int t = threadIdx.x, words = (a.mbw + 31) >> 5;
    for (;;) {
        if (t == 0) s_row = atomicAdd(&a.counters[0], 1);
        for (int k = t; k < words; k += INTRA_THREADS) s_mask[k] = 0;
        __syncthreads();
        const int row = s_row;
        if (row >= a.mbh) return;
        for (int c = t; c < a.mbw; c += INTRA_THREADS)
            if (a.bt[row * a.mbw + c].block_type & 1) atomicOr(&s_mask[c >> 5], 1u << (c & 31));
        __syncthreads();
        auto next_intra = [&](int c) {   // first intra column >= c, or mbw
            for (int k = c >> 5; k < words; k++) {
                const unsigned v = s_mask[k] & (k == (c >> 5) ? ~0u << (c & 31) : ~0u);
                if (v) return min(k * 32 + __ffs(v) - 1, a.mbw);
            }
            return a.mbw;
        };
        int c = next_intra(0);
        int seen[kSeenRows];   // thread 0: progress of rows row-1, row-2, ... as last read
#pragma unroll
        for (int k = 0; k < kSeenRows; k++) seen[k] = -1;
        if (t == 0) st_release(&a.progress[row], c - 1);
        while (c < a.mbw) {
            if (t == 0) {
                int lo, need;
                intra_reach(a, a.bt[row * a.mbw + c], row, c, lo, need);
                s_ok = need < 0 || lo >= row || wait_rows(a, lo, row - 1, need, seen);
            }
            __syncthreads();
            if (!s_ok) return;   // the error word is set; rows below give up in turn
            decode_mb<INTRA_THREADS, true>(a, row, c, t, s_pred, s_buf, s_nb, s_win, [] { __syncthreads(); });
            __threadfence();
            __syncthreads();
            c = next_intra(c + 1);
            if (t == 0) st_release(&a.progress[row], c - 1);
        }
        __syncthreads();   // s_row and s_mask are rewritten for the next row
    }
}

// SAO parameters each macroblock is filtered with (sao.cpp:113-120): a merged
// macroblock takes its left (else upper) neighbour's own entry -- one level,
// not followed further: the entropy decoder leaves a merged macroblock's own
// parameters cleared (unserialize.cpp:579-596).
__global__ void k_dec_sao_resolve(const evxg_sao_info *raw, evxg_sao_info *res, int mbw, int mbh)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= mbw * mbh) return;
    const int bx = m % mbw, by = m / mbw;
    const evxg_sao_info &in = raw[m];
    const evxg_sao_info &src = (in.merge_left && bx > 0) ? raw[m - 1] : ((in.merge_above && by > 0) ? raw[m - mbw] : in);
    evxg_sao_info o = in;
    o.luma = src.luma;
    o.chroma = src.chroma;
    res[m] = o;
}

// YUV 4:2:0 -> RGB24 (convert.cpp:15-18, :162-223), one thread per 2x2 pixel
// quad, cropped to the visible size.
__device__ __forceinline__ uint8_t sat8(int v) { return (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v)); }
__global__ void k_dec_rgb(const int16_t *set, int W, int H, int w, int h, uint8_t *rgb)
{
    const int qx = blockIdx.x * blockDim.x + threadIdx.x, qy = blockIdx.y;
    if (qx >= w / 2 || qy >= h / 2) return;
    const int16_t *Y = set, *U = set + (size_t)W * H, *V = U + (size_t)(W / 2) * (H / 2);
    const int u = U[(size_t)qy * (W / 2) + qx] - 128, v = V[(size_t)qy * (W / 2) + qx] - 128;
#pragma unroll
    for (int dy = 0; dy < 2; dy++)
#pragma unroll
        for (int dx = 0; dx < 2; dx++) {
            const int x = 2 * qx + dx, y = 2 * qy + dy;
            const int l = 256 * (Y[(size_t)y * W + x] - 16);
            uint8_t *o = rgb + ((size_t)y * w + x) * 3;
            o[0] = sat8((l + 358 * v + 128) >> 8);
            o[1] = sat8((l - 88 * u - 182 * v + 128) >> 8);
            o[2] = sat8((l + 452 * u + 128) >> 8);
        }
}

// The encoder's peek() maps (evx3enc.cpp:454-543), one thread per visible
// pixel, from the block of the block table it lies in.
__global__ void k_peek_map(const evxg_block_desc *bt, int mbw, int w, int h, int which, uint8_t *rgb)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= w || y >= h) return;
    const evxg_block_desc &d = bt[(x / 16) + (y / 16) * mbw];
    const int bt_ = d.block_type;
    const bool copy = bt_ & 4;
    int r = 0, g = 0, b = 0;
    switch (which) {
    case EVXG_PEEK_BLOCK_TABLE: r = 255 * (bt_ & 1); g = 255 * ((bt_ >> 1) & 1); b = 255 * ((bt_ >> 2) & 1); break;
    case EVXG_PEEK_QUANT_TABLE:
        if (copy) r = 255;
        else r = g = b = 255 - 15 * d.q_index;
        break;
    case EVXG_PEEK_BLOCK_VARIANCE:
        if (copy) r = 255;
        else r = g = b = min(max(d.variance / 30, 0), 255);
        break;
    case EVXG_PEEK_SPMP_TABLE:
        if (d.sp_pred) { g = 255 * d.sp_amount; b = 255 * !d.sp_amount; }
        break;
    default: break;
    }
    uint8_t *o = rgb + ((size_t)y * w + x) * 3;
    o[0] = (uint8_t)r; o[1] = (uint8_t)g; o[2] = (uint8_t)b;
}

}  // namespace

int peek_rgb(const int16_t *planes, const evxg_block_desc *bt, int which, int W, int H, int mbw, int w, int h,
             uint8_t *out, cudaStream_t st)
{
    if (which == EVXG_PEEK_SOURCE || which == EVXG_PEEK_DESTINATION) {
        const int cw = std::min(w, W), ch = std::min(h, H);
        k_dec_rgb<<<dim3((cw / 2 + 127) / 128, ch / 2), 128, 0, st>>>(planes, W, H, w, h, out);
    } else {
        k_peek_map<<<dim3((w + 127) / 128, h), 128, 0, st>>>(bt, mbw, w, h, which, out);
    }
    CK(cudaGetLastError());
    return EVXG_SUCCESS;
}
}  // namespace evxg

using namespace evxg;

struct evxg_decoder {
    uint32_t vw, vh, W, H, mbw, mbh;
    size_t plane_elems;
    evxg_config cfg;
    int16_t *dpb[4], *lev, *snap, *sao_orig;
    evxg_block_desc *bt;
    evxg_sao_info *sao, *sao_res;      // as decoded / each macroblock's parameters with merges resolved
    int *sao_flags, *sync;
    uint8_t *rgb;
    int num_sms;
    long long timeout_ns;
    cudaStream_t aux;                  // deblocking beside the intra wavefront
    cudaEvent_t ev_aux[2];             // inter pass done / deblocking done
    // Entropy-decoded state of the host side (evx_context of the reference's
    // decoder): the tables persist from frame to frame, since a slice
    // rewrites only the fields it codes.
    std::vector<evxg_block_desc> hbt, hprev;
    std::vector<evxg_sao_info> hsao;
    std::vector<int16_t> hlev;
    uint32_t next_index;
};

static int decoder_zero(evxg_decoder *d, cudaStream_t st)   // every plane and table zero, like a new context
{
    const size_t pb = d->plane_elems * sizeof(int16_t), nblk = (size_t)d->mbw * d->mbh;
    for (int i = 0; i < 4; i++) CK(cudaMemsetAsync(d->dpb[i], 0, pb, st));
    CK(cudaMemsetAsync(d->lev, 0, pb, st));
    CK(cudaMemsetAsync(d->bt, 0, nblk * sizeof(evxg_block_desc), st));
    CK(cudaMemsetAsync(d->sao, 0, nblk * sizeof(evxg_sao_info), st));
    CK(cudaMemsetAsync(d->sync, 0, (3 * d->mbh + 5) * sizeof(int), st));
    return EVXG_SUCCESS;
}

extern "C" {

int evxg_decoder_create(uint32_t width, uint32_t height, const evxg_config *cfg, evxg_decoder **out)
{
    if (!out || !width || !height || width > 65535 || height > 65535 || (width & 1) || (height & 1))
        return fail(EVXG_ERROR_INVALIDARG, "evxg_decoder_create: width/height must be even and in 2..65534");
    *out = nullptr;
    evxg_config c;
    evxg_config_default(&c);
    if (cfg) {
        const int rc = check_config(cfg, "evxg_decoder_create");
        if (rc) return rc;
        c = *cfg;
    }
    evxg_decoder *d = new (std::nothrow) evxg_decoder();
    if (!d) return fail(EVXG_ERROR_OUTOFMEMORY, "evxg_decoder_create: host allocation");
    d->cfg = c;
    d->vw = width; d->vh = height;
    d->W = (width + 15) & ~15u; d->H = (height + 15) & ~15u;
    d->mbw = d->W / 16; d->mbh = d->H / 16;
    d->plane_elems = (size_t)d->W * d->H + 2 * (size_t)(d->W / 2) * (d->H / 2);
    d->timeout_ns = 5000000000LL;
    const size_t pb = d->plane_elems * sizeof(int16_t), nblk = (size_t)d->mbw * d->mbh;
    try {
        d->hbt.assign(nblk, evxg_block_desc{});
        d->hprev.assign(nblk, evxg_block_desc{});
        d->hsao.assign(nblk, evxg_sao_info{});
        d->hlev.assign(d->plane_elems, 0);
    } catch (const std::bad_alloc &) {
        delete d;
        return fail(EVXG_ERROR_OUTOFMEMORY, "evxg_decoder_create: host allocation");
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&d->num_sms, cudaDevAttrMultiProcessorCount, dev);
    for (int i = 0; i < 4 && e == cudaSuccess; i++) e = cudaMalloc(&d->dpb[i], pb);
    if (e == cudaSuccess) e = cudaMalloc(&d->lev, pb);
    if (e == cudaSuccess) e = cudaMalloc(&d->snap, pb);
    if (e == cudaSuccess) e = cudaMalloc(&d->sao_orig, pb);
    if (e == cudaSuccess) e = cudaMalloc(&d->bt, nblk * sizeof(evxg_block_desc));
    if (e == cudaSuccess) e = cudaMalloc(&d->sao, nblk * sizeof(evxg_sao_info));
    if (e == cudaSuccess) e = cudaMalloc(&d->sao_res, nblk * sizeof(evxg_sao_info));
    if (e == cudaSuccess) e = cudaMalloc(&d->sao_flags, kSaoPasses * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&d->sync, (3 * d->mbh + 5) * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&d->rgb, (size_t)width * height * 3);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&d->aux, cudaStreamNonBlocking);
    for (int i = 0; i < 2 && e == cudaSuccess; i++) e = cudaEventCreateWithFlags(&d->ev_aux[i], cudaEventDisableTiming);
    cudaStream_t zs = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&zs, cudaStreamNonBlocking);
    if (e == cudaSuccess && decoder_zero(d, zs)) e = cudaErrorUnknown;
    if (e == cudaSuccess) max_active_clusters();   // the filter kernels' shared-memory limits, once per device
    if (e == cudaSuccess) e = cudaStreamSynchronize(zs);
    if (zs) cudaStreamDestroy(zs);
    if (e != cudaSuccess) {
        const int rc = cuda_fail(e, "evxg_decoder_create");
        evxg_decoder_destroy(d);
        return rc;
    }
    d->next_index = 0;
    *out = d;
    return EVXG_SUCCESS;
}

int evxg_decoder_destroy(evxg_decoder *d)
{
    if (!d) return EVXG_ERROR_INVALIDARG;
    for (int i = 0; i < 4; i++) cudaFree(d->dpb[i]);
    cudaFree(d->lev); cudaFree(d->snap); cudaFree(d->sao_orig);
    cudaFree(d->bt); cudaFree(d->sao); cudaFree(d->sao_res); cudaFree(d->sao_flags); cudaFree(d->sync); cudaFree(d->rgb);
    if (d->aux) { cudaStreamSynchronize(d->aux); cudaStreamDestroy(d->aux); }
    for (int i = 0; i < 2; i++)
        if (d->ev_aux[i]) cudaEventDestroy(d->ev_aux[i]);
    delete d;
    return EVXG_SUCCESS;
}

int evxg_decoder_set_timeout_ns(evxg_decoder *d, int64_t ns)
{
    if (!d || ns <= 0) return fail(EVXG_ERROR_INVALIDARG, "evxg_decoder_set_timeout_ns: null decoder or ns <= 0");
    d->timeout_ns = ns;
    return EVXG_SUCCESS;
}

int evxg_decoder_reset(evxg_decoder *d, void *cuda_stream)
{
    if (!d) return fail(EVXG_ERROR_INVALIDARG, "evxg_decoder_reset: null decoder");
    const cudaStream_t st = (cudaStream_t)cuda_stream;
    const int rc = decoder_zero(d, st);
    if (rc) return rc;
    std::fill(d->hbt.begin(), d->hbt.end(), evxg_block_desc{});
    std::fill(d->hprev.begin(), d->hprev.end(), evxg_block_desc{});
    std::fill(d->hsao.begin(), d->hsao.end(), evxg_sao_info{});
    std::fill(d->hlev.begin(), d->hlev.end(), (int16_t)0);
    d->next_index = 0;
    CK(cudaStreamSynchronize(st));
    return EVXG_SUCCESS;
}

int evxg_decoder_decode_record(evxg_decoder *d, const uint8_t *data, uint64_t len, uint8_t *rgb, evxg_frame *frame_out,
                               uint64_t *consumed, void *cuda_stream)
{
    if (!d || !data) return fail(EVXG_ERROR_INVALIDARG, "evxg_decoder_decode_record: null argument");
    // default build: u32 size, 18-byte evx_frame, slice; without B frames: 10-byte evx_frame, slice
    const bool sized = d->cfg.b_frames;
    const uint64_t fbytes = sized ? 18 : 10, head = sized ? 4 : 0;
    if (len < head + fbytes) return fail(EVXG_ERROR_INVALID_RESOURCE, "evxg_decoder_decode_record: record truncated");
    uint64_t body = len - head;
    if (sized) {
        uint32_t n = 0;
        std::memcpy(&n, data, 4);
        if (n < fbytes || n > body) return fail(EVXG_ERROR_INVALID_RESOURCE, "evxg_decoder_decode_record: bad record size");
        body = n;
    }
    evxg_frame f{};
    std::memcpy(&f, data + head, fbytes);
    if (f.index != d->next_index)   // evx3dec.cpp:86-96
        return fail(EVXG_ERROR_INVALID_RESOURCE, "evxg_decoder_decode_record: frame index out of sequence");
    uint64_t used = 0;
    int rc = evxg_unserialize_slice(&d->cfg, d->W, d->H, &f, data + head + fbytes, body - fbytes, d->hbt.data(),
                                    d->hprev.data(), d->hsao.data(), d->hlev.data(), &used);
    if (rc) return rc;
    rc = evxg_decode_frame(d, &f, d->hbt.data(), d->hsao.data(), d->hlev.data(), 0, rgb, 0, cuda_stream);
    if (!rc) rc = evxg_decoder_sync(d, cuda_stream);
    if (rc) return rc;
    if (!(d->cfg.b_frames && f.type == EVXG_FRAME_BIDIR)) d->hprev = d->hbt;   // decode.cpp:601-609
    d->next_index++;
    if (frame_out) *frame_out = f;
    if (consumed) *consumed = sized ? head + body : fbytes + used;
    return EVXG_SUCCESS;
}

int evxg_decode_frame(evxg_decoder *d, const evxg_frame *fin, const evxg_block_desc *blocks, const evxg_sao_info *sao,
                      const int16_t *levels, int tables_on_device, uint8_t *rgb, int rgb_on_device, void *cuda_stream)
{
    if (!d || !fin || !blocks || !sao || !levels) return fail(EVXG_ERROR_INVALIDARG, "evxg_decode_frame: null argument");
    evxg_frame f;
    int rc = check_frame_config(d->cfg, fin, "evxg_decode_frame", &f);
    if (rc) return rc;
    const cudaStream_t st = (cudaStream_t)cuda_stream;
    const size_t pb = d->plane_elems * sizeof(int16_t), nblk = (size_t)d->mbw * d->mbh;
    const cudaMemcpyKind in = tables_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    CK(cudaMemcpyAsync(d->bt, blocks, nblk * sizeof(evxg_block_desc), in, st));
    CK(cudaMemcpyAsync(d->sao, sao, nblk * sizeof(evxg_sao_info), in, st));
    CK(cudaMemcpyAsync(d->lev, levels, pb, in, st));
    CK(cudaMemsetAsync(d->sync, 0xFF, 3 * d->mbh * sizeof(int), st));
    CK(cudaMemsetAsync(d->sync + 3 * d->mbh, 0, 4 * sizeof(int), st));
    // An I/P frame has no intra macroblocks more often than not; a host table shows it.
    bool any_intra = true;
    if (!tables_on_device) {
        any_intra = false;
        for (size_t i = 0; i < nblk && !any_intra; i++) any_intra = blocks[i].block_type & 1;
    }
    const int dest = f.dpb_slot;
    if (any_intra) CK(cudaMemcpyAsync(d->snap, d->dpb[dest], pb, cudaMemcpyDeviceToDevice, st));

    DecArgs a{};
    a.W = (int)d->W; a.H = (int)d->H; a.mbw = (int)d->mbw; a.mbh = (int)d->mbh;
    a.type = f.type; a.dest = dest;
    a.b_frames = d->cfg.b_frames; a.R = d->cfg.ref_count; a.index = (int)f.index;
    for (int i = 0; i < 4; i++) a.planes[i] = d->dpb[i];
    a.snap = d->snap; a.lev = d->lev; a.bt = d->bt;
    a.progress = d->sync; a.counters = d->sync + 3 * d->mbh; a.error = d->sync + 3 * d->mbh + 4;
    a.timeout_ns = d->timeout_ns;
    if (f.type != EVXG_FRAME_INTRA) {
        const unsigned blocks_needed = (unsigned)((nblk + INTER_WARPS - 1) / INTER_WARPS);
        k_dec_inter<<<std::min<unsigned>(blocks_needed, (unsigned)d->num_sms * 8), 32 * INTER_WARPS, 0, st>>>(a);
    }
    // With an intra wavefront, deblocking trails it on a stream of its own (a
    // row is final once its progress word reaches the last column) and writes
    // the deblocked frame to the SAO pristine copy: the wavefront still reads
    // the slot's unfiltered reconstruction.
    const bool overlap = any_intra && d->aux && deblock_shared_bytes((int)d->W) > 0;
    if (overlap) CK(cudaEventRecord(d->ev_aux[0], st));   // the inter macroblocks are in the slot
    if (any_intra) k_dec_intra<<<std::min<unsigned>(d->mbh, (unsigned)d->num_sms * 4), INTRA_THREADS, 0, st>>>(a);

    FrameArgs fa{};   // the encoder's in-loop filters on the decoded slot
    fa.W = a.W; fa.H = a.H; fa.mbw = a.mbw; fa.mbh = a.mbh; fa.vis_w = (int)d->vw; fa.vis_h = (int)d->vh;
    fa.type = f.type; fa.quality = f.quality; fa.dpb = dest;
    for (int i = 0; i < 4; i++) fa.planes[i] = d->dpb[i];
    fa.lev = d->lev; fa.bt = d->bt; fa.sao = d->sao_res; fa.sao_orig = d->sao_orig; fa.sao_flags = d->sao_flags;
    fa.progress = a.progress; fa.counters = a.counters; fa.error = a.error; fa.timeout_ns = d->timeout_ns;
    fa.active = 1; fa.plane_elems = d->plane_elems;
    if (overlap) {
        FrameArgs da = fa;
        da.db_out = d->sao_orig;
        da.db_wait = 1;
        CK(cudaStreamWaitEvent(d->aux, d->ev_aux[0], 0));
        k_deblock<<<kDeblockCtas, kDeblockThreads, deblock_shared_bytes((int)d->W), d->aux>>>(da);
        CK(cudaEventRecord(d->ev_aux[1], d->aux));
    }
    k_dec_sao_resolve<<<(unsigned)((nblk + 255) / 256), 256, 0, st>>>(d->sao, d->sao_res, a.mbw, a.mbh);
    if (overlap) {
        CK(cudaStreamWaitEvent(st, d->ev_aux[1], 0));
        CK(cudaMemcpyAsync(d->dpb[dest], d->sao_orig, pb, cudaMemcpyDeviceToDevice, st));
    } else {
        k_deblock<<<kDeblockCtas, kDeblockThreads, deblock_shared_bytes((int)d->W), st>>>(fa);
        CK(cudaMemcpyAsync(d->sao_orig, d->dpb[dest], pb, cudaMemcpyDeviceToDevice, st));
    }
    CK(cudaMemsetAsync(d->sao_flags, 0, kSaoPasses * sizeof(int), st));
    for (int p = 0; p < kSaoPasses; p++) k_sao_fix<<<d->num_sms * 8, 256, 0, st>>>(fa, p);
    k_sao_restore<<<d->num_sms * 4, 256, 0, st>>>(fa, kSaoPasses - 1);
    k_sao_apply<<<(d->mbh + 7) / 8, 256, 0, st>>>(fa, kSaoPasses - 1);
    if (rgb) {
        uint8_t *dst = rgb_on_device ? rgb : d->rgb;
        const int w = (int)std::min(d->vw, d->W), h = (int)std::min(d->vh, d->H);
        k_dec_rgb<<<dim3((w / 2 + 127) / 128, h / 2), 128, 0, st>>>(d->dpb[dest], a.W, a.H, w, h, dst);
        if (!rgb_on_device) CK(cudaMemcpyAsync(rgb, d->rgb, (size_t)d->vw * d->vh * 3, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaGetLastError());
    return EVXG_SUCCESS;
}

int evxg_decoder_sync(evxg_decoder *d, void *cuda_stream)
{
    if (!d) return fail(EVXG_ERROR_INVALIDARG, "evxg_decoder_sync: null decoder");
    CK(cudaStreamSynchronize((cudaStream_t)cuda_stream));
    int err = 0;
    CK(cudaMemcpy(&err, d->sync + 3 * d->mbh + 4, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) {
        CK(cudaMemset(d->sync + 3 * d->mbh + 4, 0, sizeof(int)));
        return fail(err, err == EVXG_ERROR_OPERATION_TIMEDOUT ? "evxg_decoder_sync: device wavefront gave up waiting (timeout)"
                                                              : "evxg_decoder_sync: invalid block descriptor in the frame");
    }
    return EVXG_SUCCESS;
}

int evxg_decoder_fetch_planes(evxg_decoder *d, uint32_t slot, int16_t *out, int to_device, void *cuda_stream)
{
    if (!d || !out || slot > 3) return fail(EVXG_ERROR_INVALIDARG, "evxg_decoder_fetch_planes: null argument or slot > 3");
    const cudaStream_t st = (cudaStream_t)cuda_stream;
    CK(cudaMemcpyAsync(out, d->dpb[slot], d->plane_elems * sizeof(int16_t),
                       to_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
    if (!to_device) CK(cudaStreamSynchronize(st));
    return EVXG_SUCCESS;
}

}  // extern "C"

// ------------------------------------------------------------- whole streams

// The reference's evx3_decoder_impl (evx3dec.cpp:12-260) over the decoder
// above: the stream header on the first call, then one frame record per
// decode(); with B frames a display buffer of B-frame-count + 2 = 5 frames,
// of which each decode() and flush() hands out at most the next one in
// display order (evx3dec.cpp:137-185, :219-241).
struct evxg_stream_decoder {
    evxg_config cfg;
    evxg_decoder *dec = nullptr;
    uint32_t width = 0, height = 0;
    struct Held {
        std::vector<uint8_t> rgb;
        uint32_t display_order = 0;
        bool valid = false;
    };
    std::vector<Held> held;   // the display buffer
    uint32_t next_display = 0;
    std::vector<uint8_t> frame;
};

static constexpr uint32_t kDisplaySlots = 5;   // EVX_B_FRAME_COUNT + 2

// Hands out the next frame in display order if the buffer has it.
static bool emit_next(evxg_stream_decoder *sd, uint8_t *rgb)
{
    for (auto &h : sd->held)
        if (h.valid && h.display_order == sd->next_display) {
            if (rgb) std::memcpy(rgb, h.rgb.data(), h.rgb.size());
            h.valid = false;
            sd->next_display++;
            return true;
        }
    return false;
}

extern "C" {

int evxg_stream_decoder_create(const evxg_config *cfg, evxg_stream_decoder **out)
{
    if (!out) return fail(EVXG_ERROR_INVALIDARG, "evxg_stream_decoder_create: null argument");
    *out = nullptr;
    evxg_config c;
    evxg_config_default(&c);
    if (cfg) {
        const int rc = check_config(cfg, "evxg_stream_decoder_create");
        if (rc) return rc;
        c = *cfg;
    }
    evxg_stream_decoder *sd = new (std::nothrow) evxg_stream_decoder();
    if (!sd) return fail(EVXG_ERROR_OUTOFMEMORY, "evxg_stream_decoder_create: host allocation");
    sd->cfg = c;
    *out = sd;
    return EVXG_SUCCESS;
}

int evxg_stream_decoder_destroy(evxg_stream_decoder *sd)
{
    if (!sd) return EVXG_ERROR_INVALIDARG;
    if (sd->dec) evxg_decoder_destroy(sd->dec);
    delete sd;
    return EVXG_SUCCESS;
}

int evxg_stream_decoder_clear(evxg_stream_decoder *sd)   // evx3dec.cpp:25-48
{
    if (!sd) return fail(EVXG_ERROR_INVALIDARG, "evxg_stream_decoder_clear: null decoder");
    if (sd->dec) evxg_decoder_destroy(sd->dec);
    sd->dec = nullptr;
    sd->width = sd->height = 0;
    sd->held.clear();
    sd->next_display = 0;
    return EVXG_SUCCESS;
}

int evxg_stream_decoder_dims(const evxg_stream_decoder *sd, uint32_t *width, uint32_t *height)
{
    if (!sd || !sd->dec) return fail(EVXG_ERROR_NOT_READY, "evxg_stream_decoder_dims: no header read yet");
    if (width) *width = sd->width;
    if (height) *height = sd->height;
    return EVXG_SUCCESS;
}

int evxg_stream_decoder_decode(evxg_stream_decoder *sd, const uint8_t *data, uint64_t len, uint64_t *consumed,
                               uint8_t *rgb, int *has_output)
{
    if (!sd || !data || !consumed) return fail(EVXG_ERROR_INVALIDARG, "evxg_stream_decoder_decode: null argument");
    *consumed = 0;
    if (has_output) *has_output = 0;
    uint64_t used = 0;
    if (!sd->dec) {   // evx3dec.cpp:50-79: the header, then the context for its size
        if (len < 14 || std::memcmp(data, "EVX1", 4) != 0)
            return fail(EVXG_ERROR_INVALID_RESOURCE, "evxg_stream_decoder_decode: no stream header");
        const uint32_t w = data[10] | (data[11] << 8), h = data[12] | (data[13] << 8);
        const int rc = evxg_decoder_create(w, h, &sd->cfg, &sd->dec);
        if (rc) return rc;
        sd->width = w;
        sd->height = h;
        used = 14;
    }
    const size_t fb = (size_t)sd->width * sd->height * 3;
    sd->frame.resize(fb);
    evxg_frame f{};
    uint64_t rec = 0;
    const int rc = evxg_decoder_decode_record(sd->dec, data + used, len - used, sd->frame.data(), &f, &rec, nullptr);
    if (rc) return rc;
    *consumed = used + rec;
    if (!sd->cfg.b_frames) {   // no reorder: every frame is output as decoded
        if (rgb) std::memcpy(rgb, sd->frame.data(), fb);
        if (has_output) *has_output = 1;
        return EVXG_SUCCESS;
    }
    size_t slot = sd->held.size();
    for (size_t s = 0; s < sd->held.size(); s++)
        if (!sd->held[s].valid) { slot = s; break; }
    if (slot >= kDisplaySlots) return fail(EVXG_ERROR_EXECUTION_FAILURE, "evxg_stream_decoder_decode: display buffer full");
    if (slot == sd->held.size()) sd->held.emplace_back();
    sd->held[slot].rgb.swap(sd->frame);
    sd->held[slot].display_order = f.display_order;
    sd->held[slot].valid = true;
    const bool out = emit_next(sd, rgb);
    if (has_output) *has_output = out;
    return EVXG_SUCCESS;
}

int evxg_stream_decoder_flush(evxg_stream_decoder *sd, uint8_t *rgb, int *has_output)
{
    if (!sd || !has_output) return fail(EVXG_ERROR_INVALIDARG, "evxg_stream_decoder_flush: null argument");
    *has_output = sd->cfg.b_frames ? emit_next(sd, rgb) : 0;
    return EVXG_SUCCESS;
}

}  // extern "C"
