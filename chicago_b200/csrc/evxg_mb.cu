// evxg_mb.cu -- the macroblock wavefront kernel: per-MB mode decision, encode
// and reconstruction of one EVX3 frame on sm_100a.
//
// Reference: src/video/encode.cpp:168-941 (classify_block, classify_block_bidir,
// encode_block, encode_slice_wpp), src/video/motion.cpp:120-840 (searches),
// src/video/decode.cpp:31-432 (decode_block), src/video/intra_pred.cpp,
// src/video/transform.cpp, src/video/quantize.cpp, src/video/interp.cpp.
//
// Schedule.  A persistent grid of CTAs claims macroblock rows in order from an
// atomic counter; a CTA processes its row left to right and starts MB (r,c)
// once row r-1 has finished column min(c+2, cols-1) (the reference's WPP waits
// for c+4, encode.cpp:866-877).  MB (r,c) reads the destination slot at columns
// c-3 .. c+3; the reads of column c+3 above row r (half-pel planes around a
// selection at the right edge of the search range) wait for row r-1 to finish
// c+3 first, and MB (r,c) writes back only after MB (r-1, c+3), whose reads
// reach its stale pixels, has finished.  Every MB therefore sees exactly the
// reconstruction the sequential raster encoder sees -- all raster-earlier MBs
// it reads are finished and no raster-later MB it reads has been written -- so
// the stale pixels the intra block-copy search and the 6-tap overshoot read in
// the destination DPB slot are the same.  Waits are bounded by a timeout that
// sets the device error word.
//
// Inside an MB, three groups of four warps run the independent work at the
// same time: the intra block-copy search, the forward (P: the nearest
// reference's) inter search, and the backward search (B), the second
// reference's search (P frames of an I/P stream with several references) or
// the intra RDO candidates (P).  In a
// search step every warp evaluates candidates of the 3x3 pattern (16 lanes do
// 4x4 luma Hadamard/SAD/MAD, 16 lanes chroma MAD) and the group leader
// replays the reference's order-dependent acceptance rule; sub-pel refinement
// runs one warp per direction (half and quarter from one 6-tap pass); DCT,
// quantisation, dequantisation and IDCT run thread-per-line and the trellis
// warp-per-block over shared memory.
#include "evxg_device.cuh"

namespace evxg {

__constant__ int16_t c_lut8[64] = {  // xftables.h:57-67 (cos table x128)
    128, 128, 128, 128, 128, 128, 128, 128, 126, 106, 71, 25, -25, -71, -106, -126,
    118, 49, -49, -118, -118, -49, 49, 118, 106, -25, -126, -71, 71, 126, 25, -106,
    91, -91, -91, 91, 91, -91, -91, 91, 71, -126, 25, 106, -106, -25, 126, -71,
    49, -118, 118, -49, -49, 118, -118, 49, 25, -71, 106, -126, 126, -106, 71, -25};
__constant__ int16_t c_qm_intra[64] = {  // quantize.cpp:14-24
    8, 10, 12, 15, 19, 23, 25, 27, 10, 12, 14, 17, 21, 25, 27, 28, 12, 14, 18, 21, 24, 26, 28, 30,
    15, 17, 21, 24, 26, 28, 30, 32, 19, 21, 24, 26, 28, 30, 32, 35, 23, 25, 26, 28, 30, 32, 35, 38,
    25, 27, 28, 30, 32, 35, 38, 41, 27, 28, 30, 32, 35, 38, 41, 45};
__constant__ int16_t c_qm_inter[64] = {  // quantize.cpp:26-36
    16, 17, 18, 19, 20, 21, 22, 23, 17, 18, 19, 20, 21, 22, 23, 24, 18, 19, 20, 21, 22, 23, 24, 25,
    19, 20, 21, 22, 23, 24, 26, 27, 20, 21, 22, 23, 25, 26, 27, 28, 21, 22, 23, 24, 26, 27, 28, 30,
    22, 23, 24, 26, 27, 28, 30, 31, 23, 24, 25, 27, 28, 30, 31, 33};
__constant__ uint8_t c_dz_intra[64] = {  // quantize.cpp:42-52
    0, 1, 1, 1, 1, 1, 2, 2, 1, 1, 1, 1, 1, 2, 2, 2, 1, 1, 1, 1, 2, 2, 2, 2, 1, 1, 1, 2, 2, 2, 2, 3,
    1, 1, 2, 2, 2, 2, 3, 3, 1, 2, 2, 2, 2, 3, 3, 3, 2, 2, 2, 2, 3, 3, 3, 3, 2, 2, 2, 3, 3, 3, 3, 3};
__constant__ uint8_t c_dz_inter[64] = {  // quantize.cpp:61-71
    2, 2, 2, 3, 3, 3, 4, 4, 2, 2, 3, 3, 3, 4, 4, 4, 2, 3, 3, 3, 4, 4, 4, 4, 3, 3, 3, 4, 4, 4, 4, 4,
    3, 3, 4, 4, 4, 4, 4, 4, 3, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4};
__constant__ uint8_t c_zigzag[64] = {  // scan.h:60-70
    0, 1, 8, 16, 9, 2, 3, 10, 17, 24, 32, 25, 18, 11, 4, 5, 12, 19, 26, 33, 40, 48, 41, 34,
    27, 20, 13, 6, 7, 14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
    58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

// Per-CTA shared copies of the tables indexed by coefficient position (a
// different position per thread), filled once at kernel start: divergent
// __constant__ reads would serialise.
__shared__ int16_t s_qm[2][64];      // 0 intra, 1 inter
__shared__ uint8_t s_dz[2][64];
__shared__ uint8_t s_scan[3][64];    // 0 zigzag, 1 row-first (vertical modes), 2 column-first (horizontal modes)
__shared__ int16_t s_lut8[64];       // cosine table, read at a different row per thread

constexpr int NT = 384;        // threads per CTA: three groups of four warps
constexpr int NW = NT / 32;
constexpr int GT = 128;        // threads per warp group
constexpr int MB_N = 384;      // 16x16 luma + 2 x 8x8 chroma, MB buffer layout Y | U | V
constexpr int MAXC = 5;        // RDO candidates (encode.cpp:279-364)
constexpr int NWIN = 6;        // 0 intra (destination slot), 1/2 forward at MB / predictor, 3/4 backward, 5 third reference

struct alignas(16) Win {
    int16_t y[WL_ROWS * WL];
    int16_t u[WC_ROWS * WC];
    int16_t v[WC_ROWS * WC];
    int ox, oy, cox, coy;      // plane coordinates of window element (0, 0)
    const int16_t *pl;         // plane set the window holds
    int valid;                 // 0: contents undefined (start of a row)
};
// Windows requested for one MB: window wi[k] around luma (bx[k], by[k]) of
// plane set pl[k]; mode[k] is decided by load_windows.
struct WinReq {
    int n;
    int wi[5], bx[5], by[5], mode[5];
    const int16_t *pl[5];
    // window 0 only: rows [fy0, fy1) (luma) and [fcy0, fcy1) (chroma) of the
    // columns just behind the new strip are read from memory again when the
    // window shifts (they were loaded before the row above finished them)
    int fy0, fy1, fcy0, fcy1;
    int staged;                // window 0 only: its new strip is in MbShared::nstrip (prefetched)
};
struct Sel {                   // evx_motion_selection, motion.cpp:53-66
    int bx, by, sad, mad, ssd;
    float cost;
    int sp_index, sp_amount, sp_enabled;
};
struct Nbr {                   // intra_pred.cpp:13-54
    int16_t top[16], left[16];
    int16_t corner;
    int ht, hl, dc;
};
struct PredIn {                // MV predictor inputs but the left neighbour (see pred_gather)
    int has[3], mx[3], my[3];  // above, above-right / above-left, temporal
};
struct alignas(4) Desc { evxg_block_desc d; };   // 4-aligned so it can be copied as 7 words

// State of one motion search, owned by one warp group.
// Half-pel planes around a selection (luma 16x16 + two 8x8 chroma blocks):
// HH = horizontal 6-tap at column centres x-1 .. x+15 for rows y-3 .. y+18,
// VV = vertical 6-tap at row centres y-1 .. y+15, DD = vertical 6-tap over HH
// (the diagonal).  Every direction's half-pel block is a sub-window of one of
// them.
template <int N>
struct HalfPlanes {
    int16_t hh[(N + 6) * (N + 1)];
    int16_t vv[(N + 1) * N];
    int16_t dd[(N + 1) * (N + 1)];
};
struct Srch {
    HalfPlanes<16> hy;
    HalfPlanes<8> hu, hv;
    int m_sad[2][9], m_mad[2][9], valid[8];   // pattern slot metrics, by step parity; sub-pel validity
    float m_cost[2][9];        // RD cost of each pattern slot
    int spm[8][4];
    Sel sel;
    int cur;                   // window the search runs in
    Desc out;
    int out_sad;
};

// Cluster form (three CTAs per macroblock row): what ranks 1 and 2 hand the
// leader for one MB, and the sequence flags the CTAs exchange.  Every field
// of Mail is written by exactly one other CTA of the cluster.
struct alignas(16) Inbox {
    // forward (P: nearest reference), backward (P: second reference), third
    // reference (P), best directional prediction
    int16_t f_pred[MB_N], b_pred[MB_N], x_pred[MB_N], d_pred[MB_N];
    Desc f_out, b_out, x_out, cd[4];
    int f_sad, b_sad, x_sad, dir_best, dir_sad, modes[3];
    float cost[4];             // P: RD costs of the intra candidates cd[0..3]
};
struct Mail {
    Inbox in[2];               // leader: results for MB n in in[n & 1] (the ranks write MB n+1's while it reads MB n's)
    Desc left;                 // ranks 1, 2: the leader's final descriptor of the previous MB
    int row_val;               // ranks 1, 2: row of the latest assignment (-1: no rows left)
    int row_seq;               // ranks 1, 2: number of row assignments made
    int dec_seq;               // ranks 1, 2: MBs whose descriptor the leader has published
    int wr_seq;                // rank 2: MBs the leader has written back to the slot
    int f_seq, d_seq;          // leader: MBs whose rank-1 / rank-2 results are in the inbox
    int16_t lcol[32];          // rank 2: the right column (Y 16, U 8, V 8) of the MB the leader wrote back last
};

struct MbShared {
    int16_t src[MB_N];
    Win win[NWIN];
    int16_t pred[7][MB_N];     // 0 intra-BC, 1 inter/fwd, 2 bwd, 3 bi, 4..6 directional candidates
    const int16_t *predp[7];   // where prediction k is (pred[k], or the cluster leader's inbox)
    Nbr nb[3];
    Srch srch[3];              // 0 intra block copy, 1 forward / P inter, 2 backward
    int thr, row_abort;
    int has_pred, sep, qx, qy;
    PredIn pin;                // cluster ranks 1, 2: predictor inputs gathered before the left neighbour is known
    int w0_early;              // cluster leader: window 0 shifts before the wavefront wait
    int modes[3], dsad[3], dir_best, dir_sad;
    int bi_sad, part[NW], dpart[3][NW];
    Desc rout[3];              // P: each reference's search result (nearest first), its SAD and prediction index
    int rsad[3], rpred[3];
    unsigned aq[MAXC][4][3];   // adaptive QP: per candidate and luma block, sum / sum of squares / count
    int cpred[MAXC], win_k, need_encode, chosen, rdo;
    WinReq req;
    Desc cd[MAXC];             // 0 intra (no prediction), 1..3 directional modes, 4 SAD winner / final
    float cost[MAXC];
    int16_t coef[MAXC][MB_N], lev[MAXC][MB_N], rec[MAXC][MB_N], tmp[MAXC][MB_N];
    Mail mail;
    // cluster leader: the next MB's source and window 0's new strip, copied
    // in asynchronously during the current MB (prefetch_next)
    alignas(16) int16_t nsrc[MB_N];
    uint4 nstrip[2 * WL_ROWS + 2 * WC_ROWS];   // luma rows x 2 chunks, then U and V rows x 1 chunk
    int pf_px, pf_py, pf_strip;
};

extern __shared__ __align__(16) unsigned char g_smem[];
__device__ __forceinline__ MbShared &SM() { return *reinterpret_cast<MbShared *>(g_smem); }

// A warp group: named barrier id, first thread, thread count.  Group 0 is the
// whole CTA (barrier 0 = __syncthreads).
struct Grp {
    int bar, t0, nt;
};
__device__ __forceinline__ void gsync(const Grp &g) { asm volatile("bar.sync %0, %1;" ::"r"(g.bar), "r"(g.nt) : "memory"); }
constexpr Grp G_ALL{0, 0, NT};
__device__ __forceinline__ Grp group(int k) { return Grp{1 + k, k * GT, GT}; }

// ---------------------------------------------------------------- helpers

__device__ __forceinline__ int blk_base(int b) { return b < 4 ? (b >> 1) * 128 + (b & 1) * 8 : 256 + (b - 4) * 64; }
__device__ __forceinline__ int blk_stride(int b) { return b < 4 ? 16 : 8; }
__device__ __forceinline__ int mb_index(int b, int r, int c)   // element (r,c) of 8x8 block b of an MB buffer
{
    return b < 4 ? (((b >> 1) * 8 + r) * 16 + (b & 1) * 8 + c) : (256 + (b - 4) * 64 + r * 8 + c);
}
__device__ __forceinline__ void clear_desc(evxg_block_desc &d)   // common.cpp:76-94
{
    d = evxg_block_desc{};
    d.block_type = INTRA_DEFAULT;
    d.intra_mode = MODE_NONE;
}
__device__ __forceinline__ void dir_from_frac(int f, int &dx, int &dy)   // motion.cpp:93-116
{
    if (f <= 2) { dy = -1; dx = f - 1; }
    else if (f == 3) { dx = -1; dy = 0; }
    else if (f == 4) { dx = 1; dy = 0; }
    else { dy = 1; dx = f - 6; }
}
__device__ __forceinline__ int frac_from_dir(int i, int j)   // motion.cpp:68-91
{
    i++; j++;
    if (j == 0) return i;
    if (j == 1) return i == 0 ? 3 : 4;
    return i + 5;
}

// 16-byte chunk loads from L2.
__device__ __forceinline__ uint4 ld16(const int16_t *p) { return __ldcg(reinterpret_cast<const uint4 *>(p)); }
__device__ __forceinline__ uint4 edge16(const int16_t *p)   // one sample repeated over a chunk
{
    const unsigned v = (unsigned short)__ldcg(p);
    const unsigned w2 = v | (v << 16);
    return make_uint4(w2, w2, w2, w2);
}
// Window origin for a luma position: 8-aligned columns (16-byte chunks).
__device__ __forceinline__ int win_ox(int bx) { return ((bx - WL_OFF) >> 3) << 3; }
__device__ __forceinline__ int win_cox(int bx) { return (((bx >> 1) - WC_OFF) >> 3) << 3; }

// One 16-byte chunk of window row r (luma: plane row by-WL_OFF+r, columns
// x0 .. x0+7; chroma likewise), rows clamped to the plane and columns outside
// it filled with the edge sample -- the clamping of interp.cpp:8-14.  Loads go
// to L2 (the slot being reconstructed is written by other SMs during the
// kernel; a window chunk is read once per MB, so L1 would not help the others).
__device__ __forceinline__ uint4 win_chunk(const int16_t *plane, int S, int rows, int y, int x0)
{
    const int16_t *row = plane + (size_t)min(max(y, 0), rows - 1) * S;
    if (x0 >= 0 && x0 + 8 <= S) return ld16(row + x0);
    return edge16(row + (x0 < 0 ? 0 : S - 1));
}

// Fill the requested windows (S.req, built by thread 0).  A window whose
// plane set and origin are unchanged is kept; one that moved right by one
// macroblock (16 luma / 8 chroma columns, same rows) -- the next MB of a row
// -- is shifted in shared memory and only its new strip is read from memory,
// one thread per window row; every other window is loaded whole, every thread
// issuing up to 4 chunk loads before storing them.  A shifted window holds
// what a fresh load would: reference slots do not change during a frame, and
// for the slot being reconstructed the caller patches each finished MB into
// window 0, while no other MB writes the retained columns before this MB
// (rows above finished them before the previous MB began; rows below trail
// by more than the window's reach).
__device__ __noinline__ void load_windows(int W, int H)
{
    MbShared &S = SM();
    WinReq &q = S.req;
    constexpr int NLC = WL / 8, NL = WL_ROWS * NLC, NCC = WC / 8, NCH = 2 * WC_ROWS * NCC, PER = NL + NCH;
    const int cw = W / 2, ch = H / 2;
    if (threadIdx.x < q.n) {
        const int k = threadIdx.x;
        Win &w = S.win[q.wi[k]];
        const int ox = win_ox(q.bx[k]), oy = q.by[k] - WL_OFF, cox = win_cox(q.bx[k]), coy = (q.by[k] >> 1) - WC_OFF;
        int mode = 0;   // 0 full load, 1 keep, 2 shift by one MB
        if (w.valid && w.pl == q.pl[k] && w.oy == oy && w.coy == coy) {
            if (w.ox == ox && w.cox == cox) mode = 1;
            else if (w.ox + 16 == ox && w.cox + 8 == cox) mode = 2;
        }
        q.mode[k] = mode;
        w.ox = ox; w.oy = oy; w.cox = cox; w.coy = coy; w.pl = q.pl[k]; w.valid = 1;
    }
    __syncthreads();
    int full[5], nf = 0, shift[5], ns = 0;
    for (int k = 0; k < q.n; k++) {
        if (q.mode[k] == 0) full[nf++] = k;
        else if (q.mode[k] == 2) shift[ns++] = k;
    }
    const int total = nf * PER;
    constexpr int B = 4;
    for (int base = 0; base < total; base += B * NT) {
        uint4 v[B];
#pragma unroll
        for (int i = 0; i < B; i++) {
            const int e = base + threadIdx.x + i * NT;
            if (e < total) {
                const int k = full[e / PER], c = e % PER;
                const Win &w = S.win[q.wi[k]];
                const int16_t *Y = q.pl[k], *U = Y + (size_t)W * H, *V = U + (size_t)cw * ch;
                if (c < NL) {
                    const int r = c / NLC, kk = c - r * NLC;
                    v[i] = win_chunk(Y, W, H, w.oy + r, w.ox + 8 * kk);
                } else {
                    const int cc = c - NL, pl = cc >= WC_ROWS * NCC, qq = cc - pl * WC_ROWS * NCC;
                    const int r = qq / NCC, kk = qq - r * NCC;
                    v[i] = win_chunk(pl ? V : U, cw, ch, w.coy + r, w.cox + 8 * kk);
                }
            }
        }
#pragma unroll
        for (int i = 0; i < B; i++) {
            const int e = base + threadIdx.x + i * NT;
            if (e < total) {
                const int k = full[e / PER], c = e % PER;
                Win &w = S.win[q.wi[k]];
                if (c < NL) {
                    const int r = c / NLC, kk = c - r * NLC;
                    *reinterpret_cast<uint4 *>(&w.y[r * WL + 8 * kk]) = v[i];
                } else {
                    const int cc = c - NL, pl = cc >= WC_ROWS * NCC, qq = cc - pl * WC_ROWS * NCC;
                    const int r = qq / NCC, kk = qq - r * NCC;
                    *reinterpret_cast<uint4 *>(&(pl ? w.v : w.u)[r * WC + 8 * kk]) = v[i];
                }
            }
        }
    }
    // Shifts: one thread per window row; the row's new chunks are requested
    // first, then the row moves left in registers.
    constexpr int RT = WL_ROWS + 2 * WC_ROWS;
    for (int e = threadIdx.x; e < ns * RT; e += NT) {
        const int k = shift[e / RT], r = e % RT;
        Win &w = S.win[q.wi[k]];
        const bool fresh = q.wi[k] == 0;
        const bool staged = fresh && q.staged;
        if (r < WL_ROWS) {
            int16_t *row = w.y + r * WL;
            const uint4 n0 = staged ? S.nstrip[2 * r] : win_chunk(q.pl[k], W, H, w.oy + r, w.ox + WL - 16);
            const uint4 n1 = staged ? S.nstrip[2 * r + 1] : win_chunk(q.pl[k], W, H, w.oy + r, w.ox + WL - 8);
            const bool again = fresh && r >= q.fy0 && r < q.fy1;
            uint4 f0, f1;
            if (again) {
                f0 = win_chunk(q.pl[k], W, H, w.oy + r, w.ox + WL - 32);
                f1 = win_chunk(q.pl[k], W, H, w.oy + r, w.ox + WL - 24);
            }
            uint4 t[NLC - 2];
#pragma unroll
            for (int j = 0; j < NLC - 2; j++) t[j] = *reinterpret_cast<const uint4 *>(row + 16 + 8 * j);
            if (again) { t[NLC - 4] = f0; t[NLC - 3] = f1; }
#pragma unroll
            for (int j = 0; j < NLC - 2; j++) *reinterpret_cast<uint4 *>(row + 8 * j) = t[j];
            *reinterpret_cast<uint4 *>(row + WL - 16) = n0;
            *reinterpret_cast<uint4 *>(row + WL - 8) = n1;
        } else {
            const int rr = r - WL_ROWS, pl = rr >= WC_ROWS, cr = rr - pl * WC_ROWS;
            const int16_t *U = q.pl[k] + (size_t)W * H, *V = U + (size_t)cw * ch;
            int16_t *row = (pl ? w.v : w.u) + cr * WC;
            const uint4 n0 = staged ? S.nstrip[2 * WL_ROWS + rr] : win_chunk(pl ? V : U, cw, ch, w.coy + cr, w.cox + WC - 8);
            const bool again = fresh && cr >= q.fcy0 && cr < q.fcy1;
            uint4 f0;
            if (again) f0 = win_chunk(pl ? V : U, cw, ch, w.coy + cr, w.cox + WC - 16);
            uint4 t[NCC - 1];
#pragma unroll
            for (int j = 0; j < NCC - 1; j++) t[j] = *reinterpret_cast<const uint4 *>(row + 8 + 8 * j);
            if (again) t[NCC - 2] = f0;
#pragma unroll
            for (int j = 0; j < NCC - 1; j++) *reinterpret_cast<uint4 *>(row + 8 * j) = t[j];
            *reinterpret_cast<uint4 *>(row + WC - 8) = n0;
        }
    }
}

// Rows of window 0 (loaded around (px, py-16)) that show MB row r-1 of the
// destination slot: window rows [y0, y1) luma and [cy0, cy1) chroma.  For
// r = 1 the rows clamped to plane row 0 (above the frame) show it too.
__device__ __forceinline__ void rows_above(int py, int &y0, int &y1, int &cy0, int &cy1)
{
    y0 = y1 = cy0 = cy1 = 0;
    if (py < 16) return;
    y1 = WL_OFF + 16; cy1 = WC_OFF + 8;                          // plane rows py-16 .. py-1
    y0 = py == 16 ? 0 : WL_OFF; cy0 = py == 16 ? 0 : WC_OFF;
}
// Read a 16-column strip of window 0 (luma columns lc.., chroma cc..) again
// for rows [y0, y1) / [cy0, cy1); threads of group g.
__device__ void refresh_strip(const Grp g, Win &w, const int16_t *plane, int W, int H, int y0, int y1, int cy0, int cy1,
                              int lc, int cc)
{
    const int gt = threadIdx.x - g.t0, cw = W / 2, ch = H / 2;
    const int16_t *U = plane + (size_t)W * H, *V = U + (size_t)cw * ch;
    const int nl = (y1 - y0) * 2, nc = (cy1 - cy0) * 2;
    for (int e = gt; e < nl + nc; e += g.nt) {
        if (e < nl) {
            const int r = y0 + e / 2, j = e % 2;
            *reinterpret_cast<uint4 *>(w.y + r * WL + lc + 8 * j) = win_chunk(plane, W, H, w.oy + r, w.ox + lc + 8 * j);
        } else {
            const int f = e - nl, p = f & 1, r = cy0 + f / 2;
            *reinterpret_cast<uint4 *>((p ? w.v : w.u) + r * WC + cc) = win_chunk(p ? V : U, cw, ch, w.coy + r, w.cox + cc);
        }
    }
}
// refresh_strip for luma columns lc.. / chroma cc.. with asynchronous copies
// (the caller commits and waits); false, copying nothing, when the strip is
// not inside the plane (edge-filled chunks).
__device__ bool refresh_strip_async(const Grp g, Win &w, const int16_t *plane, int W, int H, int y0, int y1, int cy0, int cy1,
                                    int lc, int cc)
{
    const int gt = threadIdx.x - g.t0, cw = W / 2, ch = H / 2;
    if (w.ox + lc < 0 || w.ox + lc + 16 > W || w.cox + cc < 0 || w.cox + cc + 8 > cw) return false;
    const int16_t *U = plane + (size_t)W * H, *V = U + (size_t)cw * ch;
    const int nl = (y1 - y0) * 2, nc = (cy1 - cy0) * 2;
    for (int e = gt; e < nl + nc; e += g.nt) {
        if (e < nl) {
            const int r = y0 + e / 2, j = e % 2;
            cp_async16(w.y + r * WL + lc + 8 * j, plane + (size_t)min(max(w.oy + r, 0), H - 1) * W + w.ox + lc + 8 * j);
        } else {
            const int f = e - nl, p = f & 1, r = cy0 + f / 2;
            cp_async16((p ? w.v : w.u) + r * WC + cc, (p ? V : U) + (size_t)min(max(w.coy + r, 0), ch - 1) * cw + w.cox + cc);
        }
    }
    return true;
}
// The newest strip (MB column c+3).
__device__ void refresh_newest(const Grp g, Win &w, const int16_t *plane, int W, int H, int y0, int y1, int cy0, int cy1)
{
    refresh_strip(g, w, plane, W, H, y0, y1, cy0, cy1, WL - 16, WC - 8);
}

// Candidate metrics (analysis.h:89-202): SAD (luma), MAD (Y, U, V) and SATD
// (luma) of the 16x16 block at plane position (x, y) against the source.  A
// warp evaluates two candidates, one per half: lane & 15 of a half owns luma
// 4x4 block lane & 15 (rows 4*(b>>2).., columns 4*(b&3)..) and chroma row
// lane & 7 of plane (lane >> 3) & 1, so every lane runs the same 16 luma and
// 8 chroma samples.  SrcLane holds that lane's source samples.
struct SrcLane {
    int y[16], c[8];
};
__device__ __forceinline__ void unpack2(unsigned w, int &lo, int &hi) { lo = (int)(int16_t)(w & 0xffffu); hi = (int)w >> 16; }
__device__ __forceinline__ SrcLane src_lane(const int16_t *src, int lane)   // src: 16-byte aligned MB buffer
{
    SrcLane o;
    const int b = lane & 15, r0 = (b >> 2) * 4, c0 = (b & 3) * 4;
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const uint2 w = *reinterpret_cast<const uint2 *>(src + (r0 + r) * 16 + c0);
        unpack2(w.x, o.y[r * 4], o.y[r * 4 + 1]);
        unpack2(w.y, o.y[r * 4 + 2], o.y[r * 4 + 3]);
    }
    const uint4 w = *reinterpret_cast<const uint4 *>(src + 256 + ((lane >> 3) & 1) * 64 + (lane & 7) * 8);
    unpack2(w.x, o.c[0], o.c[1]); unpack2(w.y, o.c[2], o.c[3]);
    unpack2(w.z, o.c[4], o.c[5]); unpack2(w.w, o.c[6], o.c[7]);
    return o;
}
// Samples x0 .. x0+3 of a 4-byte aligned row, any x0 >= 0: three words, two
// byte permutes picking the aligned pairs (the third word is read also when
// x0 is even; every window row has room for it).
__device__ __forceinline__ void ld4(const int16_t *row, int x0, int v[4])
{
    const unsigned *w = reinterpret_cast<const unsigned *>(row) + (x0 >> 1);
    const unsigned a = w[0], b = w[1], c = w[2], sel = (x0 & 1) ? 0x5432u : 0x3210u;
    unpack2(__byte_perm(a, b, sel), v[0], v[1]);
    unpack2(__byte_perm(b, c, sel), v[2], v[3]);
}
// This lane's share of the metrics of the candidate at (x, y) in window w.
__device__ __forceinline__ void half_metrics(const SrcLane &sl, const Win &w, int x, int y, int lane, int &sad, int &mad, int &satd)
{
    const int b = lane & 15, r0 = (b >> 2) * 4, c0 = (b & 3) * 4;
    const int lx = x - w.ox, ly = y - w.oy;
    sad = 0; mad = 0; satd = 0;
    int t[16];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        int v[4], d[4];
        ld4(w.y + (ly + r0 + r) * WL, lx + c0, v);
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int df = sl.y[r * 4 + c] - v[c], a = iabs32(df);
            sad += a;
            mad = max(mad, a);
            d[c] = (int16_t)df;   // analysis.h:97 stores the difference as int16
        }
        // hadamard_4x4 (analysis.h:44-85): the row pass, then the column pass below
        t[r * 4 + 0] = (d[0] + d[1]) + (d[2] + d[3]); t[r * 4 + 1] = (d[0] - d[1]) + (d[2] - d[3]);
        t[r * 4 + 2] = (d[0] + d[1]) - (d[2] + d[3]); t[r * 4 + 3] = (d[0] - d[1]) - (d[2] - d[3]);
    }
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int a = t[c], bb = t[4 + c], cc = t[8 + c], e = t[12 + c];
        satd += iabs32((a + bb) + (cc + e)) + iabs32((a - bb) + (cc - e)) +
                iabs32((a + bb) - (cc + e)) + iabs32((a - bb) - (cc - e));
    }
    const int cx = (x >> 1) - w.cox, cy = (y >> 1) - w.coy;
    const int16_t *pp = (((lane >> 3) & 1) ? w.v : w.u) + (cy + (lane & 7)) * WC;
    int v[8];
    ld4(pp, cx, v);
    ld4(pp, cx + 4, v + 4);
#pragma unroll
    for (int c = 0; c < 8; c++) mad = max(mad, iabs32(sl.c[c] - v[c]));
}
// Sum / max over each half of the warp (every lane gets its half's value).
__device__ __forceinline__ int half_sum(int v, int lane)
{
    const int lo = __reduce_add_sync(0xffffffffu, lane < 16 ? v : 0), hi = __reduce_add_sync(0xffffffffu, lane < 16 ? 0 : v);
    return lane < 16 ? lo : hi;
}
__device__ __forceinline__ int half_max(int v, int lane)   // v >= 0
{
    const int lo = __reduce_max_sync(0xffffffffu, lane < 16 ? v : 0), hi = __reduce_max_sync(0xffffffffu, lane < 16 ? 0 : v);
    return lane < 16 ? lo : hi;
}
// RD cost of an integer candidate: (float)satd + lambda * (|mvx| + |mvy| + 1)
// with the motion vector taken as int16 (motion.cpp:136-146).
__device__ __forceinline__ float cand_cost(int satd, int x, int y, int px, int py, float lambda)
{
    const int16_t mx = (int16_t)(x - px), my = (int16_t)(y - py);
    return rd_cost(satd, lambda, (unsigned)(iabs16(mx) + iabs16(my) + 1));
}

// Integer candidate acceptance test (motion.cpp:148-177) against selection s.
__device__ __forceinline__ bool takes_int(const Sel &s, int sad, int mad, int ssd, float cost, int thr)
{
    if (s.mad < thr) return mad < s.mad || (mad == s.mad && ssd < s.ssd);
    return (cost < s.cost || ((cost == s.cost && ssd < s.ssd) && sad < SAD_THRESHOLD)) || mad < thr;
}
// The same, applied (one thread); the candidate's cost comes from cand_cost.
__device__ __forceinline__ void accept_int(Sel &s, int x, int y, int sad, int mad, float cost, int px, int py, int thr)
{
    const int ssd = (x - px) * (x - px) + (y - py) * (y - py);
    if (takes_int(s, sad, mad, ssd, cost, thr)) { s.bx = x; s.by = y; s.sad = sad; s.ssd = ssd; s.mad = mad; s.cost = cost; }
}

// Replay of an ordered candidate list by one warp: lane k holds candidate k
// (ok = valid).  Each round every later lane tests the rule against the
// current selection and the first one that takes it becomes the selection --
// exactly the sequential loop, whose selection changes only at the
// candidates it takes -- until no lane takes it (or, with stop_on_copy, the
// selection's MAD drops below the threshold: the early exit).  take(s) is the
// lane's test, adopt(s, k) copies candidate k (from its lane) into s.
template <class Take, class Adopt>
__device__ __forceinline__ void warp_replay(Sel &s, bool ok, int lane, int thr, bool stop_on_copy, Take take, Adopt adopt)
{
    int last = -1;
    for (;;) {
        const unsigned b = __ballot_sync(0xffffffffu, ok && lane > last && take(s));
        if (!b) return;
        last = __ffs((int)b) - 1;
        adopt(s, last);
        if (stop_on_copy && s.mad < thr) return;
    }
}

// One pattern step (perform_intra/inter_motion_search, motion.cpp:348-406) on
// a warp group, from selection s: every warp evaluates two slots of the 3x3
// pattern (validity is decided identically by all lanes) into the metrics
// buffer of step parity par, then every warp replays the reference's loop
// order in registers, with its early exit, and returns the new selection --
// the same in every warp, so no second barrier is needed (a buffer is
// rewritten two steps later, after the next step's barrier).
//
// When the pattern is centred on the selection (l = t = -st) its centre slot
// is the selection itself, whose SAD, MAD and cost are already in s: every
// selection but the intra search's starting point was accepted from a
// candidate evaluation (its stored sad/mad/cost are that candidate's), and
// that starting point lies in the excluded region, so it is never valid.
// The eight remaining slots take one round of four warps.
__device__ __noinline__ Sel run_step(const Grp g, int si, int wi, bool intra, int l, int t, int st, int px, int py,
                                     int W, int H, float lambda, Sel s, int par)
{
    MbShared &S = SM();
    Srch &sr = S.srch[si];
    const int gt = threadIdx.x - g.t0, gw = gt >> 5, lane = gt & 31, nw = g.nt >> 5;
    const int bx = s.bx, by = s.by;
    const bool centred = l == -st && t == -st;
    const int n = centred ? 8 : 9;
    auto valid = [&](int x, int y) {
        return !(intra && y > py - 16 && x > px - 16) && !(x < 0 || x > W - 16 || y < 0 || y > H - 16);
    };
    if (2 * gw < n) {
        const SrcLane sl = src_lane(S.src, lane);
        for (int j0 = 2 * gw; j0 < n; j0 += 2 * nw) {
            const int j = j0 + (lane >> 4);
            const int k = centred && j >= 4 ? j + 1 : j;
            const int x = bx + l + (k % 3) * st, y = by + t + (k / 3) * st;
            const bool ok = j < n && valid(x, y);
            int sad = 0, mad = 0, satd = 0;
            if (ok) half_metrics(sl, S.win[wi], x, y, lane, sad, mad, satd);
            sad = half_sum(sad, lane); mad = half_max(mad, lane); satd = (half_sum(satd, lane) + 1) >> 1;
            if ((lane & 15) == 0 && ok) {
                sr.m_sad[par][k] = sad; sr.m_mad[par][k] = mad; sr.m_cost[par][k] = cand_cost(satd, x, y, px, py, lambda);
            }
        }
    }
    gsync(g);
    // the reference's loop order, with its early exit (every warp)
    const int k = lane < 9 ? lane : 0;
    const int x = bx + l + (k % 3) * st, y = by + t + (k / 3) * st;
    const int ssd = (x - px) * (x - px) + (y - py) * (y - py);
    bool ok;
    int sad, mad;
    float cost;
    if (centred && k == 4) {   // the selection itself; invalid only as the intra search's starting point
        ok = !(intra && y > py - 16 && x > px - 16);
        sad = s.sad; mad = s.mad; cost = s.cost;
    } else {
        ok = valid(x, y); sad = sr.m_sad[par][k]; mad = sr.m_mad[par][k]; cost = sr.m_cost[par][k];
    }
    ok = ok && lane < 9;
    warp_replay(s, ok, lane, S.thr, true,
                [&](const Sel &c) { return takes_int(c, sad, mad, ssd, cost, S.thr); },
                [&](Sel &c, int from) {
                    c.bx = __shfl_sync(0xffffffffu, x, from); c.by = __shfl_sync(0xffffffffu, y, from);
                    c.sad = __shfl_sync(0xffffffffu, sad, from); c.mad = __shfl_sync(0xffffffffu, mad, from);
                    c.ssd = __shfl_sync(0xffffffffu, ssd, from); c.cost = __shfl_sync(0xffffffffu, cost, from);
                });
    return s;
}

// Half-pel planes for one plane block (window plane pl, stride S, selection at
// window coordinates (lx, ly)), computed by the group's threads.
template <int N>
__device__ __forceinline__ void half_planes_a(HalfPlanes<N> &hp, const int16_t *pl, int S, int lx, int ly, int gt, int nt)
{
    constexpr int NH = (N + 6) * (N + 1), NV = (N + 1) * N;
    for (int e = gt; e < NH + NV; e += nt) {
        if (e < NH) {
            const int t = e / (N + 1), c = e % (N + 1);
            const int16_t *rp = pl + (ly - 3 + t) * S + lx - 1 + c;
            hp.hh[e] = tap6(rp[-2], rp[-1], rp[0], rp[1], rp[2], rp[3]);
        } else {
            const int k = e - NH, r = k / N, c = k % N;
            const int16_t *cp = pl + (ly - 1 + r) * S + lx + c;
            hp.vv[k] = tap6(cp[-2 * S], cp[-S], cp[0], cp[S], cp[2 * S], cp[3 * S]);
        }
    }
}
template <int N>
__device__ __forceinline__ void half_planes_b(HalfPlanes<N> &hp, int gt, int nt)
{
    for (int e = gt; e < (N + 1) * (N + 1); e += nt) {
        const int r = e / (N + 1), c = e % (N + 1);
        const int16_t *h = hp.hh + r * (N + 1) + c;
        hp.dd[e] = tap6(h[0], h[N + 1], h[2 * (N + 1)], h[3 * (N + 1)], h[4 * (N + 1)], h[5 * (N + 1)]);
    }
}
// Half-pel sample (r, c) of direction (dx, dy) from the planes (interp.cpp:52-164).
template <int N>
__device__ __forceinline__ int half_at(const HalfPlanes<N> &hp, int dx, int dy, int r, int c)
{
    const int cx = c + (dx > 0), ry = r + (dy > 0);
    if (dx && !dy) return hp.hh[(r + 3) * (N + 1) + cx];
    if (!dx && dy) return hp.vv[ry * N + c];
    return hp.dd[ry * (N + 1) + cx];
}

// Sub-pel refinement around selection s (motion.cpp:180-261, :408-483); the
// result goes to sr.sel (every thread of the group reads it after the final
// barrier).  The interpolation reads only the selection, which the
// refinement does not move, so the three half-pel planes are built once and
// each direction's half and quarter blocks (quarter = (full + half + 1) >> 1)
// are read from them.  One warp per direction, every lane the same share:
// luma column lane & 15, rows 8*(lane >> 4) .. +7, and chroma plane lane >> 4,
// column lane & 7, rows 4*((lane >> 3) & 1) .. +3.
__device__ __noinline__ void run_subpel(const Grp g, int si, int wi, bool intra, int px, int py, int W, int H, Sel s)
{
    MbShared &S = SM();
    Srch &sr = S.srch[si];
    const Win &w = S.win[wi];
    const int gt = threadIdx.x - g.t0, gw = gt >> 5, lane = gt & 31, nw = g.nt >> 5;
    const int bx = s.bx, by = s.by;
    const int lx = bx - w.ox, ly = by - w.oy, cx = (bx >> 1) - w.cox, cy = (by >> 1) - w.coy;
    half_planes_a<16>(sr.hy, w.y, WL, lx, ly, gt, g.nt);
    for (int p = 0; p < 2; p++) half_planes_a<8>(p ? sr.hv : sr.hu, p ? w.v : w.u, WC, cx, cy, gt, g.nt);
    gsync(g);
    half_planes_b<16>(sr.hy, gt, g.nt);
    for (int p = 0; p < 2; p++) half_planes_b<8>(p ? sr.hv : sr.hu, gt, g.nt);
    gsync(g);
    if (gw < 8) {
        const int lc = lane & 15, r0 = (lane >> 4) * 8;
        const int pl = lane >> 4, cc = lane & 7, cr0 = ((lane >> 3) & 1) * 4;
        const HalfPlanes<8> &hc = pl ? sr.hv : sr.hu;
        const int16_t *fy = w.y + (ly + r0) * WL + lx + lc, *fc = (pl ? w.v : w.u) + (cy + cr0) * WC + cx + cc;
        int sy[8], sc[4];
#pragma unroll
        for (int r = 0; r < 8; r++) sy[r] = S.src[(r0 + r) * 16 + lc];
#pragma unroll
        for (int r = 0; r < 4; r++) sc[r] = S.src[256 + pl * 64 + (cr0 + r) * 8 + cc];
        for (int k = gw; k < 8; k += nw) {
            const int r = k < 4 ? k : k + 1, i = r % 3 - 1, j = r / 3 - 1;
            const int x = bx + i, y = by + j;
            const bool ok = !(intra && y > py - 16 && x > px - 16) && !(x < 0 || x > W - 16 || y < 0 || y > H - 16);
            if (lane == 0) sr.valid[k] = ok;
            if (!ok) continue;
            // direction (i, j)'s half-pel block inside a plane (half_at)
            const int16_t *hy, *hcp;
            int ys, cs;
            if (i && !j) { hy = sr.hy.hh + 3 * 17 + (i > 0); ys = 17; hcp = hc.hh + 3 * 9 + (i > 0); cs = 9; }
            else if (!i && j) { hy = sr.hy.vv + (j > 0) * 16; ys = 16; hcp = hc.vv + (j > 0) * 8; cs = 8; }
            else { hy = sr.hy.dd + (j > 0) * 17 + (i > 0); ys = 17; hcp = hc.dd + (j > 0) * 9 + (i > 0); cs = 9; }
            hy += r0 * ys + lc; hcp += cr0 * cs + cc;
            int sh = 0, mh = 0, sq = 0, mq = 0;
#pragma unroll
            for (int rr = 0; rr < 8; rr++) {
                const int half = hy[rr * ys], full = fy[rr * WL];
                const int q = (int16_t)((full + half + 1) >> 1);
                const int ah = iabs32(sy[rr] - half), aq = iabs32(sy[rr] - q);
                sh += ah; sq += aq; mh = max(mh, ah); mq = max(mq, aq);
            }
#pragma unroll
            for (int rr = 0; rr < 4; rr++) {
                const int half = hcp[rr * cs], full = fc[rr * WC];
                const int q = (int16_t)((full + half + 1) >> 1);
                mh = max(mh, iabs32(sc[rr] - half)); mq = max(mq, iabs32(sc[rr] - q));
            }
            sh = warp_sum(sh); mh = warp_max(mh); sq = warp_sum(sq); mq = warp_max(mq);
            if (lane == 0) { sr.spm[k][0] = sh; sr.spm[k][1] = mh; sr.spm[k][2] = sq; sr.spm[k][3] = mq; }
        }
    }
    gsync(g);
    if (gw == 0) {   // 8 directions x (half, quarter), in the reference's order
        const int thr = S.thr;
        s.sp_index = 0; s.sp_amount = 0; s.sp_enabled = 0;
        const int k = (lane >> 1) & 7, q = lane & 1, r = k < 4 ? k : k + 1;
        const bool ok = lane < 16 && sr.valid[k];
        const int sad = sr.spm[k][q * 2], mad = sr.spm[k][q * 2 + 1];
        const int idx = frac_from_dir(r % 3 - 1, r / 3 - 1);
        warp_replay(s, ok, lane, thr, false,
                    [&](const Sel &c) { return c.mad < thr ? (mad < c.mad) : ((sad < c.sad && sad < SAD_THRESHOLD) || mad < thr); },
                    [&](Sel &c, int from) {
                        c.sp_enabled = 1; c.sp_amount = __shfl_sync(0xffffffffu, q, from);
                        c.sp_index = __shfl_sync(0xffffffffu, idx, from);
                        c.sad = __shfl_sync(0xffffffffu, sad, from); c.mad = __shfl_sync(0xffffffffu, mad, from);
                    });
        if (lane == 0) sr.sel = s;
    }
    gsync(g);
}

// Prediction block of search si's result into out: the integer block at (x, y)
// of window wi, or its half / quarter-pel block in direction spi, read from
// the half-pel planes run_subpel built around the same selection
// (interp.cpp:52-164; quarter = (full + half + 1) >> 1).
__device__ __noinline__ void materialize(const Grp g, int si, int wi, int x, int y, int spp, int spa, int spi, int16_t *out)
{
    MbShared &S = SM();
    const Win &w = S.win[wi];
    const Srch &sr = S.srch[si];
    const int gt = threadIdx.x - g.t0;
    const int lx = x - w.ox, ly = y - w.oy, cx = (x >> 1) - w.cox, cy = (y >> 1) - w.coy;
    int dx = 0, dy = 0;
    if (spp) dir_from_frac(spi, dx, dy);
    for (int e = gt; e < MB_N; e += g.nt) {
        int full, half = 0;
        if (e < 256) {
            const int r = e >> 4, c = e & 15;
            full = w.y[(ly + r) * WL + lx + c];
            if (spp) half = half_at<16>(sr.hy, dx, dy, r, c);
        } else {
            const int p = (e - 256) >> 6, k = (e - 256) & 63, r = k >> 3, c = k & 7;
            full = (p ? w.v : w.u)[(cy + r) * WC + cx + c];
            if (spp) half = half_at<8>(p ? sr.hv : sr.hu, dx, dy, r, c);
        }
        out[e] = !spp ? (int16_t)full : (spa ? (int16_t)((full + half + 1) >> 1) : (int16_t)half);
    }
}

__device__ void fill_desc(const Sel &s, int px, int py, bool intra, int thr, evxg_block_desc &o)   // motion.cpp:542-564
{
    clear_desc(o);
    o.block_type = intra ? BT_INTRA : 0;
    if (s.bx != px || s.by != py || s.sp_enabled) o.block_type |= BT_MOTION;
    if (s.mad < thr) o.block_type |= BT_COPY;
    o.motion_x = (int16_t)(s.bx - px);
    o.motion_y = (int16_t)(s.by - py);
    o.sp_pred = (uint8_t)s.sp_enabled;
    o.sp_amount = (uint8_t)s.sp_amount;
    o.sp_index = (uint8_t)s.sp_index;
}

// Directional intra predictor value at (x, y) of an N x N block (intra_pred.cpp:60-174).
__device__ __forceinline__ int16_t intra_px(int mode, const Nbr &nb, int n, int x, int y)
{
    auto ref = [&](int i) -> int { return i < n ? nb.left[n - 1 - i] : (i == n ? nb.corner : nb.top[i - n - 1]); };
    switch (mode) {
    case 0: return (int16_t)nb.dc;
    case 1: return nb.top[x];
    case 2: return nb.left[y];
    case 3: {
        const int k = x + y;
        return (int16_t)((nb.top[min(k, n - 1)] + 2 * nb.top[min(k + 1, n - 1)] + nb.top[min(k + 2, n - 1)] + 2) >> 2);
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

// --------------------------------------------------- transform / quantisation

__device__ __forceinline__ int16_t luma_dc_scale(int qp)   // quantize.cpp:74-83
{
    if (qp < 5) return (int16_t)max(qp << 1, 2);
    if (qp < 9) return (int16_t)(qp << 1);
    if (qp < 25) return (int16_t)(qp + 8);
    return (int16_t)((qp << 1) - 16);
}
__device__ __forceinline__ int16_t chroma_dc_scale(int qp)   // quantize.cpp:85-92
{
    if (qp < 5) return (int16_t)max(qp << 1, 2);
    if (qp < 25) return (int16_t)((qp + 13) >> 1);
    return (int16_t)(qp - 6);
}
__device__ __forceinline__ int16_t quant_coeff(int16_t sv, int qp, int o, bool intra, bool chroma)   // quantize.cpp:120-252
{
    if (intra) {
        if (o == 0) return (int16_t)rdiv(sv, chroma ? chroma_dc_scale(qp) : luma_dc_scale(qp));
        int16_t qf = (int16_t)rdiv(sv * 16, s_qm[0][o]);
        if (qp >= 16) qf = (int16_t)(qf - (int16_t)((sgn16(qf) * qp * s_dz[0][o]) >> 1));
        return (int16_t)rdiv(qf, qp << 1);
    }
    const int16_t qf = (int16_t)rdiv(sv * 16, s_qm[1][o]);
    int wgt = s_dz[1][o];
    if (qp >= 16) wgt = min(wgt + 1, 6);
    const int16_t dz = (int16_t)((sgn16(qf) * qp * wgt) >> 1);
    return (int16_t)rdiv(qf - dz, qp << 1);
}
__device__ __forceinline__ int16_t dequant_coeff(int16_t lv, int qp, int o, bool intra, bool chroma)   // quantize.cpp:271-332
{
    if (intra && o == 0) return (int16_t)(lv * (chroma ? chroma_dc_scale(qp) : luma_dc_scale(qp)));
    return (int16_t)((2 * lv * s_qm[intra ? 0 : 1][o] * qp) / 16);
}
__device__ __forceinline__ unsigned coeff_bits(int16_t lv)   // quantize.cpp:517-532
{
    if (lv == 0) return 1;
    const int a = min((int)iabs16(lv), 255);
    unsigned b = 2;
    if (a > 1) b += 1;
    if (a > 2) b += 1 + 2 * req_bits8(a - 3 + 1);
    else b += 1;
    return b;
}
__device__ __forceinline__ int scan_kind(int mode)   // scan.h:154-159
{
    return (mode == 1 || mode == 5) ? 1 : ((mode == 2 || mode == 6) ? 2 : 0);
}
// Outputs i0 .. i0+NO-1 of a forward 8-point line (transform.cpp:264-284).
template <int NO>
__device__ __forceinline__ void fdct8_part(const int in[8], int i0, int16_t out[NO])
{
#pragma unroll
    for (int q = 0; q < NO; q++) {
        const int i = i0 + q;
        int t = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) t += in[k] * s_lut8[i * 8 + k];
        t = i == 0 ? (t * 45) / 128 : t / 2;
        out[q] = (int16_t)rdiv(t, 128);
    }
}
// Outputs i0 .. i0+NO-1 of an inverse 8-point line, per-term truncation
// (transform.cpp:330-349).
template <int NO>
__device__ __forceinline__ void idct8_part(const int in[8], int i0, int out[NO])
{
#pragma unroll
    for (int q = 0; q < NO; q++) {
        const int i = i0 + q;
        int t = ((in[0] * s_lut8[i]) * 45) / 128;
#pragma unroll
        for (int k = 1; k < 8; k++) t += (in[k] * s_lut8[k * 8 + i]) / 2;
        out[q] = rdiv(t, 128);
    }
}
__device__ __forceinline__ bool intra_quant(int bt) { return (bt & BT_INTRA) && !(bt & BT_MOTION); }   // quantize.cpp:457

// Trellis of one 8x8 block (quantize.cpp:536-613) in place on an MB buffer,
// one warp: lane l owns scan positions l and l+32.  The reference's tail trim
// walks down from the last significant position zeroing levels until the
// first one worth keeping, so it zeroes every nonzero level above the highest
// "keep" position; the forward refinement decides each position on its own.
// Both become per-position RD tests plus ballots.
__device__ void trellis_warp(int16_t *lev, const int16_t *coef, int b, int qp, bool intra, int mode, float lambda,
                             int lane)
{
    const bool chroma = b >= 4;
    const uint8_t *scan = s_scan[scan_kind(mode)];
    int o[2], e[2], c[2];
    int16_t l[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        o[h] = scan[lane + 32 * h];
        e[h] = mb_index(b, o[h] >> 3, o[h] & 7);
        l[h] = lev[e[h]];
        c[h] = coef[e[h]];
    }
    auto last_sig = [&]() {
        const unsigned n0 = __ballot_sync(0xffffffffu, l[0] != 0), n1 = __ballot_sync(0xffffffffu, l[1] != 0);
        return n1 ? 63 - __clz((int)n1) : (n0 ? 31 - __clz((int)n0) : -1);
    };
    int last = last_sig();
    if (last < 0) return;
    bool keep[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int p = lane + 32 * h;
        keep[h] = false;
        if (l[h] != 0 && p >= 1 && p <= last) {
            const int dk = c[h] - (int)dequant_coeff(l[h], qp, o[h], intra, chroma), dz = c[h];
            const float ck = __fadd_rn(__int2float_rn(wmul(dk, dk)), __fmul_rn(lambda, __uint2float_rn(coeff_bits(l[h]))));
            const float cz = __fadd_rn(__int2float_rn(wmul(dz, dz)), __fmul_rn(lambda, __uint2float_rn(coeff_bits(0))));
            keep[h] = !(cz <= ck);
        }
    }
    const unsigned k0 = __ballot_sync(0xffffffffu, keep[0]), k1 = __ballot_sync(0xffffffffu, keep[1]);
    const int stop = k1 ? 63 - __clz((int)k1) : (k0 ? 31 - __clz((int)k0) : 0);
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int p = lane + 32 * h;
        if (l[h] != 0 && p > stop && p <= last) l[h] = 0;
    }
    last = last_sig();
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int p = lane + 32 * h;
        if (last >= 1 && l[h] != 0 && p >= 1 && p <= last) {
            const int16_t rl = (int16_t)(l[h] - sgn16(l[h]));
            const int dk = c[h] - (int)dequant_coeff(l[h], qp, o[h], intra, chroma);
            const int dr = c[h] - (int)dequant_coeff(rl, qp, o[h], intra, chroma);
            const float ck = __fadd_rn(__int2float_rn(wmul(dk, dk)), __fmul_rn(lambda, __uint2float_rn(coeff_bits(l[h]))));
            const float cr = __fadd_rn(__int2float_rn(wmul(dr, dr)), __fmul_rn(lambda, __uint2float_rn(coeff_bits(rl))));
            if (cr < ck) l[h] = rl;
        }
        lev[e[h]] = l[h];
    }
}

// encode_block + decode_block for candidates k0 .. k0+nc-1 on a warp group
// (encode.cpp:481-750, decode.cpp:31-432); with S.rdo set also their RD cost
// (encode.cpp:39-164).  One warp runs one 8x8 block through the whole chain
// -- forward DCT rows and columns, quantisation, trellis, dequantisation,
// inverse DCT and prediction -- synchronising only with itself, each lane
// computing two outputs of a line.  The adaptive QP needs the MB's four luma
// blocks: each block's warp leaves its partial sums, and after one barrier
// every warp combines the same four (the sums wrap modulo 2^32 like the
// reference's, so the order does not matter).
__device__ __noinline__ void encode_candidates(const Grp g, const FrameArgs &a, int k0, int nc)
{
    MbShared &S = SM();
    const int gt = threadIdx.x - g.t0, gw = gt >> 5, lane = gt & 31, nw = g.nt >> 5;
    const int l4 = lane >> 2, i0 = (lane & 3) * 2;   // line and first of two outputs
    // The chain runs once per MB and block, so its code is kept compact (one
    // loop body per transform direction): the kernel's instruction footprint,
    // not its arithmetic, bounds these phases.
    for (int j = gw; j < nc * 6; j += nw) {   // forward DCT and AQ partial sums
        const int k = k0 + j / 6, b = j % 6;
        const int bb = blk_base(b), bs = blk_stride(b);
        if (S.cd[k].d.block_type & BT_COPY) continue;
        const int16_t *pr = S.cpred[k] >= 0 ? S.predp[S.cpred[k]] : nullptr;
#pragma unroll 1
        for (int h = 0; h < 2; h++) {   // residual (int16) into coef
            const int e = bb + l4 * bs + i0 + h;
            S.coef[k][e] = (int16_t)(pr ? S.src[e] - pr[e] : S.src[e]);
        }
        __syncwarp();
        int16_t out[2];
#pragma unroll 1
        for (int pass = 0; pass < 2; pass++) {   // rows: coef -> tmp, then columns: tmp -> coef
            const int rs = pass ? 1 : bs, cs = pass ? bs : 1;
            const int16_t *X = pass ? S.tmp[k] : S.coef[k];
            int16_t *Y = pass ? S.coef[k] : S.tmp[k];
            int in[8];
#pragma unroll
            for (int t = 0; t < 8; t++) in[t] = X[bb + l4 * rs + t * cs];
            fdct8_part<2>(in, i0, out);
            Y[bb + l4 * rs + i0 * cs] = out[0];
            Y[bb + l4 * rs + (i0 + 1) * cs] = out[1];
            __syncwarp();
        }
        if (b < 4) {   // variance of the nonzero luma coefficients except the MB's first (quantize.cpp:97-118, analysis.h:251-275)
            unsigned sum = 0, sq = 0, cnt = 0;
#pragma unroll 1
            for (int h = 0; h < 2; h++) {
                const int e = bb + (i0 + h) * bs + l4;
                const int t = out[h];
                if (e != 0 && t) { sum += (unsigned)t; sq += (unsigned)wmul(t, t); cnt++; }
            }
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                sum += __shfl_xor_sync(0xffffffffu, sum, o);
                sq += __shfl_xor_sync(0xffffffffu, sq, o);
                cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
            }
            if (lane == 0) { S.aq[k][b][0] = sum; S.aq[k][b][1] = sq; S.aq[k][b][2] = cnt; }
        }
    }
    gsync(g);
    for (int j = gw; j < nc * 6; j += nw) {   // quantise, trellis, reconstruct
        const int k = k0 + j / 6, b = j % 6;
        const int bb = blk_base(b), bs = blk_stride(b);
        const int bt = S.cd[k].d.block_type;
        const int16_t *pr = S.cpred[k] >= 0 ? S.predp[S.cpred[k]] : nullptr;
        if (bt & BT_COPY) {
#pragma unroll 1
            for (int h = 0; h < 2; h++) {
                const int e = bb + l4 * bs + i0 + h;
                S.rec[k][e] = pr ? pr[e] : (int16_t)0;
            }
            continue;
        }
        unsigned sum = 0, sq = 0, cnt = 0;
#pragma unroll
        for (int q = 0; q < 4; q++) { sum += S.aq[k][q][0]; sq += S.aq[k][q][1]; cnt += S.aq[k][q][2]; }
        const int var = cnt > 0 ? (int)(sq - (unsigned)rdiv(wmul((int)sum, (int)sum), (int)cnt)) : 0;
        const int aqi = min(max(lg2u((unsigned)var) >> 1, 1), MAXQ);
        const int delta = min(max((int)((int16_t)((int16_t)aqi - (int16_t)a.quality) >> 1), -6), 6);
        const int q_index = min(max(a.quality + delta, 1), MAXQ);
        if (b == 0 && lane == 0) { S.cd[k].d.q_index = (uint8_t)q_index; S.cd[k].d.variance = (int16_t)var; }
        const bool chroma = b >= 4, iq = intra_quant(bt);
        const int qp = chroma ? min(q_index + 2, MAXQ) : q_index;
#pragma unroll 1
        for (int h = 0; h < 2; h++) {
            const int o = lane + 32 * h, e = bb + (o >> 3) * bs + (o & 7);
            S.lev[k][e] = quant_coeff(S.coef[k][e], qp, o, iq, chroma);
        }
        __syncwarp();
        trellis_warp(S.lev[k], S.coef[k], b, qp, iq, S.cd[k].d.intra_mode, a.lambda, lane);
        __syncwarp();
#pragma unroll 1
        for (int h = 0; h < 2; h++) {   // dequantised levels into coef (the trellis no longer needs it)
            const int o = lane + 32 * h, e = bb + (o >> 3) * bs + (o & 7);
            S.coef[k][e] = dequant_coeff(S.lev[k][e], qp, o, iq, chroma);
        }
        __syncwarp();
#pragma unroll 1
        for (int pass = 0; pass < 2; pass++) {   // columns: coef -> tmp, then rows + prediction: tmp -> rec
            const int rs = pass ? bs : 1, cs = pass ? 1 : bs;
            const int16_t *X = pass ? S.tmp[k] : S.coef[k];
            int16_t *Y = pass ? S.rec[k] : S.tmp[k];
            const int16_t *P = pass ? pr : nullptr;
            int in[8], out2[2];
#pragma unroll
            for (int t = 0; t < 8; t++) in[t] = X[bb + l4 * rs + t * cs];
            idct8_part<2>(in, i0, out2);
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int e = bb + l4 * rs + (i0 + h) * cs;
                Y[e] = (int16_t)(P ? out2[h] + P[e] : out2[h]);
            }
            __syncwarp();
        }
    }
    gsync(g);
    if (S.rdo)
        for (int ci = gw; ci < nc; ci += nw) {   // J = (float)SSD_y + lambda * (float)bits
            const int k = k0 + ci;
            const evxg_block_desc &d = S.cd[k].d;
            const int bt = d.block_type;
            int ssd = 0;
            for (int e = lane; e < 256; e += 32) {
                const int df = S.src[e] - S.rec[k][e];
                ssd = (int)((unsigned)ssd + (unsigned)wmul(df, df));
            }
            ssd = warp_sum(ssd);
            // Rate of the residual: the reference's quantised and reconstructed
            // blocks share one staging buffer (encode.cpp:151, :158), so the
            // estimate reads the reconstruction.
            unsigned nz = 0, cb = 0;
            if (!(bt & BT_COPY)) {
                const int b = lane >> 3, r = lane & 7;
#pragma unroll
                for (int c = 0; c < 8; c++) {
                    const int16_t v = S.rec[k][mb_index(b, r, c)];
                    if (v) {
                        nz++;
                        const int av = min((int)iabs16(v), 255);
                        cb += 2;
                        if (av > 1) cb += 1;
                        if (av > 2) cb += 1 + 2 * req_bits8(av - 3 + 1);
                        else cb += 1;
                    }
                }
#pragma unroll
                for (int o = 1; o < 8; o <<= 1) {
                    nz += __shfl_xor_sync(0xffffffffu, nz, o);
                    cb += __shfl_xor_sync(0xffffffffu, cb, o);
                }
            }
            unsigned blkbits = ((lane & 7) == 0 && !(bt & BT_COPY)) ? (unsigned)(req_bits8(nz + 1) * 2 + 1) + cb : 0;
            blkbits += __shfl_xor_sync(0xffffffffu, blkbits, 8);
            blkbits += __shfl_xor_sync(0xffffffffu, blkbits, 16);
            if (lane == 0) {   // estimate_block_bits header part (encode.cpp:39-78)
                unsigned bits = 3;
                if (!(bt & BT_INTRA)) bits += 2;
                if (bt & BT_MOTION) {
                    bits += 2 * req_bits8(iabs16(d.motion_x) + 1) + 2 * req_bits8(iabs16(d.motion_y) + 1);
                    bits += d.sp_pred ? 5 : 1;
                }
                if (!(bt & BT_COPY)) {
                    if (bt == INTRA_DEFAULT) bits += 3;
                    bits += 2 * req_bits8(iabs32(d.q_index) + 1);
                    bits += blkbits;
                }
                S.cost[k] = rd_cost(ssd, a.lambda, bits);
            }
        }
    gsync(g);
}

// ------------------------------------------------------------- searches

__device__ bool wait_progress(const FrameArgs &a, int r, int need);

// Intra block-copy search in the current frame (motion.cpp:485-565), window 0.
// With strip_pending, column c+2's rows above are still being copied into
// window 0 (the callers' older commit group): the first step does not read
// them (its candidates end at column c+1), the others wait for them.
__device__ __noinline__ void intra_bc_search(const Grp g, const FrameArgs &a, int px, int py, bool strip_pending)
{
    MbShared &S = SM();
    Srch &sr = S.srch[0];
    const int gt = threadIdx.x - g.t0;
    if (gt < 32) {   // best_sad starts at the source's own SAD (analysis.h:133-145)
        int s = 0;
        for (int e = gt; e < 256; e += 32) s += iabs16(S.src[e]);
        s = warp_sum(s);
        if (gt == 0) {
            sr.sel.bx = px; sr.sel.by = py; sr.sel.sad = s; sr.sel.mad = INT_MAX; sr.sel.ssd = INT_MAX;
            sr.sel.cost = __int2float_rn(s); sr.sel.sp_index = 0; sr.sel.sp_amount = 0; sr.sel.sp_enabled = 0;
        }
    }
    gsync(g);
    Sel s = run_step(g, 0, 0, true, -SEARCH_RADIUS, -(SEARCH_RADIUS << 1), SEARCH_RADIUS, px, py, a.W, a.H, a.lambda, sr.sel, 0);
    if (strip_pending) {
        cp_async_wait_group<1>();   // this thread's strip copies; the prefetch group may go on
        gsync(g);
    }
    if (s.mad >= S.thr) {
        int par = 1;
        for (int st = SEARCH_RADIUS >> 1; st > 0; st >>= 1, par ^= 1) {
            s = run_step(g, 0, 0, true, -st, -st, st, px, py, a.W, a.H, a.lambda, s, par);
            if (s.mad < S.thr) break;
        }
    }
    {
        // The wavefront starts MB (r, c) once row r-1 has finished column c+2.
        // The half-pel planes around a selection at x >= px+28 reach column
        // c+3 (chroma from px+28, luma from px+30); if they reach it above row
        // r, wait for row r-1 to finish c+3 and read that strip of window 0
        // again.  (Integer candidates end at px+46, inside column c+2.)  A
        // wait that gives up leaves the error word set; the frame has failed.
        const int row = py / 16, col = px / 16;
        if (row > 0 && col + 3 < a.mbw && s.bx >= px + 28 && s.by <= py + 5) {
            if (gt == 0) wait_progress(a, row - 1, col + 3);
            gsync(g);
            int y0, y1, cy0, cy1;
            rows_above(py, y0, y1, cy0, cy1);
            refresh_newest(g, S.win[0], a.planes[a.dpb], a.W, a.H, y0, y1, cy0, cy1);
            gsync(g);
        }
    }
    run_subpel(g, 0, 0, true, px, py, a.W, a.H, s);
    if (gt == 0) {
        fill_desc(sr.sel, px, py, true, S.thr, sr.out.d);
        sr.out_sad = sr.sel.sad;
    }
    gsync(g);
    if (sr.out.d.block_type & BT_MOTION)
        materialize(g, 0, 0, sr.sel.bx, sr.sel.by, sr.sel.sp_enabled, sr.sel.sp_amount, sr.sel.sp_index, S.pred[0]);
    gsync(g);
}

// MV predictor (motion.cpp:271-346) from the live block table and, for P
// frames, the previous frame's table.  Its inputs other than the left
// neighbour -- the MB above, above-right (else above-left) and the temporal
// entry -- are gathered first (pred_gather: row r-1 must have finished column
// c+1), then combined with the left neighbour (pred_combine).  left, when
// given, replaces the table entry of the left neighbour (the cluster form
// hands it over in shared memory before the leader writes the table).
__device__ void pred_gather(const FrameArgs &a, int idx, bool temporal, PredIn &o)
{
    // Every candidate entry's first three words are read at once (one round
    // trip), then the reference's order picks among them.
    const int mbw = a.mbw, bx = idx % mbw, by = idx / mbw;
    auto words = [&](const evxg_block_desc *t, int i, int4 &w) {
        const int *p = reinterpret_cast<const int *>(t + i);
        w.x = __ldcg(p); w.y = __ldcg(p + 1); w.z = __ldcg(p + 2);
    };
    int4 wt = {0, 0, 0, 0}, wr = {0, 0, 0, 0}, wl = {0, 0, 0, 0}, wp = {0, 0, 0, 0};
    if (by > 0) words(a.bt, idx - mbw, wt);
    if (by > 0 && bx + 1 < mbw) words(a.bt, idx - mbw + 1, wr);
    if (by > 0 && bx > 0) words(a.bt, idx - mbw - 1, wl);
    if (temporal) words(a.prev, idx, wp);
    // word 0 block_type; word 1 bytes 2..3 motion_x; word 2 bytes 0..1 motion_y
    static_assert(offsetof(evxg_block_desc, motion_x) == 6 && offsetof(evxg_block_desc, motion_y) == 8, "descriptor layout");
    auto take = [&](int k, const int4 &w) { o.has[k] = 1; o.mx[k] = (int16_t)(w.y >> 16); o.my[k] = (int16_t)(w.z & 0xffff); };
    o.has[0] = o.has[1] = o.has[2] = 0;
    if (by > 0 && (wt.x & BT_MOTION)) take(0, wt);
    if (by > 0 && bx + 1 < mbw && (wr.x & BT_MOTION)) take(1, wr);
    else if (by > 0 && bx > 0 && (wl.x & BT_MOTION)) take(1, wl);
    if (temporal && (wp.x & BT_MOTION)) take(2, wp);
}
__device__ void pred_combine(const FrameArgs &a, int idx, const PredIn &p, const evxg_block_desc *left, int &ox, int &oy)
{
    const int bx = idx % a.mbw;
    int mx[3], my[3], n = 0;
    if (bx > 0) {
        if (left) {
            if (left->block_type & BT_MOTION) { mx[n] = left->motion_x; my[n] = left->motion_y; n++; }
        } else if (__ldcg(&a.bt[idx - 1].block_type) & BT_MOTION) {
            mx[n] = __ldcg(&a.bt[idx - 1].motion_x); my[n] = __ldcg(&a.bt[idx - 1].motion_y); n++;
        }
    }
    for (int k = 0; k < 2; k++)
        if (p.has[k]) { mx[n] = p.mx[k]; my[n] = p.my[k]; n++; }
    if (n < 3 && p.has[2]) { mx[n] = p.mx[2]; my[n] = p.my[2]; n++; }
    if (n == 0) { ox = 0; oy = 0; }
    else if (n == 1) { ox = mx[0]; oy = my[0]; }
    else if (n == 2) { ox = (int16_t)((mx[0] + mx[1]) / 2); oy = (int16_t)((my[0] + my[1]) / 2); }
    else {
        int v[2];
        for (int k = 0; k < 2; k++) {
            int p0 = k ? my[0] : mx[0], q = k ? my[1] : mx[1], r = k ? my[2] : mx[2], t;
            if (p0 > q) { t = p0; p0 = q; q = t; }
            if (q > r) q = r;
            if (p0 > q) q = p0;
            v[k] = q;
        }
        ox = v[0]; oy = v[1];
    }
}
// One thread: the MB's search predictor (has_pred, sep, qx, qy) from its inputs.
__device__ void set_predictor(const FrameArgs &a, int idx, int px, int py, const PredIn &p, const evxg_block_desc *left)
{
    MbShared &S = SM();
    int pmx, pmy;
    pred_combine(a, idx, p, left, pmx, pmy);
    S.has_pred = (pmx || pmy);
    S.qx = min(max(px + pmx, 0), a.W - 16);
    S.qy = min(max(py + pmy, 0), a.H - 16);
    S.sep = S.has_pred && (S.qx != px || S.qy != py);
}

// The inter search's first candidates on warp 0 of g: the MB position in
// window wa (half 0, unless done) and the predictor (half 1, when pred), in
// wb when that differs.
__device__ __noinline__ void first_candidates(const Grp g, const FrameArgs &a, int si, int wa, int wb, int px, int py,
                                              bool mb, bool pred)
{
    MbShared &S = SM();
    Srch &sr = S.srch[si];
    const int gt = threadIdx.x - g.t0, gw = gt >> 5, lane = gt & 31;
    if (gw != 0) return;
    const SrcLane sl = src_lane(S.src, lane);
    const bool hp = lane >= 16, ok = hp ? pred : mb;
    int sad = 0, mad = 0, satd = 0;
    if (ok) half_metrics(sl, S.win[hp && S.sep ? wb : wa], hp ? S.qx : px, hp ? S.qy : py, lane, sad, mad, satd);
    sad = half_sum(sad, lane); mad = half_max(mad, lane); satd = (half_sum(satd, lane) + 1) >> 1;
    if (lane == 0 && ok) { sr.m_sad[0][0] = sad; sr.m_mad[0][0] = mad; sr.m_cost[0][0] = rd_cost(satd, a.lambda, 1u); }
    if (lane == 16 && ok) { sr.m_sad[0][1] = sad; sr.m_mad[0][1] = mad; sr.m_cost[0][1] = cand_cost(satd, S.qx, S.qy, px, py, a.lambda); }
}

// Inter search (motion.cpp:567-679) on one warp group: window wa holds the
// reference around the MB, wb around the predictor when that differs.  With
// first_done the MB position's metrics are in place already (first_candidates).
__device__ __noinline__ void inter_search(const Grp g, const FrameArgs &a, int si, int wa, int wb, int px, int py,
                                          int16_t *pred_out, bool first_done)
{
    MbShared &S = SM();
    Srch &sr = S.srch[si];
    const int gt = threadIdx.x - g.t0;
    first_candidates(g, a, si, wa, wb, px, py, !first_done, S.has_pred);
    gsync(g);
    if (gt == 0) {
        Sel s;
        s.bx = px; s.by = py; s.sad = sr.m_sad[0][0]; s.mad = sr.m_mad[0][0]; s.ssd = INT_MAX;
        s.cost = sr.m_cost[0][0];
        s.sp_index = 0; s.sp_amount = 0; s.sp_enabled = 0;
        if (S.has_pred) accept_int(s, S.qx, S.qy, sr.m_sad[0][1], sr.m_mad[0][1], sr.m_cost[0][1], px, py, S.thr);
        sr.sel = s;
        sr.cur = (S.sep && s.bx == S.qx && s.by == S.qy) ? wb : wa;
    }
    gsync(g);
    const int wi = sr.cur;
    Sel s = sr.sel;
    if (s.mad >= S.thr) {
        int r = SEARCH_RADIUS;   // adaptive radius, motion.cpp:640-646
        if (s.sad < SAD_THRESHOLD / 4) r = SEARCH_RADIUS / 4;
        else if (s.sad < SAD_THRESHOLD / 2) r = SEARCH_RADIUS / 2;
        int par = 0;
        for (int st = r; st > 0; st >>= 1, par ^= 1) {
            s = run_step(g, si, wi, false, -st, -st, st, px, py, a.W, a.H, a.lambda, s, par);
            if (s.mad < S.thr) break;
        }
        run_subpel(g, si, wi, false, px, py, a.W, a.H, s);
    }
    materialize(g, si, wi, sr.sel.bx, sr.sel.by, sr.sel.sp_enabled, sr.sel.sp_amount, sr.sel.sp_index, pred_out);
    if (gt == 0) {
        fill_desc(sr.sel, px, py, false, S.thr, sr.out.d);
        sr.out_sad = sr.sel.sad;
    }
    gsync(g);
}

// Directional intra: 3 predictions and the best by luma SAD (intra_pred.cpp:219-289).
__device__ __noinline__ void directional_intra(const Grp g)
{
    MbShared &S = SM();
    const int gt = threadIdx.x - g.t0, gw = gt >> 5, lane = gt & 31, nw = g.nt >> 5;
    const int m0 = S.modes[0], m1 = S.modes[1], m2 = S.modes[2];
    int s0 = 0, s1 = 0, s2 = 0;   // luma SADs, accumulated where the predictions are made
    for (int e = gt; e < MB_N; e += g.nt) {
        int16_t v0, v1, v2;
        if (e < 256) {
            const int x = e & 15, y = e >> 4;
            v0 = intra_px(m0, S.nb[0], 16, x, y); v1 = intra_px(m1, S.nb[0], 16, x, y); v2 = intra_px(m2, S.nb[0], 16, x, y);
            const int sv = S.src[e];
            s0 += iabs32(sv - v0); s1 += iabs32(sv - v1); s2 += iabs32(sv - v2);
        } else {
            const int q = e - 256, pl = q >> 6, k = q & 63;
            const Nbr &nb = S.nb[1 + pl];
            v0 = intra_px(m0, nb, 8, k & 7, k >> 3); v1 = intra_px(m1, nb, 8, k & 7, k >> 3); v2 = intra_px(m2, nb, 8, k & 7, k >> 3);
        }
        S.pred[4][e] = v0; S.pred[5][e] = v1; S.pred[6][e] = v2;
    }
    s0 = warp_sum(s0); s1 = warp_sum(s1); s2 = warp_sum(s2);
    if (lane == 0) { S.dpart[0][gw] = s0; S.dpart[1][gw] = s1; S.dpart[2][gw] = s2; }
    gsync(g);
    if (gt == 0) {
        int best = INT_MAX, bm = 0;
        for (int m = 0; m < 3; m++) {
            int t = 0;
            for (int w = 0; w < nw; w++) t += S.dpart[m][w];
            S.dsad[m] = t;
            if (t < best) { best = t; bm = m; }
        }
        S.dir_best = bm; S.dir_sad = best;
    }
    gsync(g);
}

// ------------------------------------------------------------- per-MB steps

__device__ void load_src_n(const FrameArgs &a, int px, int py, int nt)   // threads 0 .. nt-1
{
    MbShared &S = SM();
    const int16_t *srcY = a.src, *srcU = a.src + (size_t)a.W * a.H, *srcV = srcU + (size_t)(a.W / 2) * (a.H / 2);
    for (int e = threadIdx.x; e < MB_N; e += nt) {
        if (e < 256) S.src[e] = __ldg(srcY + (size_t)(py + (e >> 4)) * a.W + px + (e & 15));
        else {
            const int pl = (e - 256) >> 6, k = (e - 256) & 63;
            S.src[e] = __ldg((pl ? srcV : srcU) + (size_t)((py >> 1) + (k >> 3)) * (a.W / 2) + (px >> 1) + (k & 7));
        }
    }
}
__device__ void load_src(const FrameArgs &a, int px, int py) { load_src_n(a, px, py, NT); }   // whole CTA

// One thread: copy threshold (motion.cpp:501), RDO flag and, when searches
// follow, the MV predictor, which serves every search of the MB.  Clears the
// window request list.
__device__ __noinline__ void setup_mb(const FrameArgs &a, int idx, int px, int py, bool need_pred, const evxg_block_desc *left)
{
    MbShared &S = SM();
    S.thr = (a.quality >> 2) + 1;
    S.rdo = a.type == EVXG_FRAME_INTER;
    S.has_pred = 0; S.sep = 0; S.qx = px; S.qy = py;
    if (need_pred) {
        PredIn p;
        pred_gather(a, idx, a.type == EVXG_FRAME_INTER, p);
        set_predictor(a, idx, px, py, p, left);
    }
    S.req.n = 0;
    S.req.fy0 = S.req.fy1 = S.req.fcy0 = S.req.fcy1 = 0;
    S.req.staged = 0;
}
// Window 0's request: the slot being reconstructed around (px, py-16), with
// the rows that show MB row r-1 read again behind the new strip.
__device__ void req_window0(const FrameArgs &a, int px, int py);
__device__ void req_window(int wi, const int16_t *pl, int bx, int by)   // one thread
{
    WinReq &q = SM().req;
    q.wi[q.n] = wi; q.pl[q.n] = pl; q.bx[q.n] = bx; q.by[q.n] = by; q.n++;
}
__device__ void req_window0(const FrameArgs &a, int px, int py)   // one thread
{
    req_window(0, a.planes[a.dpb], px, py - 16);
    WinReq &q = SM().req;
    rows_above(py, q.fy0, q.fy1, q.fcy0, q.fcy1);
}

// Cluster rank 2: the directional neighbours in two parts.  nbr_top (threads
// 0..34, before the left neighbour is final): the top rows and corners from
// the destination slot.  nbr_left_modes (warp 0, ends with a CTA barrier):
// the left columns from the mail, then nbr_derive.
__device__ void nbr_top(const FrameArgs &a, int px, int py)
{
    MbShared &S = SM();
    const int tid = threadIdx.x, cw = a.W / 2, ch = a.H / 2;
    const bool ht = py > 0, hl = px > 0;
    const int16_t *D = a.planes[a.dpb];
    auto plane = [&](int p) { return p == 0 ? D : D + (size_t)a.W * a.H + (size_t)(p - 1) * cw * ch; };
    if (tid < 32) {   // luma top 0..15, U 16..23, V 24..31
        const int p = tid < 16 ? 0 : (tid < 24 ? 1 : 2), k = p ? (tid - 16) & 7 : tid;
        const int cy = p ? py >> 1 : py, cx = p ? px >> 1 : px;
        S.nb[p].top[k] = ht ? __ldcg(plane(p) + (size_t)(cy - 1) * (p ? cw : a.W) + cx + k) : (int16_t)128;
    } else if (tid < 35) {
        const int p = tid - 32, cy = p ? py >> 1 : py, cx = p ? px >> 1 : px;
        S.nb[p].corner = (ht && hl) ? __ldcg(plane(p) + (size_t)(cy - 1) * (p ? cw : a.W) + cx - 1) : (int16_t)0;
    }
}
// Warp 0 of the CTA (ends with a CTA barrier): the directional neighbours
// from top(p, k), left(p, k) and corner(p) (plane p, sample k; samples
// outside the frame are 128), the corner fallbacks, each plane's DC and the
// gradient-pruned candidate modes (intra_pred.cpp:13-54, :225-260).
template <class Top, class Left, class Corner>
__device__ void nbr_derive(int px, int py, Top top_of, Left left_of, Corner corner_of)
{
    MbShared &S = SM();
    const int tid = threadIdx.x;
    const bool ht = py > 0, hl = px > 0;
    if (tid < 32) {
        const int lane = tid, p = lane < 16 ? 0 : (lane < 24 ? 1 : 2), k = p ? (lane - 16) & 7 : lane;
        Nbr &nb = S.nb[p];
        const int top = ht ? (int)top_of(p, k) : 128, left = hl ? (int)left_of(p, k) : 128;
        nb.top[k] = (int16_t)top; nb.left[k] = (int16_t)left;
        // DC of each plane: top (if any) and left (if any) samples
        const int v = (ht ? top : 0) + (hl ? left : 0);
        const int sy = __reduce_add_sync(0xffffffffu, p == 0 ? v : 0), su = __reduce_add_sync(0xffffffffu, p == 1 ? v : 0),
                  sv = __reduce_add_sync(0xffffffffu, p == 2 ? v : 0);
        // luma gradients along the top row and the left column
        const int tprev = __shfl_up_sync(0xffffffffu, top, 1), lprev = __shfl_up_sync(0xffffffffu, left, 1);
        const bool gl = p == 0 && k >= 1;
        const int gh = __reduce_add_sync(0xffffffffu, gl && ht ? iabs32(top - tprev) : 0);
        const int gv = __reduce_add_sync(0xffffffffu, gl && hl ? iabs32(left - lprev) : 0);
        __syncwarp();
        if (lane < 3) {
            Nbr &q = S.nb[lane];
            const int nn = lane ? 8 : 16, cnt = (ht ? nn : 0) + (hl ? nn : 0), sum = lane == 0 ? sy : (lane == 1 ? su : sv);
            q.ht = ht; q.hl = hl;
            q.corner = (ht && hl) ? (int16_t)corner_of(lane) : (ht ? q.top[0] : (hl ? q.left[0] : (int16_t)128));
            q.dc = cnt > 0 ? (int16_t)((sum + cnt / 2) / cnt) : 128;
        }
        if (lane == 0) {
            S.modes[0] = 0;
            if (gv > gh * 3 / 2) { S.modes[1] = 2; S.modes[2] = 6; }
            else if (gh > gv * 3 / 2) { S.modes[1] = 1; S.modes[2] = 5; }
            else { S.modes[1] = 3; S.modes[2] = 4; }
        }
    }
    __syncthreads();
}
// Rank 2, after nbr_top and the write-back wait: left columns from the mail.
__device__ void nbr_left_modes(int px, int py)
{
    MbShared &S = SM();
    nbr_derive(px, py, [&](int p, int k) { return S.nb[p].top[k]; },
               [&](int p, int k) { return S.mail.lcol[p == 0 ? k : 8 + 8 * p + k]; }, [&](int p) { return S.nb[p].corner; });
}

// P frames: the intra RDO candidates -- intra without prediction and the
// three directional modes (encode.cpp:295-336); one thread.
__device__ void intra_candidates()
{
    MbShared &S = SM();
    clear_desc(S.cd[0].d); S.cpred[0] = -1;
    for (int m = 0; m < 3; m++) {
        clear_desc(S.cd[1 + m].d);
        S.cd[1 + m].d.intra_mode = (uint8_t)S.modes[m];
        S.cpred[1 + m] = 4 + m;
    }
}

// B frames: bi-prediction (f + b + 1) >> 1 into pred[3] and its SAD over Y,
// U and V (motion.cpp:778-813); whole CTA, ends with thread 0 holding bi_sad.
__device__ void bi_prediction()
{
    MbShared &S = SM();
    const int tid = threadIdx.x;
    int s = 0;
    for (int e = tid; e < MB_N; e += NT) {
        const int av = (S.predp[1][e] + S.predp[2][e] + 1) >> 1;
        S.pred[3][e] = (int16_t)av;
        s += iabs32(S.src[e] - av);
    }
    s = warp_sum(s);
    if ((tid & 31) == 0) S.part[tid >> 5] = s;
    __syncthreads();
    if (tid == 0) {
        int t = 0;
        for (int k = 0; k < NW; k++) t += S.part[k];
        S.bi_sad = t;
    }
}

// Candidate decision by SAD (encode.cpp:168-277, :374-470); one thread.
// Sets cd[4]/cpred[4] to the winner and need_encode, or (P frames whose winner
// is an intra candidate, already encoded) points win_k at that candidate.
__device__ __noinline__ void decide(const FrameArgs &a)
{
    MbShared &S = SM();
    evxg_block_desc best = S.srch[0].out.d;
    int bsad = S.srch[0].out_sad, bpred = (best.block_type & BT_MOTION) ? 0 : -1;
    if (a.type == EVXG_FRAME_INTER) {
        // Each reference in turn, nearest first: a copy block wins over a
        // non-copy one either way, else the smaller SAD -- without B frames
        // after a distance bias (int)(lambda * 2 * offset) on the farther
        // references, and the descriptor names the offset (encode.cpp:182-247).
        for (int k = 0; k < a.nref; k++) {
            evxg_block_desc in = S.rout[k].d;
            in.prediction_target = (uint8_t)(a.ip_mode ? k + 1 : a.ref_fwd);
            const int bias = a.ip_mode ? __float2int_rz(__fmul_rn(a.lambda, __int2float_rn(2 * (k + 1)))) : 0;
            const bool ci = in.block_type & BT_COPY, cb = best.block_type & BT_COPY;
            if (ci != cb) { if (ci) { best = in; bsad = S.rsad[k]; bpred = S.rpred[k]; } }
            else if (S.rsad[k] + bias < bsad) { best = in; bsad = S.rsad[k]; bpred = S.rpred[k]; }
        }
    } else if (a.type == EVXG_FRAME_BIDIR) {
        evxg_block_desc f = S.srch[1].out.d, b = S.srch[2].out.d;
        f.prediction_mode = 0; f.prediction_target = (uint8_t)a.ref_fwd;
        b.prediction_mode = 1; b.prediction_target = (uint8_t)a.ref_bwd;
        if (S.srch[1].out_sad < bsad) { best = f; bsad = S.srch[1].out_sad; bpred = 1; }
        if (S.srch[2].out_sad < bsad) { best = b; bsad = S.srch[2].out_sad; bpred = 2; }
        const int bias = __float2int_rz(__fmul_rn(a.lambda, 8.0f));
        if (S.bi_sad + bias < bsad) {
            evxg_block_desc bi;
            clear_desc(bi);
            bi.block_type = INTER_MOTION_DELTA; bi.prediction_mode = 2;
            bi.prediction_target = (uint8_t)a.ref_fwd;
            bi.motion_x = f.motion_x; bi.motion_y = f.motion_y;
            bi.sp_pred = f.sp_pred; bi.sp_amount = f.sp_amount; bi.sp_index = f.sp_index;
            bi.prediction_target_b = (uint8_t)a.ref_bwd;
            bi.motion_x_b = b.motion_x; bi.motion_y_b = b.motion_y;
            bi.sp_pred_b = b.sp_pred; bi.sp_amount_b = b.sp_amount; bi.sp_index_b = b.sp_index;
            best = bi; bsad = S.bi_sad; bpred = 3;
        }
    }
    int dir_k = -1;
    if (S.dir_sad < bsad) {
        clear_desc(best);
        best.intra_mode = (uint8_t)S.modes[S.dir_best];
        bsad = S.dir_sad;
        bpred = 4 + S.dir_best;
        dir_k = 1 + S.dir_best;
    }
    if (a.type == EVXG_FRAME_INTER && best.block_type == INTRA_DEFAULT) {
        // already encoded with the intra RDO candidates
        S.win_k = best.intra_mode == MODE_NONE ? 0 : dir_k;
        S.need_encode = 0;
    } else {
        S.cd[4].d = best; S.cpred[4] = bpred;
        S.win_k = 4; S.need_encode = 1;
    }
}

__device__ void rdo_choose()   // one thread: RDO order -- SAD winner, intra default, the 3 modes (encode.cpp:279-336)
{
    MbShared &S = SM();
    int ch = S.win_k;
    if (S.rdo) {
        float bc = S.cost[ch];
        if (S.cd[S.win_k].d.block_type != INTRA_DEFAULT && S.cost[0] < bc) { ch = 0; bc = S.cost[0]; }
        for (int k = 1; k <= 3; k++) if (S.cost[k] < bc) { ch = k; bc = S.cost[k]; }
    }
    S.chosen = ch;
}

// Write-back of the chosen candidate (rec / lev, possibly another CTA's shared
// memory): reconstruction into the DPB slot and window 0, levels (non-copy
// blocks), descriptor; whole CTA, ends with a fence before the progress release.
__device__ void write_back(const FrameArgs &a, int px, int py, int idx, const int16_t *rec, const int16_t *lev)
{
    MbShared &S = SM();
    const int tid = threadIdx.x;
    const int ch = S.chosen;
    const bool copy = S.cd[ch].d.block_type & BT_COPY;
    int16_t *dst = a.planes[a.dpb];
    int16_t *dU = dst + (size_t)a.W * a.H, *dV = dU + (size_t)(a.W / 2) * (a.H / 2);
    int16_t *lY = a.lev, *lU = a.lev + (size_t)a.W * a.H, *lV = lU + (size_t)(a.W / 2) * (a.H / 2);
    Win &w0 = S.win[0];   // the next MB's window 0 is this one shifted: keep it equal to the slot
    for (int e = tid; e < MB_N; e += NT) {
        const int16_t rv = rec[e];
        if (e < 256) {
            const int r = e >> 4, c = e & 15;
            const size_t o = (size_t)(py + r) * a.W + px + c;
            dst[o] = rv;
            if (!copy) lY[o] = lev[e];
            w0.y[(py + r - w0.oy) * WL + px + c - w0.ox] = rv;
        } else {
            const int pl = (e - 256) >> 6, k = (e - 256) & 63, r = k >> 3, c = k & 7;
            const size_t oc = (size_t)((py >> 1) + r) * (a.W / 2) + (px >> 1) + c;
            (pl ? dV : dU)[oc] = rv;
            if (!copy) (pl ? lV : lU)[oc] = lev[e];
            (pl ? w0.v : w0.u)[((py >> 1) + r - w0.coy) * WC + (px >> 1) + c - w0.cox] = rv;
        }
    }
    // Window rows clamped to plane row 0 or H-1 and chunks left of the plane
    // hold copies of edge pixels that the patch above does not update: after
    // an MB on the top, bottom or left edge the next MB loads window 0 afresh.
    if (tid == 0 && (px == 0 || py == 0 || py + 16 == a.H)) w0.valid = 0;
    if (tid < 7) reinterpret_cast<int *>(a.bt + idx)[tid] = reinterpret_cast<const int *>(&S.cd[ch].d)[tid];
    // the caller publishes with a release store by one thread after a CTA
    // barrier: the barrier orders every writer's stores before the release,
    // whose ordering is cumulative
}

// Thread 0: wait until row r has finished column need (the wavefront's
// progress words); false once the error word is set or the wait times out.
__device__ bool wait_progress(const FrameArgs &a, int r, int need)
{
    const unsigned long long t0 = globaltimer_ns();
    while (ld_acquire(&a.progress[r]) < need) {
        if (*(volatile int *)a.error) return false;
        if ((long long)(globaltimer_ns() - t0) > a.timeout_ns) {
            atomicCAS(a.error, 0, EVXG_ERROR_OPERATION_TIMEDOUT);
            return false;
        }
        __nanosleep(64);
    }
    return true;
}

__device__ void init_tables()
{
    const int tid = threadIdx.x;
    if (tid < 7) SM().predp[tid] = SM().pred[tid];
    if (tid < 64) {
        s_qm[0][tid] = c_qm_intra[tid]; s_qm[1][tid] = c_qm_inter[tid];
        s_dz[0][tid] = c_dz_intra[tid]; s_dz[1][tid] = c_dz_inter[tid];
        s_scan[0][tid] = c_zigzag[tid];
        s_scan[1][tid] = (uint8_t)tid;
        s_scan[2][tid] = (uint8_t)((tid & 7) * 8 + (tid >> 3));
        s_lut8[tid] = c_lut8[tid];
    }
}

// ------------------------------------------------- single-CTA form, per MB

__device__ void process_mb(const FrameArgs &a, int row, int col)
{
    MbShared &S = SM();
    const int tid = threadIdx.x;
    const int px = col * 16, py = row * 16, idx = row * a.mbw + col;

    load_src(a, px, py);
    if (tid == 0) {
        setup_mb(a, idx, px, py, a.type != EVXG_FRAME_INTRA, nullptr);
        req_window0(a, px, py);   // intra window: the slot being reconstructed
        if (a.type != EVXG_FRAME_INTRA) {
            const int16_t *r1 = a.planes[a.type == EVXG_FRAME_INTER ? a.ref_slot[0] : a.ref_fwd];
            req_window(1, r1, px, py);
            if (S.sep) req_window(2, r1, S.qx, S.qy);
        }
        if (a.type == EVXG_FRAME_BIDIR || (a.type == EVXG_FRAME_INTER && a.nref >= 2)) {
            const int16_t *r2 = a.planes[a.type == EVXG_FRAME_BIDIR ? a.ref_bwd : a.ref_slot[1]];
            req_window(3, r2, px, py);
            if (S.sep) req_window(4, r2, S.qx, S.qy);
        }
    }
    __syncthreads();
    load_windows(a.W, a.H);
    __syncthreads();
    {   // directional neighbours from window 0
        const Win &w = S.win[0];
        auto at = [&](int p, int y, int x) -> int16_t {
            return p == 0 ? w.y[(y - w.oy) * WL + x - w.ox] : (p == 1 ? w.u : w.v)[(y - w.coy) * WC + x - w.cox];
        };
        auto cy = [&](int p) { return p ? py >> 1 : py; };
        auto cx = [&](int p) { return p ? px >> 1 : px; };
        nbr_derive(px, py, [&](int p, int k) { return at(p, cy(p) - 1, cx(p) + k); },
                   [&](int p, int k) { return at(p, cy(p) + k, cx(p) - 1); }, [&](int p) { return at(p, cy(p) - 1, cx(p) - 1); });
    }

    // Independent work runs concurrently on three warp groups.  P frames
    // with several references (no B frames) search the second one where B
    // frames search backwards, and the third one afterwards on the whole CTA
    // in the first reference's windows.
    const bool multi = a.type == EVXG_FRAME_INTER && a.nref >= 2;
    const int gi = tid / GT;
    const Grp g = group(gi);
    if (gi == 0) {
        intra_bc_search(g, a, px, py, false);
        if (a.type == EVXG_FRAME_BIDIR || multi) directional_intra(g);
    } else if (gi == 1) {
        if (a.type == EVXG_FRAME_INTRA) directional_intra(g);
        else inter_search(g, a, 1, 1, 2, px, py, S.pred[1], false);
    } else {
        if (a.type == EVXG_FRAME_BIDIR || multi) {
            inter_search(g, a, 2, 3, 4, px, py, S.pred[2], false);
        } else if (a.type == EVXG_FRAME_INTER) {
            // The intra RDO candidates do not depend on the searches
            // (encode.cpp:295-336): two of them are encoded while the
            // searches run, the other two with the SAD winner afterwards
            // (candidates 2..4 on the whole CTA), which balances the groups.
            directional_intra(g);
            if (tid - g.t0 == 0) intra_candidates();
            gsync(g);
            encode_candidates(g, a, 0, 2);
        }
    }
    __syncthreads();
    if (a.type == EVXG_FRAME_INTER && tid == 0) {
        for (int k = 0; k < 2 && k < a.nref; k++) { S.rout[k] = S.srch[1 + k].out; S.rsad[k] = S.srch[1 + k].out_sad; S.rpred[k] = 1 + k; }
        if (a.nref >= 3) {   // the third reference: window 5 at the MB, window 2 again at the predictor; pred[3]
            S.req.n = 0; S.req.fy0 = S.req.fy1 = S.req.fcy0 = S.req.fcy1 = 0; S.req.staged = 0;
            req_window(5, a.planes[a.ref_slot[2]], px, py);
            if (S.sep) req_window(2, a.planes[a.ref_slot[2]], S.qx, S.qy);
        }
    }
    if (a.type == EVXG_FRAME_INTER && a.nref >= 3) {
        __syncthreads();
        load_windows(a.W, a.H);
        __syncthreads();
        inter_search(G_ALL, a, 1, 5, 2, px, py, S.pred[3], false);
        if (tid == 0) { S.rout[2] = S.srch[1].out; S.rsad[2] = S.srch[1].out_sad; S.rpred[2] = 3; }
    }
    if (a.type == EVXG_FRAME_BIDIR) bi_prediction();
    if (tid == 0) {
        if (multi) intra_candidates();
        decide(a);
    }
    __syncthreads();
    if (multi) encode_candidates(G_ALL, a, 0, S.need_encode ? 5 : 4);
    else if (a.type == EVXG_FRAME_INTER) encode_candidates(G_ALL, a, 2, S.need_encode ? 3 : 2);
    else if (S.need_encode) encode_candidates(G_ALL, a, 4, 1);
    if (tid == 0) {
        rdo_choose();
        if (row == 1) wait_progress(a, 0, min(col + 3, a.mbw - 1));   // see mb_row
    }
    __syncthreads();
    write_back(a, px, py, idx, S.rec[S.chosen], S.lev[S.chosen]);
}

// One macroblock row, left to right (single-CTA form); false once a wait
// gave up (the error word is set).
__device__ bool mb_row(const FrameArgs &a, int row)
{
    MbShared &S = SM();
    const int tid = threadIdx.x;
    for (int col = 0; col < a.mbw; ++col) {
        if (tid == 0) {
            // MB (r,c) reads the destination slot at columns c-3 .. c+3 (intra
            // block-copy candidates x in [px-31, px+31], 6-tap overshoot
            // -3..+18).  It starts once row r-1 has finished column c+2,
            // which covers every read above it but the half-pel planes that
            // reach column c+3 (intra_bc_search waits for those).  Its reads of
            // stale pixels below (rows r+1, r+2) come from window 0, whose
            // strips were read from memory when they came into view, at
            // MB (r, c-3) or earlier -- before row r+1 can have written them --
            // except in row 0, whose every MB reads its window afresh (the top
            // edge); so MBs of row 1 write back only after MB (0, c+3) has
            // finished (row 2 then follows through row 1's schedule).  Every
            // MB reads what the sequential raster encoder reads.  The
            // reference waits for c+4 (encode.cpp:866-877).
            S.row_abort = row > 0 && !wait_progress(a, row - 1, min(col + 2, a.mbw - 1));
        }
        __syncthreads();
        if (S.row_abort) return false;
        process_mb(a, row, col);
        __syncthreads();
        if (tid == 0) st_release(&a.progress[row], col);   // release: ordered after the barrier, so after every thread's stores
    }
    __syncthreads();
    return true;
}

__global__ void __launch_bounds__(NT, 1) k_mb_wavefront(FrameArgs a0)
{
    MbShared &S = SM();
    __shared__ int s_row;
    __shared__ FrameArgs a;   // the parameters in shared memory (a kernel parameter read by reference lives in local memory)
    const int tid = threadIdx.x;
    init_tables();
    if (tid == 0) a = a0;
    __syncthreads();
    for (;;) {
        if (tid == 0) s_row = atomicAdd(&a.counters[0], 1);
        if (tid < NWIN) S.win[tid].valid = 0;   // windows are reused only along a row
        __syncthreads();
        const int row = s_row;
        if (row >= a.mbh || !mb_row(a, row)) return;
    }
}

// Batched form: the rows of every stream of a tick form one queue of
// (stream, row) items, claimed in queue order; within a stream the queue keeps
// row order, so a row always waits on a row that a running CTA has claimed.
__global__ void __launch_bounds__(NT, 1) k_mb_wavefront_b(const FrameArgs *args, const int2 *queue, const int *qlen,
                                                           int *qctr)
{
    MbShared &S = SM();
    __shared__ int s_item;
    __shared__ FrameArgs sa;
    const int tid = threadIdx.x;
    init_tables();
    __syncthreads();
    const int nq = __ldg(qlen);
    for (;;) {
        if (tid == 0) s_item = atomicAdd(qctr, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= nq) return;
        const int2 q = queue[item];
        if (tid == 0) sa = args[q.x];
        if (tid < NWIN) S.win[tid].valid = 0;
        __syncthreads();
        if (!mb_row(sa, q.y)) return;   // the tick has failed; every wait of it now gives up
    }
}

// ------------------------------------------- cluster form: three CTAs per row
//
// A cluster of three CTAs encodes one macroblock row; each search gets a whole
// CTA (12 warps: a pattern step's eight candidates in one round) instead of a
// warp group.
//   rank 0, the leader: waits for the wavefront, runs the intra block-copy
//     search, takes the other ranks' results, decides, encodes the winner
//     and writes the MB back.
//   rank 1: the forward (P: the) inter search.
//   rank 2: the backward search (B frames), then directional intra; for P
//     frames also encodes the four intra RDO candidates.
// The inter searches need only the MV predictor, i.e. the descriptors of the
// left MB and of row r-1 up to column c+1, so ranks 1 and 2 start MB c as soon
// as the leader has decided MB c-1 and search while the leader still encodes
// MB c-1 and runs MB c's intra search.  Directional intra needs MB c-1's
// reconstruction and row r-1 up to column c.
//
// Hand-over is through distributed shared memory: peers store results into
// the leader's inbox (and the leader its decision into the peers' mail), then
// a thread releases a sequence number at cluster scope, which the reader
// acquires.  A writer refills a mail field only after the reader has
// signalled that it is done with the previous content, so one copy of each
// suffices.  Every wait is bounded; once any CTA gives up it sets the error
// word, the others see it in their next wait, and all three reach the final
// cluster barrier (no CTA exits while a peer may still access its shared
// memory).

__device__ __forceinline__ unsigned cluster_rank()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void cluster_barrier()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
template <class T>
__device__ __forceinline__ T *peer(T *p, unsigned rank)   // the same shared-memory object in CTA `rank`
{
    T *r;
    asm volatile("mapa.u64 %0, %1, %2;" : "=l"(r) : "l"(p), "r"(rank));
    return r;
}
__device__ __forceinline__ void st_release_cl(int *p, int v)
{
    asm volatile("st.release.cluster.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_cl() { asm volatile("fence.acq_rel.cluster;" ::: "memory"); }
__device__ __forceinline__ void st_relaxed_cl(int *p, int v)   // after fence_cl: a release
{
    asm volatile("st.relaxed.cluster.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_acquire_cl(const int *p)
{
    int v;
    asm volatile("ld.acquire.cluster.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
// Thread 0: wait until a mail flag of this CTA reaches v.
__device__ bool wait_mail(const int *flag, int v, const FrameArgs &a)
{
    const unsigned long long t0 = globaltimer_ns();
    while (ld_acquire_cl(flag) < v) {
        if (*(volatile int *)a.error) return false;
        if ((long long)(globaltimer_ns() - t0) > a.timeout_ns) {
            atomicCAS(a.error, 0, EVXG_ERROR_OPERATION_TIMEDOUT);
            return false;
        }
        __nanosleep(20);
    }
    return true;
}
__device__ __forceinline__ void copy_block(int16_t *to, const int16_t *from)   // 384 samples, whole CTA
{
    for (int c = threadIdx.x; c < MB_N / 8; c += NT) reinterpret_cast<uint4 *>(to)[c] = reinterpret_cast<const uint4 *>(from)[c];
}
__device__ void publish_decision(const evxg_block_desc &d, int n)   // leader, one thread
{
    MbShared &S = SM();
    for (unsigned p = 1; p < 3; p++) {
        int *to = reinterpret_cast<int *>(peer(&S.mail.left, p));
        for (int i = 0; i < 7; i++) to[i] = reinterpret_cast<const int *>(&d)[i];
    }
    fence_cl();   // one fence releases both descriptors
    st_relaxed_cl(peer(&S.mail.dec_seq, 1), n);
    st_relaxed_cl(peer(&S.mail.dec_seq, 2), n);
}

__device__ __forceinline__ void bar_sync(int id, int nt) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nt) : "memory"); }

// Window 0 moved on by one MB (new origin nox / ncox): every row shifts left
// in shared memory and takes its new strip, from nstrip (prefetched) or from
// memory; one thread per row, threads 0 .. WL_ROWS + 2*WC_ROWS - 1.  The
// origin fields are left to the caller.
__device__ void shift_window0(const FrameArgs &a, int nox, int ncox, bool staged)
{
    MbShared &S = SM();
    Win &w = S.win[0];
    const int r = threadIdx.x, cw = a.W / 2, ch = a.H / 2;
    const int16_t *D = a.planes[a.dpb];
    constexpr int NLC = WL / 8, NCC = WC / 8;
    if (r < WL_ROWS) {
        int16_t *rowp = w.y + r * WL;
        const uint4 n0 = staged ? S.nstrip[2 * r] : win_chunk(D, a.W, a.H, w.oy + r, nox + WL - 16);
        const uint4 n1 = staged ? S.nstrip[2 * r + 1] : win_chunk(D, a.W, a.H, w.oy + r, nox + WL - 8);
        uint4 t[NLC - 2];
#pragma unroll
        for (int j = 0; j < NLC - 2; j++) t[j] = *reinterpret_cast<const uint4 *>(rowp + 16 + 8 * j);
#pragma unroll
        for (int j = 0; j < NLC - 2; j++) *reinterpret_cast<uint4 *>(rowp + 8 * j) = t[j];
        *reinterpret_cast<uint4 *>(rowp + WL - 16) = n0;
        *reinterpret_cast<uint4 *>(rowp + WL - 8) = n1;
    } else if (r < WL_ROWS + 2 * WC_ROWS) {
        const int rr = r - WL_ROWS, pl = rr >= WC_ROWS, cr = rr - pl * WC_ROWS;
        const int16_t *P = D + (size_t)a.W * a.H + (pl ? (size_t)cw * ch : 0);
        int16_t *rowp = (pl ? w.v : w.u) + cr * WC;
        const uint4 n0 = staged ? S.nstrip[2 * WL_ROWS + rr] : win_chunk(P, cw, ch, w.coy + cr, ncox + WC - 8);
        uint4 t[NCC - 1];
#pragma unroll
        for (int j = 0; j < NCC - 1; j++) t[j] = *reinterpret_cast<const uint4 *>(rowp + 8 + 8 * j);
#pragma unroll
        for (int j = 0; j < NCC - 1; j++) *reinterpret_cast<uint4 *>(rowp + 8 * j) = t[j];
        *reinterpret_cast<uint4 *>(rowp + WC - 8) = n0;
    }
}

// Leader, whole CTA, after the wavefront wait of MB (row, col): start copying
// the next MB's source and window 0's new strip for it (MB column c+4) into
// nsrc / nstrip.  Row r-2 has finished column c+4 (row r-1 finished c+2 after
// it), rows r and below have not reached it, and row r-1's pixels there are
// read again on demand, as for any newest strip; so the strip holds what the
// next MB would read itself.  Strips beyond the right edge (edge-filled
// chunks) are left to the next MB.
__device__ void prefetch_next(const FrameArgs &a, int row, int col, int nt)
{
    MbShared &S = SM();
    const int tid = threadIdx.x;
    const int ncol = col + 1;
    if (ncol >= a.mbw) {
        if (tid == 0) S.pf_px = -1;
        return;
    }
    const int npx = ncol * 16, npy = row * 16, cw = a.W / 2, ch = a.H / 2;
    const int16_t *Y = a.src, *U = Y + (size_t)a.W * a.H, *V = U + (size_t)cw * ch;
    if (tid < 48) {   // source: 16 luma rows x 2 chunks, 8 + 8 chroma rows
        const int16_t *from;
        int16_t *to;
        if (tid < 32) { from = Y + (size_t)(npy + (tid >> 1)) * a.W + npx + (tid & 1) * 8; to = S.nsrc + (tid >> 1) * 16 + (tid & 1) * 8; }
        else {
            const int k = tid - 32, pl = k >> 3, r = k & 7;
            from = (pl ? V : U) + (size_t)((npy >> 1) + r) * cw + (npx >> 1);
            to = S.nsrc + 256 + pl * 64 + r * 8;
        }
        cp_async16(to, from);
    }
    const Win &w = S.win[0];
    const int nox = win_ox(npx), ncox = win_cox(npx);
    const bool strip = w.valid && nox + WL <= a.W && ncox + WC <= cw;
    if (strip) {
        const int16_t *D = a.planes[a.dpb], *DU = D + (size_t)a.W * a.H, *DV = DU + (size_t)cw * ch;
        for (int e = tid; e < 2 * WL_ROWS + 2 * WC_ROWS; e += nt) {
            const int16_t *from;
            if (e < 2 * WL_ROWS) {
                const int r = e >> 1, y = min(max(w.oy + r, 0), a.H - 1);
                from = D + (size_t)y * a.W + nox + WL - 16 + (e & 1) * 8;
            } else {
                const int rr = e - 2 * WL_ROWS, pl = rr >= WC_ROWS, cr = rr - pl * WC_ROWS;
                const int y = min(max(w.coy + cr, 0), ch - 1);
                from = (pl ? DV : DU) + (size_t)y * cw + ncox + WC - 8;
            }
            cp_async16(&S.nstrip[e], from);
        }
    }
    if (tid == 0) { S.pf_px = npx; S.pf_py = npy; S.pf_strip = strip; }
}

// Leader: MB (row, col), the n-th MB of this cluster.
__device__ bool leader_mb(const FrameArgs &a, int row, int col, int n)
{
    MbShared &S = SM();
    const int tid = threadIdx.x;
    const int px = col * 16, py = row * 16, idx = row * a.mbw + col;
    // Before the wavefront wait: the source and, when window 0 moves on by
    // one MB, its shift and new strip (column c+3, whose rows above are read
    // again on demand) -- both prefetched during the previous MB when it was
    // in this row; the rows above of column c+2 are read after the wait.  A
    // window loaded whole is loaded after the wait.  Warps 0..10 do this
    // part (named barrier 1) while the last warp may still be making the
    // previous MB's releases; it joins at the CTA barrier before the search.
    constexpr int NP = NT - 32;
    if (tid < NP) {
        // (window 0's fields are as the previous MB, which ended with a CTA barrier, left them)
        Win &w = S.win[0];
        const int nox = win_ox(px), ncox = win_cox(px);
        const int16_t *dst = a.planes[a.dpb];
        const bool early = w.valid && w.pl == dst && w.oy == py - 16 - WL_OFF && w.coy == ((py - 16) >> 1) - WC_OFF &&
                           w.ox + 16 == nox && w.cox + 8 == ncox;
        cp_async_wait_all();
        bar_sync(1, NP);   // every prefetch copy has landed; every thread has compared window 0's origin
        const bool pf = S.pf_px == px && S.pf_py == py;
        if (pf) { if (tid < MB_N / 8) reinterpret_cast<uint4 *>(S.src)[tid] = reinterpret_cast<const uint4 *>(S.nsrc)[tid]; }
        else load_src_n(a, px, py, NP);
        if (early) shift_window0(a, nox, ncox, pf && S.pf_strip);
        if (tid == 0) {
            setup_mb(a, idx, px, py, false, nullptr);
            S.w0_early = early;
            if (early) { w.ox = nox; w.cox = ncox; }
            else req_window(0, dst, px, py - 16);
            S.row_abort = row > 0 && !wait_progress(a, row - 1, min(col + 2, a.mbw - 1));   // see mb_row
        }
        bar_sync(1, NP);
        if (!S.row_abort) {
            if (early && row > 0) {   // column c+2's rows above: copied while the search's first step runs
                int y0, y1, cy0, cy1;
                rows_above(py, y0, y1, cy0, cy1);
                const Grp gp{1, 0, NP};
                if (!refresh_strip_async(gp, S.win[0], dst, a.W, a.H, y0, y1, cy0, cy1, WL - 32, WC - 16))
                    refresh_strip(gp, S.win[0], dst, a.W, a.H, y0, y1, cy0, cy1, WL - 32, WC - 16);
            }
            cp_async_commit();
            prefetch_next(a, row, col, NP);
            cp_async_commit();
        }
    }
    __syncthreads();
    if (S.row_abort) return false;
    if (!S.w0_early) {
        load_windows(a.W, a.H);
        __syncthreads();
    }
    intra_bc_search(G_ALL, a, px, py, true);
    if (tid == 0)
        S.row_abort = !((a.type == EVXG_FRAME_INTRA || wait_mail(&S.mail.f_seq, n, a)) && wait_mail(&S.mail.d_seq, n, a));
    __syncthreads();
    if (S.row_abort) return false;
    const Inbox &in = S.mail.in[n & 1];
    if (tid == 0) {   // the predictions are read where the ranks left them
        S.predp[1] = in.f_pred; S.predp[2] = in.b_pred; S.predp[4 + in.dir_best] = in.d_pred;
        S.predp[3] = a.type == EVXG_FRAME_INTER ? in.x_pred : S.pred[3];   // third reference, or the bi-prediction
        S.srch[1].out = in.f_out; S.srch[1].out_sad = in.f_sad;
        S.srch[2].out = in.b_out; S.srch[2].out_sad = in.b_sad;
        if (a.type == EVXG_FRAME_INTER) {
            S.rout[0] = in.f_out; S.rsad[0] = in.f_sad; S.rpred[0] = 1;
            S.rout[1] = in.b_out; S.rsad[1] = in.b_sad; S.rpred[1] = 2;
            S.rout[2] = in.x_out; S.rsad[2] = in.x_sad; S.rpred[2] = 3;
        }
        S.dir_best = in.dir_best; S.dir_sad = in.dir_sad;
        for (int m = 0; m < 3; m++) S.modes[m] = in.modes[m];
        if (a.type == EVXG_FRAME_INTER)
            for (int k = 0; k < 4; k++) { S.cd[k] = in.cd[k]; S.cost[k] = in.cost[k]; S.cpred[k] = k ? 3 + k : -1; }
    }
    __syncthreads();
    if (a.type == EVXG_FRAME_BIDIR) bi_prediction();
    if (tid == 0) {
        decide(a);
        if (a.type != EVXG_FRAME_INTER) publish_decision(S.cd[4].d, n);   // encoding does not change the modes or MVs
    }
    __syncthreads();
    if (S.need_encode) encode_candidates(G_ALL, a, 4, 1);
    if (tid == 0) {
        rdo_choose();
        if (a.type == EVXG_FRAME_INTER) publish_decision(S.cd[S.chosen].d, n);
    }
    __syncthreads();
    if (tid == 0 && row == 1) wait_progress(a, 0, min(col + 3, a.mbw - 1));   // see mb_row
    __syncthreads();
    const int ch = S.chosen;
    const bool remote = a.type == EVXG_FRAME_INTER && ch < 4;   // an intra candidate encoded by rank 2
    const int16_t *rec = remote ? peer(S.rec[ch], 2) : S.rec[ch];
    write_back(a, px, py, idx, rec, remote ? peer(S.lev[ch], 2) : S.lev[ch]);
    if (tid < 32)   // the right column, rank 2's left neighbour for the next MB (released with wr_seq)
        peer(S.mail.lcol, 2)[tid] = rec[tid < 16 ? tid * 16 + 15 : 256 + ((tid - 16) >> 3) * 64 + ((tid - 16) & 7) * 8 + 7];
    __syncthreads();
    if (tid == NT - 32) {   // releases, ordered after the barrier (so after every thread's stores), by
        st_release(&a.progress[row], col);     // the last warp: thread 0 goes on to the next MB's waits
        st_release_cl(peer(&S.mail.wr_seq, 2), n);
    }
    return true;
}

// Search k of search_mb: its state, its windows at the MB and at the
// predictor, its prediction buffer.  Searches 0 and 1 use the forward and
// backward resources; search 2 (a third reference) the intra search's state
// and window 0 (unused on ranks 1 and 2), window 5 and the bi-prediction buffer.
__device__ __forceinline__ int sm_srch(int k) { return k == 2 ? 0 : 1 + k; }
__device__ __forceinline__ int sm_wa(int k) { return k == 2 ? 5 : 1 + 2 * k; }
__device__ __forceinline__ int sm_wb(int k) { return k == 2 ? 0 : 2 + 2 * k; }
__device__ __forceinline__ int sm_pred(int k) { return k == 2 ? 3 : 1 + k; }

// The reference plane set of search k and its result slot in the leader's
// inbox (0 forward / nearest, 1 backward / second, 2 third reference): with
// bwd the backward search, else B frames' forward search or P frames' k-th
// reference.
__device__ __forceinline__ const int16_t *sm_ref(const FrameArgs &a, int k, bool bwd)
{
    return a.planes[bwd ? a.ref_bwd : (a.type == EVXG_FRAME_INTER ? a.ref_slot[k] : a.ref_fwd)];
}
__device__ __forceinline__ int sm_out(int k, bool bwd) { return bwd ? 1 : k; }

// Ranks 1 and 2: ns inter searches of the n-th MB (see sm_ref), handed to the
// leader's inbox (the caller releases the sequence flag); several searches
// run side by side on equal warp groups.  What does not depend on the left
// neighbour's decision -- the source, the predictor's other inputs (row r-1
// has finished column c+1), the windows around the MB and their metrics --
// comes before the wait for the leader's decision of the previous MB.
__device__ bool search_mb(const FrameArgs &a, int row, int col, int n, int ns, bool bwd)
{
    MbShared &S = SM();
    const int tid = threadIdx.x;
    const int px = col * 16, py = row * 16, idx = row * a.mbw + col;
    if (tid == 0) S.row_abort = row > 0 && !wait_progress(a, row - 1, min(col + 1, a.mbw - 1));
    __syncthreads();
    if (S.row_abort) return false;
    load_src(a, px, py);
    if (tid == 0) {
        setup_mb(a, idx, px, py, false, nullptr);
        pred_gather(a, idx, a.type == EVXG_FRAME_INTER, S.pin);
        for (int k = 0; k < ns; k++) req_window(sm_wa(k), sm_ref(a, k, bwd), px, py);
    }
    __syncthreads();
    load_windows(a.W, a.H);
    __syncthreads();
    const int gsz = NT / ns, k = tid / gsz;   // this thread's search and its group (named barriers 5..7)
    const Grp g = ns == 1 ? G_ALL : Grp{5 + k, k * gsz, gsz};
    first_candidates(g, a, sm_srch(k), sm_wa(k), sm_wb(k), px, py, true, false);
    if (tid == 0) {
        S.row_abort = !wait_mail(&S.mail.dec_seq, n - 1, a);
        if (!S.row_abort) {
            set_predictor(a, idx, px, py, S.pin, col > 0 ? &S.mail.left.d : nullptr);
            S.req.n = 0;
            if (S.sep)
                for (int j = 0; j < ns; j++) req_window(sm_wb(j), sm_ref(a, j, bwd), S.qx, S.qy);
        }
    }
    __syncthreads();
    if (S.row_abort) return false;
    if (S.req.n) {
        load_windows(a.W, a.H);
        __syncthreads();
    }
    inter_search(g, a, sm_srch(k), sm_wa(k), sm_wb(k), px, py, S.pred[sm_pred(k)], true);
    __syncthreads();
    Inbox *in = peer(&S.mail.in[n & 1], 0);
    for (int j = 0; j < ns; j++) {
        const int o = sm_out(j, bwd);
        int16_t *to = o == 0 ? in->f_pred : (o == 1 ? in->b_pred : in->x_pred);
        copy_block(to, S.pred[sm_pred(j)]);
        if (tid == 0) {
            Desc &d = o == 0 ? in->f_out : (o == 1 ? in->b_out : in->x_out);
            int &sad = o == 0 ? in->f_sad : (o == 1 ? in->b_sad : in->x_sad);
            d = S.srch[sm_srch(j)].out;
            sad = S.srch[sm_srch(j)].out_sad;
        }
    }
    return true;
}

// Rank 1: the forward search (B frames), or every reference's search (P
// frames: one to three, side by side).
__device__ bool fwd_mb(const FrameArgs &a, int row, int col, int n)
{
    if (a.type == EVXG_FRAME_INTRA) return true;
    if (!search_mb(a, row, col, n, a.type == EVXG_FRAME_INTER ? a.nref : 1, false)) return false;
    __syncthreads();
    if (threadIdx.x == 0) st_release_cl(peer(&SM().mail.f_seq, 0), n);
    return true;
}

__device__ bool aux_mb(const FrameArgs &a, int row, int col, int n)   // rank 2
{
    MbShared &S = SM();
    const int tid = threadIdx.x;
    const int px = col * 16, py = row * 16;
    // B frames: the backward search.
    const bool searched = a.type == EVXG_FRAME_BIDIR;
    if (searched && !search_mb(a, row, col, n, 1, true)) return false;
    // Directional intra reads row r-1 up to column c from the destination
    // slot (the search has waited for column c+1) and the right column of
    // MB (r, c-1), which the leader hands over in lcol with wr_seq.
    if (tid == 0) S.row_abort = !searched && row > 0 && !wait_progress(a, row - 1, col);
    __syncthreads();
    if (S.row_abort) return false;
    if (!searched) {
        load_src(a, px, py);
        if (tid == 0) setup_mb(a, row * a.mbw + col, px, py, false, nullptr);
    }
    nbr_top(a, px, py);
    if (tid == 0) S.row_abort = !wait_mail(&S.mail.wr_seq, n - 1, a);
    __syncthreads();
    if (S.row_abort) return false;
    nbr_left_modes(px, py);
    directional_intra(G_ALL);
    if (a.type == EVXG_FRAME_INTER) {
        if (tid == 0) intra_candidates();
        __syncthreads();
        encode_candidates(G_ALL, a, 0, 4);
    }
    Inbox *in = peer(&S.mail.in[n & 1], 0);
    if (a.type != EVXG_FRAME_INTER) copy_block(in->d_pred, S.pred[4 + S.dir_best]);
    if (tid == 0) {
        in->dir_best = S.dir_best; in->dir_sad = S.dir_sad;
        for (int m = 0; m < 3; m++) in->modes[m] = S.modes[m];
        if (a.type == EVXG_FRAME_INTER)
            for (int k = 0; k < 4; k++) { in->cd[k] = S.cd[k]; in->cost[k] = S.cost[k]; }
    }
    __syncthreads();
    if (tid == 0) st_release_cl(peer(&S.mail.d_seq, 0), n);
    return true;
}

// Rows for a cluster: the leader claims them (single form: the frame's row
// counter; batched form: the tick's (stream, row) queue) and passes each on
// to ranks 1 and 2; every CTA then works on the row with that stream's
// parameters (a copy in its shared memory in the batched form).
template <bool kBatched>
__device__ void cluster_main(const FrameArgs &a0, const FrameArgs *args, const int2 *queue, const int *qlen, int *qctr)
{
    MbShared &S = SM();
    __shared__ int s_item;
    __shared__ FrameArgs sa;
    const int tid = threadIdx.x;
    const unsigned rank = cluster_rank();
    init_tables();
    if (tid == 0) {
        S.mail.row_seq = 0; S.mail.dec_seq = 0; S.mail.wr_seq = 0; S.mail.f_seq = 0; S.mail.d_seq = 0;
        S.row_abort = 0; S.pf_px = -1;
        sa = kBatched ? args[0] : a0;   // batched: every stream of a tick shares the error word and the timeout
    }
    const int nq = kBatched ? __ldg(qlen) : a0.mbh;
    cluster_barrier();   // every CTA's mail is initialised before any peer writes to it
    const FrameArgs &w = sa;   // for the waits before a row is known
    int n = 0;
    for (int k = 1;; k++) {
        if (tid == 0) {
            if (rank == 0) {
                const int r = atomicAdd(kBatched ? qctr : &a0.counters[0], 1);
                s_item = r < nq ? r : -1;
                for (unsigned p = 1; p < 3; p++) {
                    *peer(&S.mail.row_val, p) = s_item;
                    st_release_cl(peer(&S.mail.row_seq, p), k);
                }
            } else {
                s_item = wait_mail(&S.mail.row_seq, k, w) ? S.mail.row_val : -1;
            }
        }
        if (tid < NWIN) S.win[tid].valid = 0;   // windows are reused only along a row
        __syncthreads();
        const int item = s_item;
        if (item < 0) break;
        int row = item;
        if (kBatched) {
            const int2 q = queue[item];
            row = q.y;
            if (tid == 0) sa = args[q.x];
            __syncthreads();
        }
        const FrameArgs &a = sa;   // shared memory: read much faster than the kernel parameter by reference
        bool ok = true;
        for (int col = 0; col < a.mbw && ok; ++col) {
            ++n;
            ok = rank == 0 ? leader_mb(a, row, col, n) : (rank == 1 ? fwd_mb(a, row, col, n) : aux_mb(a, row, col, n));
            // The leader's MB ends with a barrier before its releases, which the
            // last warp makes while the others start the next MB.
            if (rank != 0) __syncthreads();
        }
        if (!ok) break;
    }
    cp_async_wait_all();
    cluster_barrier();   // no CTA leaves while a peer may still access its shared memory
}

__global__ void __cluster_dims__(3, 1, 1) __launch_bounds__(NT, 1) k_mb_cluster(FrameArgs a)
{
    cluster_main<false>(a, nullptr, nullptr, nullptr, nullptr);
}
__global__ void __cluster_dims__(3, 1, 1) __launch_bounds__(NT, 1) k_mb_cluster_b(const FrameArgs *args, const int2 *queue,
                                                                                 const int *qlen, int *qctr)
{
    cluster_main<true>(args[0], args, queue, qlen, qctr);
}

size_t mb_shared_bytes() { return sizeof(MbShared); }
int mb_threads() { return NT; }

}  // namespace evxg
