// evxg_serialize.cpp -- host entropy coder of the EVX3 bitstream: the part of
// engine_encode_frame that stays on the CPU (reference serialize_slice,
// src/video/serialize.cpp:624-686), written for this library.  It turns the
// tables the GPU pipeline produces (block table, previous block table, SAO
// table, quantised level planes) into the frame's slice bytes, identical to
// the reference's for the same tables.
//
// Binarisation and coding, as the reference defines the format:
//   * every binary decision goes through one adaptive binary arithmetic coder
//     with 32-bit range (abac.cpp): the probability of a 0 is the ratio of a
//     context's two counts, counts start at 1 and are halved (keeping them odd)
//     once their sum reaches 65536; interval rescaling emits bits as soon as
//     the interval lies in one half (E1/E2) and defers them while it straddles
//     the middle half (E3);
//   * multi-bit fields go least significant bit first, all through one
//     context; integers use exponential-Golomb codes (golomb.cpp) -- a signed
//     value v is coded as the unsigned index 2|v| + (v < 0) (0 for v == 0);
//   * residual 8x8 blocks use a significance map in scan order (stream.cpp:
//     996-1075): last significant position, per-position significance flags,
//     then per coefficient greater-than-1 / greater-than-2 flags, a Golomb
//     remainder and a sign through the coder's own adaptive model.
// Every context starts afresh with each slice, so slices of different frames
// can be coded on different threads at the same time.
#include <cstdint>
#include <cstring>
#include <vector>

#include "evxg.h"

namespace evxg {
int fail(int code, const char *what);
}

namespace {

constexpr int BT_INTRA = 1, BT_MOTION = 2, BT_COPY = 4, INTRA_DEFAULT = 1;

// Output bits, least significant bit of each byte first (bitstream.cpp),
// gathered 64 at a time.
struct BitSink {
    std::vector<uint8_t> bytes;
    uint64_t acc = 0;   // pending bits, the oldest in bit 0
    int n = 0;
    void put(unsigned b)
    {
        acc |= (uint64_t)(b & 1u) << n;
        if (++n == 64) spill();
    }
    void put_run(unsigned b, uint32_t count)   // count copies of bit b
    {
        while (count) {
            const int k = (int)(count < (uint32_t)(64 - n) ? count : (uint32_t)(64 - n));
            if (b) acc |= (k == 64 ? ~0ull : ((1ull << k) - 1)) << n;
            n += k;
            count -= (uint32_t)k;
            if (n == 64) spill();
        }
    }
    void spill()
    {
        for (int i = 0; i < 8; i++) bytes.push_back((uint8_t)(acc >> (8 * i)));
        acc = 0;
        n = 0;
    }
    void close()   // the last partial byte, its unused high bits 0
    {
        for (int i = 0; i < (n + 7) / 8; i++) bytes.push_back((uint8_t)(acc >> (8 * i)));
        acc = 0;
        n = 0;
    }
};

// Adaptive model of one binary decision: counts of 0s and of 1s seen.
struct Model {
    uint32_t c[2] = {1, 1};
};

// floor(n / d) for n < 2^48 and 2 <= d < 2^16 -- the split of the coder's
// interval, span * count0 / (count0 + count1), whose counts stay below 2^16 --
// as the high half of n * r[d], r[d] = floor(2^64 / d) + 1: the product
// exceeds n / d by less than n / 2^64 < 2^-16 <= 1 / d, too little to reach
// the next integer, so the quotient is exact without a division per decision.
struct Reciprocals {
    uint64_t r[65536];
    Reciprocals()
    {
        r[0] = r[1] = 0;
        for (uint32_t d = 2; d < 65536; d++) r[d] = (uint64_t)((((unsigned __int128)1) << 64) / d) + 1;
    }
};
const Reciprocals &reciprocals()
{
    static const Reciprocals t;
    return t;
}
inline uint64_t div_small(uint64_t n, uint32_t d, const uint64_t *r)
{
    return d == 1 ? n : (uint64_t)(((unsigned __int128)n * r[d]) >> 64);
}

class Coder {
public:
    explicit Coder(BitSink &s) : out_(s), rcp_(reciprocals().r) {}

    // One decision through model m.
    void code(unsigned bit, Model &m)
    {
        bit &= 1u;
        const uint64_t span = (uint64_t)(hi_ - lo_);
        const uint32_t split = lo_ + (uint32_t)div_small(span * m.c[0], m.c[0] + m.c[1], rcp_);
        if (bit) lo_ = split + 1;
        else hi_ = split;
        if (++m.c[bit] + m.c[bit ^ 1u] >= 65536u) {
            m.c[0] = (m.c[0] >> 1) | 1u;
            m.c[1] = (m.c[1] >> 1) | 1u;
        }
        renormalise();
    }
    // A decision through the coder's own model (the residual signs).
    void code_own(unsigned bit) { code(bit, own_); }
    // n bits of v, least significant first, through model m.
    void code_bits(uint32_t v, int n, Model &m)
    {
        for (int i = 0; i < n; i++) code((v >> i) & 1u, m);
    }
    // Exponential-Golomb code of index k (k + 1 needs nb bits): nb - 1 zeros,
    // then k + 1 from its most significant bit down.
    void code_golomb(uint32_t k, Model &m)
    {
        const uint32_t v = k + 1;
        int nb = 0;
        while ((v >> nb) > 1u) nb++;
        for (int i = 0; i < nb; i++) code(0, m);
        for (int i = nb; i >= 0; i--) code((v >> i) & 1u, m);
    }
    void code_unsigned(uint16_t v, Model &m) { code_golomb(v, m); }
    void code_signed(int16_t v, Model &m)
    {
        const int32_t a = v < 0 ? -(int32_t)v : v;
        code_golomb(v == 0 ? 0u : (((uint32_t)a << 1) | (v < 0 ? 1u : 0u)) - 1u, m);
    }
    // Close the interval: one more deferred bit, then the side of the quarter
    // mark low lies on (abac.cpp:359-391).
    void finish()
    {
        e3_++;
        emit(lo_ < kQuarter ? 0u : 1u);
    }

private:
    static constexpr uint32_t kTop = 0x80000000u, kQuarter = 0x3FFFFFFFu, kThreeQuarters = 0xBFFFFFFDu;
    void emit(unsigned b)
    {
        out_.put(b);
        out_.put_run(b ^ 1u, e3_);
        e3_ = 0;
    }
    void renormalise()
    {
        for (;;) {
            const uint32_t same = ~(hi_ ^ lo_);
            if (same & kTop) {
                // The k leading bits low and high share are decided, one
                // after another (each doubling the interval); the bits
                // deferred so far follow the first of them.  (low < high,
                // so k < 32.)
                const int k = __builtin_clz(~same);
                emit(hi_ >> 31);
                for (int i = 30; i > 31 - k; i--) out_.put((hi_ >> i) & 1u);
                hi_ = (hi_ << k) | ((1u << k) - 1u);
                lo_ <<= k;
            } else if (hi_ <= kThreeQuarters && lo_ > kQuarter) {   // straddling the middle: defer
                hi_ = ((hi_ - (kQuarter + 1)) << 1) | 1u;
                lo_ = (lo_ - (kQuarter + 1)) << 1;
                e3_++;
            } else {
                return;
            }
        }
    }
    BitSink &out_;
    const uint64_t *rcp_;
    uint32_t lo_ = 0, hi_ = 0xFFFFFFFFu, e3_ = 0;
    Model own_;
};

// The slice's metadata models (common.h:141-171): one per field.
struct MetaModels {
    Model block_type, intra_mode, target, mvd_x, mvd_y, sp_pred, sp_amount, sp_index, qdelta;
    Model mpm_flag, mpm_idx;
    Model sao_merge, sao_type, sao_eo_class, sao_offset, sao_band;
    Model b_mode, b_target, b_mvd_x, b_mvd_y, b_sp_pred, b_sp_amount, b_sp_index;
};

// Residual models: a set for intra-default blocks and one for the others,
// each 64 significance flags, the last-position count (64; 65..67 unused),
// greater-than-1 and greater-than-2 flags per position group and previous
// state (68..75, 76..83), remainders per group (84..87).
constexpr int kSetSize = 88, kLast = 64, kGt1 = 68, kGt2 = 76, kRem = 84;

const uint8_t kZigzag[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
                             12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
                             35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
                             58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

// Scan position pos of an 8x8 block: zigzag, or row by row after vertical
// prediction (modes 1, 5), or column by column after horizontal prediction
// (modes 2, 6) of an intra-default block (scan.h:150-159).
inline int scan_at(int kind, int pos) { return kind == 0 ? kZigzag[pos] : (kind == 1 ? pos : (pos & 7) * 8 + (pos >> 3)); }
inline int scan_kind_of(const evxg_block_desc &d)
{
    if (d.block_type != INTRA_DEFAULT) return 0;
    const int m = d.intra_mode;
    return (m == 1 || m == 5) ? 1 : ((m == 2 || m == 6) ? 2 : 0);
}
inline int position_group(int pos) { return pos == 0 ? 0 : (pos <= 10 ? 1 : (pos <= 40 ? 2 : 3)); }
inline uint16_t magnitude(int16_t v) { return v == INT16_MIN ? (uint16_t)INT16_MAX : (uint16_t)(v < 0 ? -v : v); }

// One 8x8 block of levels (row stride `stride`) whose DC is coded as the
// difference to `pred_dc` (serialize.cpp:14-34, stream.cpp:996-1075).
void code_block(Coder &c, Model *set, const int16_t *blk, int stride, int16_t pred_dc, int kind)
{
    int16_t v[64];
    for (int r = 0; r < 8; r++) std::memcpy(v + 8 * r, blk + (size_t)r * stride, 16);
    v[0] = (int16_t)(v[0] - pred_dc);
    int last = -1;
    for (int pos = 63; pos >= 0; pos--)
        if (v[scan_at(kind, pos)]) { last = pos; break; }
    c.code_unsigned((uint16_t)(last + 1), set[kLast]);
    if (last < 0) return;
    for (int pos = 0; pos < last; pos++) c.code(v[scan_at(kind, pos)] != 0, set[pos]);
    int above1 = 0;   // a coefficient earlier in the scan was greater than 1
    for (int pos = 0; pos <= last; pos++) {
        const int16_t x = v[scan_at(kind, pos)];
        if (!x) continue;
        const int grp = position_group(pos), st = above1;
        const uint16_t m = magnitude(x);
        c.code(m > 1, set[kGt1 + 2 * grp + st]);
        if (m > 1) {
            above1 = 1;
            c.code(m > 2, set[kGt2 + 2 * grp + st]);
            if (m > 2) c.code_unsigned((uint16_t)(m - 3), set[kRem + grp]);
        }
        c.code_own(x < 0);
    }
}

// The MV predictor of block i (motion.cpp:271-346): median of the left, top
// and top-right (else top-left) motion vectors, then the co-located one of
// the previous table, averaged when there are two.
void mv_predictor(const evxg_block_desc *bt, const evxg_block_desc *prev, uint32_t mbw, uint32_t i, int16_t &px,
                  int16_t &py)
{
    const uint32_t bx = i % mbw, by = i / mbw;
    int16_t mx[3], my[3];
    int n = 0;
    auto take = [&](const evxg_block_desc &d) {
        if (d.block_type & BT_MOTION) { mx[n] = d.motion_x; my[n] = d.motion_y; n++; return true; }
        return false;
    };
    if (bx > 0) take(bt[i - 1]);
    if (by > 0) take(bt[i - mbw]);
    if (!(by > 0 && bx + 1 < mbw && take(bt[i - mbw + 1])) && by > 0 && bx > 0) take(bt[i - mbw - 1]);
    if (n < 3 && prev) take(prev[i]);
    auto mid = [](int16_t a, int16_t b, int16_t c) {
        if (a > b) { const int16_t t = a; a = b; b = t; }
        if (b > c) b = c;
        return a > b ? a : b;
    };
    if (n == 0) { px = 0; py = 0; }
    else if (n == 1) { px = mx[0]; py = my[0]; }
    else if (n == 2) { px = (int16_t)((mx[0] + mx[1]) / 2); py = (int16_t)((my[0] + my[1]) / 2); }
    else { px = mid(mx[0], mx[1], mx[2]); py = mid(my[0], my[1], my[2]); }
}

// floor(log2) of the DPB slot count: bits of a prediction target (serialize.cpp:233).
inline int target_bits(int ref_count)
{
    int b = 0;
    while ((ref_count >> (b + 1)) > 0) b++;
    return b;
}

void code_metadata(Coder &c, MetaModels &mm, const evxg_block_desc *bt, const evxg_block_desc *prev, uint32_t mbw,
                   uint32_t n, int tbits, bool bidir)   // serialize.cpp:184-300
{
    int16_t last_q = 0;
    for (uint32_t i = 0; i < n; i++) {
        const evxg_block_desc &d = bt[i];
        c.code_bits((uint32_t)d.block_type, 3, mm.block_type);
        if (d.block_type == INTRA_DEFAULT) {   // most probable modes: left and top (common.cpp:287-312)
            const uint32_t bx = i % mbw, by = i / mbw;
            const int left = (bx > 0 && bt[i - 1].block_type == INTRA_DEFAULT) ? bt[i - 1].intra_mode : 0;
            const int top = (by > 0 && bt[i - mbw].block_type == INTRA_DEFAULT) ? bt[i - mbw].intra_mode : 0;
            const int m0 = left, m1 = left == top ? (left == 0 ? 1 : 0) : top;
            const bool hit = d.intra_mode == m0 || d.intra_mode == m1;
            c.code(hit, mm.mpm_flag);
            if (hit) c.code(d.intra_mode == m1, mm.mpm_idx);
            else c.code_bits(d.intra_mode, 3, mm.intra_mode);
        }
        if (!(d.block_type & BT_INTRA)) c.code_bits(d.prediction_target, tbits, mm.target);
        if (d.block_type & BT_MOTION) {
            int16_t px, py;
            mv_predictor(bt, prev, mbw, i, px, py);
            c.code_signed((int16_t)(d.motion_x - px), mm.mvd_x);
            c.code_signed((int16_t)(d.motion_y - py), mm.mvd_y);
            c.code(d.sp_pred, mm.sp_pred);
            if (d.sp_pred) {
                c.code(d.sp_amount, mm.sp_amount);
                c.code_bits(d.sp_index, 3, mm.sp_index);
            }
        }
        if (bidir && !(d.block_type & BT_INTRA)) {   // second reference, its vector coded as is
            c.code_bits(d.prediction_mode, 2, mm.b_mode);
            if (d.prediction_mode == 2) {
                c.code_bits(d.prediction_target_b, tbits, mm.b_target);
                c.code_signed(d.motion_x_b, mm.b_mvd_x);
                c.code_signed(d.motion_y_b, mm.b_mvd_y);
                c.code(d.sp_pred_b, mm.b_sp_pred);
                if (d.sp_pred_b) {
                    c.code(d.sp_amount_b, mm.b_sp_amount);
                    c.code_bits(d.sp_index_b, 3, mm.b_sp_index);
                }
            }
        }
        if (!(d.block_type & BT_COPY)) {
            c.code_signed((int16_t)(d.q_index - last_q), mm.qdelta);
            last_q = d.q_index;
        }
    }
}

void code_sao(Coder &c, MetaModels &mm, const evxg_sao_info *sao, uint32_t mbw, uint32_t n)   // serialize.cpp:564-620
{
    for (uint32_t i = 0; i < n; i++) {
        const evxg_sao_info &s = sao[i];
        if (i % mbw > 0) c.code(s.merge_left, mm.sao_merge);
        if (!s.merge_left && i / mbw > 0) c.code(s.merge_above, mm.sao_merge);
        if (s.merge_left || s.merge_above) continue;
        for (const evxg_sao_params *p : {&s.luma, &s.chroma}) {
            c.code_bits(p->type, 2, mm.sao_type);
            if (p->type == 1) c.code_bits(p->eo_class, 2, mm.sao_eo_class);
            else if (p->type == 2) c.code_signed((int16_t)p->band_position, mm.sao_band);
            if (p->type != 0)
                for (int k = 0; k < 4; k++) c.code_signed(p->offsets[k], mm.sao_offset);
        }
    }
}

// Residuals of one plane (serialize.cpp:45-147): 16x16 luma macroblocks as
// four 8x8 blocks, or 8x8 chroma blocks, raster order, copy blocks skipped.
// The first DC is predicted from the left neighbour's nearest block (the
// block above at the left edge), the others within the macroblock from its
// first and third blocks.
void code_plane(Coder &c, Model *sets, const evxg_block_desc *bt, const int16_t *pl, int w, int h, bool luma)
{
    const int n = luma ? 16 : 8;
    uint32_t i = 0;
    for (int y = 0; y < h; y += n)
        for (int x = 0; x < w; x += n, i++) {
            const evxg_block_desc &d = bt[i];
            if (d.block_type & BT_COPY) continue;
            int16_t pdc = 0;
            if (x >= n) pdc = pl[(size_t)y * w + x - 8];
            else if (y >= n) pdc = pl[(size_t)(y - 8) * w + x];
            Model *set = sets + (d.block_type == INTRA_DEFAULT ? 0 : kSetSize);
            const int kind = scan_kind_of(d);
            const int16_t *b = pl + (size_t)y * w + x;
            code_block(c, set, b, w, pdc, kind);
            if (luma) {
                code_block(c, set, b + 8, w, b[0], kind);
                code_block(c, set, b + 8 * (size_t)w, w, b[0], kind);
                code_block(c, set, b + 8 * (size_t)w + 8, w, b[8 * (size_t)w], kind);
            }
        }
}

// ------------------------------------------------------------- decoding

// The arithmetic decoder of abac.cpp:165-559: a 32-bit window on the input,
// read most significant bit first (after 32 leading bits; past the end of the
// input the last bit read repeats), the interval split exactly as the coder
// splits it, and the same rescalings, each pulling one more input bit.  The
// coder emits one bit per rescaling plus two to close, so the slice's length
// follows from the decoder's own count.
class SliceDecoder {
public:
    SliceDecoder(const uint8_t *d, uint64_t n) : d_(d), nbits_(n * 8), rcp_(reciprocals().r)
    {
        uint32_t b = 0;
        for (int i = 0; i < 32; i++) {
            if (pos_ < nbits_) b = bit_at(pos_++);
            value_ = (value_ << 1) | b;
        }
    }
    unsigned decode(Model &m)
    {
        const uint32_t mid = lo_ + (uint32_t)div_small((uint64_t)(hi_ - lo_) * m.c[0], m.c[0] + m.c[1], rcp_);
        // The value lies in [low, high] for any slice of this format; outside
        // it the data is something else (flagged; the caller stops).
        bad_ |= (value_ < lo_) | (value_ > hi_);
        const unsigned bit = value_ > mid;   // selects, not branches: the decisions are unpredictable
        hi_ = bit ? hi_ : mid;
        lo_ = bit ? mid + 1 : lo_;
        if (++m.c[bit] + m.c[bit ^ 1u] >= 65536u) {
            m.c[0] = (m.c[0] >> 1) | 1u;
            m.c[1] = (m.c[1] >> 1) | 1u;
        }
        rescale();
        return bit;
    }
    unsigned decode_own() { return decode(own_); }
    uint32_t decode_bits(int n, Model &m)   // least significant bit first
    {
        uint32_t v = 0;
        for (int i = 0; i < n; i++) v |= decode(m) << i;
        return v;
    }
    // Exponential-Golomb code: the number k + 1 whose leading zeros precede it
    // (stream.cpp:713-778).  Returns k + 1; more than 32 leading zeros is no
    // code of this format.
    uint32_t decode_golomb_number(Model &m)
    {
        int zeros = 0;
        unsigned b = decode(m);
        while (!b) {
            if (++zeros > 32 || bad_) { bad_ = true; return 1; }
            b = decode(m);
        }
        uint32_t v = 1;
        for (int i = 0; i < zeros; i++) v = (v << 1) | decode(m);
        return v;
    }
    uint16_t decode_unsigned(Model &m) { return (uint16_t)(decode_golomb_number(m) - 1u); }
    int16_t decode_signed(Model &m)   // stream.cpp:780-857: low bit the sign, the rest the magnitude
    {
        int zeros = 0;
        unsigned b = decode(m);
        while (!b) {
            if (++zeros > 32 || bad_) { bad_ = true; return 0; }
            b = decode(m);
        }
        int16_t r = 1;
        for (int i = 0; i < zeros; i++) r = (int16_t)((r << 1) | (int)decode(m));
        const int16_t sign = (int16_t)(1 - 2 * (r & 1));
        int16_t out = (int16_t)(sign * ((r >> 1) & 0x7FFF));
        if (2 * zeros + 1 > 32) out = (int16_t)(out | 0x8000);
        return out;
    }
    bool bad() const { return bad_; }
    uint64_t bytes_used() const { return (shifts_ + 2 + 7) / 8; }

private:
    static constexpr uint32_t kQuarter = 0x3FFFFFFFu, kThreeQuarters = 0xBFFFFFFDu;
    unsigned bit_at(uint64_t i) const { return (d_[i >> 3] >> (i & 7)) & 1u; }
    // The next input bit; within one rescaling, past the end of the input the
    // last bit read repeats (0 if none was read yet), as abac.cpp:306-349 reads.
    unsigned next_bit()
    {
        if (pos_ < nbits_) last_ = bit_at(pos_++);
        return last_;
    }
    // abac.cpp:306-349.  When low and high share their k leading bits, k
    // rescalings in a row shift them out (a lower-half one doubles the
    // interval, an upper-half one subtracts the half first -- the bit the
    // shift drops anyway, since the value lies in the interval and shares
    // those bits), so they happen at once; middle-half rescalings one by one.
    void rescale()
    {
        last_ = 0;
        for (;;) {
            const uint32_t same = ~(hi_ ^ lo_);
            if (same & 0x80000000u) {   // low < high, so k < 32
                const int k = __builtin_clz(~same);
                uint32_t in = 0;
                for (int i = 0; i < k; i++) in = (in << 1) | next_bit();
                hi_ = (hi_ << k) | ((1u << k) - 1u);
                lo_ <<= k;
                value_ = (value_ << k) | in;
                shifts_ += (uint64_t)k;
            } else if (hi_ <= kThreeQuarters && lo_ > kQuarter) {
                hi_ = ((hi_ - (kQuarter + 1)) << 1) | 1u;
                lo_ = (lo_ - (kQuarter + 1)) << 1;
                value_ = ((value_ - (kQuarter + 1)) << 1) | next_bit();
                shifts_++;
            } else {
                return;
            }
        }
    }
    const uint8_t *d_;
    uint64_t nbits_, pos_ = 0, shifts_ = 0;
    const uint64_t *rcp_;
    unsigned last_ = 0;
    uint32_t lo_ = 0, hi_ = 0xFFFFFFFFu, value_ = 0;
    Model own_;
    bool bad_ = false;
};

// One 8x8 block: levels in raster order into blk (row stride `stride`), the
// DC coded as the difference to pred_dc (unserialize.cpp:13-29,
// stream.cpp:1077-1158).
bool decode_block(SliceDecoder &c, Model *set, int16_t *blk, int stride, int16_t pred_dc, int kind)
{
    int16_t v[64] = {};
    const uint16_t n = c.decode_unsigned(set[kLast]);
    if (n > 64) return false;
    if (n) {
        const int last = n - 1;
        uint8_t sig[64] = {};
        for (int pos = 0; pos < last; pos++) sig[pos] = (uint8_t)c.decode(set[pos]);
        sig[last] = 1;
        int above1 = 0;
        for (int pos = 0; pos <= last; pos++) {
            if (!sig[pos]) continue;
            const int grp = position_group(pos), st = above1;
            uint16_t m = 1;
            if (c.decode(set[kGt1 + 2 * grp + st])) {
                above1 = 1;
                m = 2;
                if (c.decode(set[kGt2 + 2 * grp + st])) m = (uint16_t)(c.decode_unsigned(set[kRem + grp]) + 3);
            }
            int16_t x = (int16_t)m;
            if (c.decode_own()) x = (int16_t)-x;
            v[scan_at(kind, pos)] = x;
        }
    }
    v[0] = (int16_t)(v[0] + pred_dc);
    for (int r = 0; r < 8; r++) std::memcpy(blk + (size_t)r * stride, v + 8 * r, 16);
    return !c.bad();
}

// unserialize_block_table_unified (unserialize.cpp:181-308): writes only the
// fields the slice codes; the rest keep the values of earlier frames.
void decode_metadata(SliceDecoder &c, MetaModels &mm, evxg_block_desc *bt, const evxg_block_desc *prev, uint32_t mbw,
                     uint32_t n, int tbits, bool bidir)
{
    int16_t last_q = 0;
    for (uint32_t i = 0; i < n && !c.bad(); i++) {
        evxg_block_desc &d = bt[i];
        d.block_type = (int32_t)c.decode_bits(3, mm.block_type);
        if (d.block_type == INTRA_DEFAULT) {
            const uint32_t bx = i % mbw, by = i / mbw;
            const int left = (bx > 0 && bt[i - 1].block_type == INTRA_DEFAULT) ? bt[i - 1].intra_mode : 0;
            const int top = (by > 0 && bt[i - mbw].block_type == INTRA_DEFAULT) ? bt[i - mbw].intra_mode : 0;
            const int m0 = left, m1 = left == top ? (left == 0 ? 1 : 0) : top;
            if (c.decode(mm.mpm_flag)) d.intra_mode = (uint8_t)(c.decode(mm.mpm_idx) ? m1 : m0);
            else d.intra_mode = (uint8_t)c.decode_bits(3, mm.intra_mode);
        }
        if (!(d.block_type & BT_INTRA)) d.prediction_target = (uint8_t)c.decode_bits(tbits, mm.target);
        if (d.block_type & BT_MOTION) {
            int16_t px, py;
            mv_predictor(bt, prev, mbw, i, px, py);
            d.motion_x = (int16_t)(c.decode_signed(mm.mvd_x) + px);
            d.motion_y = (int16_t)(c.decode_signed(mm.mvd_y) + py);
            d.sp_pred = (uint8_t)c.decode(mm.sp_pred);
            if (d.sp_pred) {
                d.sp_amount = (uint8_t)c.decode(mm.sp_amount);
                d.sp_index = (uint8_t)c.decode_bits(3, mm.sp_index);
            }
        }
        if (bidir && !(d.block_type & BT_INTRA)) {
            d.prediction_mode = (uint8_t)c.decode_bits(2, mm.b_mode);
            if (d.prediction_mode == 2) {
                d.prediction_target_b = (uint8_t)c.decode_bits(tbits, mm.b_target);
                d.motion_x_b = c.decode_signed(mm.b_mvd_x);
                d.motion_y_b = c.decode_signed(mm.b_mvd_y);
                d.sp_pred_b = (uint8_t)c.decode(mm.b_sp_pred);
                if (d.sp_pred_b) {
                    d.sp_amount_b = (uint8_t)c.decode(mm.b_sp_amount);
                    d.sp_index_b = (uint8_t)c.decode_bits(3, mm.b_sp_index);
                }
            }
        }
        if (!(d.block_type & BT_COPY)) {
            d.q_index = (uint8_t)(c.decode_signed(mm.qdelta) + last_q);
            last_q = d.q_index;
        }
    }
}

void decode_sao(SliceDecoder &c, MetaModels &mm, evxg_sao_info *sao, uint32_t mbw, uint32_t n)   // unserialize.cpp:573-632
{
    for (uint32_t i = 0; i < n && !c.bad(); i++) {
        evxg_sao_info &s = sao[i];
        s = evxg_sao_info{};
        if (i % mbw > 0) s.merge_left = (uint8_t)c.decode(mm.sao_merge);
        if (!s.merge_left && i / mbw > 0) s.merge_above = (uint8_t)c.decode(mm.sao_merge);
        if (s.merge_left || s.merge_above) continue;
        for (evxg_sao_params *p : {&s.luma, &s.chroma}) {
            p->type = (uint8_t)c.decode_bits(2, mm.sao_type);
            if (p->type == 1) p->eo_class = (uint8_t)c.decode_bits(2, mm.sao_eo_class);
            else if (p->type == 2) p->band_position = (uint8_t)c.decode_signed(mm.sao_band);
            if (p->type != 0)
                for (int k = 0; k < 4; k++) p->offsets[k] = (int8_t)c.decode_signed(mm.sao_offset);
        }
    }
}

// Residuals of one plane (unserialize.cpp:43-148), the mirror of code_plane.
bool decode_plane(SliceDecoder &c, Model *sets, const evxg_block_desc *bt, int16_t *pl, int w, int h, bool luma)
{
    const int n = luma ? 16 : 8;
    uint32_t i = 0;
    for (int y = 0; y < h; y += n)
        for (int x = 0; x < w; x += n, i++) {
            const evxg_block_desc &d = bt[i];
            if (d.block_type & BT_COPY) continue;
            int16_t pdc = 0;
            if (x >= n) pdc = pl[(size_t)y * w + x - 8];
            else if (y >= n) pdc = pl[(size_t)(y - 8) * w + x];
            Model *set = sets + (d.block_type == INTRA_DEFAULT ? 0 : kSetSize);
            const int kind = scan_kind_of(d);
            int16_t *b = pl + (size_t)y * w + x;
            if (!decode_block(c, set, b, w, pdc, kind)) return false;
            if (luma) {
                if (!decode_block(c, set, b + 8, w, b[0], kind) ||
                    !decode_block(c, set, b + 8 * (size_t)w, w, b[0], kind) ||
                    !decode_block(c, set, b + 8 * (size_t)w + 8, w, b[8 * (size_t)w], kind))
                    return false;
            }
        }
    return true;
}

}  // namespace

extern "C" {

int evxg_serialize_slice(const evxg_config *cfg, uint32_t aligned_w, uint32_t aligned_h, const evxg_frame *frame,
                         const evxg_block_desc *blocks, const evxg_block_desc *prev_blocks, const evxg_sao_info *sao,
                         const int16_t *levels, uint8_t *out, uint64_t capacity, uint64_t *out_len)
{
    using evxg::fail;
    if (!frame || !blocks || !prev_blocks || !sao || !levels || !out_len)
        return fail(EVXG_ERROR_INVALIDARG, "evxg_serialize_slice: null argument");
    if (!aligned_w || !aligned_h || (aligned_w & 15) || (aligned_h & 15))
        return fail(EVXG_ERROR_INVALIDARG, "evxg_serialize_slice: aligned size must be a non-zero multiple of 16");
    evxg_config c;
    evxg_config_default(&c);
    if (cfg) c = *cfg;
    if (c.ref_count < 1 || c.ref_count > 4) return fail(EVXG_ERROR_INVALIDARG, "evxg_serialize_slice: bad reference count");
    const uint32_t mbw = aligned_w / 16, n = mbw * (aligned_h / 16);
    BitSink sink;
    sink.bytes.reserve((size_t)aligned_w * aligned_h / 4);
    Coder coder(sink);
    MetaModels mm;
    std::vector<Model> sets(2 * kSetSize);
    code_metadata(coder, mm, blocks, prev_blocks, mbw, n, target_bits(c.ref_count),
                  c.b_frames && frame->type == EVXG_FRAME_BIDIR);
    code_sao(coder, mm, sao, mbw, n);
    const size_t ny = (size_t)aligned_w * aligned_h, nc = (size_t)(aligned_w / 2) * (aligned_h / 2);
    code_plane(coder, sets.data(), blocks, levels, (int)aligned_w, (int)aligned_h, true);
    code_plane(coder, sets.data(), blocks, levels + ny, (int)aligned_w / 2, (int)aligned_h / 2, false);
    code_plane(coder, sets.data(), blocks, levels + ny + nc, (int)aligned_w / 2, (int)aligned_h / 2, false);
    coder.finish();
    sink.close();   // the slice ends on a byte boundary: the last byte's unused bits stay 0
    *out_len = sink.bytes.size();
    if (sink.bytes.size() > capacity) return fail(EVXG_ERROR_CAPACITY_LIMIT, "evxg_serialize_slice: output buffer too small");
    std::memcpy(out, sink.bytes.data(), sink.bytes.size());
    return EVXG_SUCCESS;
}

int evxg_stream_header(const evxg_config *cfg, uint32_t width, uint32_t height, uint8_t out[14])
{
    if (!out || !width || !height || width > 65535 || height > 65535)
        return evxg::fail(EVXG_ERROR_INVALIDARG, "evxg_stream_header: bad argument");
    evxg_config c;
    evxg_config_default(&c);
    if (cfg) c = *cfg;
    // evx_header (common.h:55-64, pack(2)): magic, size, reference count,
    // padding, version 3.11, visible width and height, little-endian.
    const uint8_t h[14] = {'E', 'V', 'X', '1', 14, 0, c.ref_count, 0, 11, 3, (uint8_t)(width & 0xFF), (uint8_t)(width >> 8),
                           (uint8_t)(height & 0xFF), (uint8_t)(height >> 8)};
    std::memcpy(out, h, 14);
    return EVXG_SUCCESS;
}

int evxg_unserialize_slice(const evxg_config *cfg, uint32_t aligned_w, uint32_t aligned_h, const evxg_frame *frame,
                           const uint8_t *data, uint64_t len, evxg_block_desc *blocks,
                           const evxg_block_desc *prev_blocks, evxg_sao_info *sao, int16_t *levels, uint64_t *consumed)
{
    using evxg::fail;
    if (!frame || !data || !blocks || !prev_blocks || !sao || !levels)
        return fail(EVXG_ERROR_INVALIDARG, "evxg_unserialize_slice: null argument");
    if (!aligned_w || !aligned_h || (aligned_w & 15) || (aligned_h & 15))
        return fail(EVXG_ERROR_INVALIDARG, "evxg_unserialize_slice: aligned size must be a non-zero multiple of 16");
    evxg_config c;
    evxg_config_default(&c);
    if (cfg) c = *cfg;
    if (c.ref_count < 1 || c.ref_count > 4)
        return fail(EVXG_ERROR_INVALIDARG, "evxg_unserialize_slice: bad reference count");
    const uint32_t mbw = aligned_w / 16, n = mbw * (aligned_h / 16);
    SliceDecoder dec(data, len);
    MetaModels mm;
    std::vector<Model> sets(2 * kSetSize);
    decode_metadata(dec, mm, blocks, prev_blocks, mbw, n, target_bits(c.ref_count),
                    c.b_frames && frame->type == EVXG_FRAME_BIDIR);
    decode_sao(dec, mm, sao, mbw, n);
    const size_t ny = (size_t)aligned_w * aligned_h, nc = (size_t)(aligned_w / 2) * (aligned_h / 2);
    const bool ok = !dec.bad() &&
                    decode_plane(dec, sets.data(), blocks, levels, (int)aligned_w, (int)aligned_h, true) &&
                    decode_plane(dec, sets.data(), blocks, levels + ny, (int)aligned_w / 2, (int)aligned_h / 2, false) &&
                    decode_plane(dec, sets.data(), blocks, levels + ny + nc, (int)aligned_w / 2, (int)aligned_h / 2, false);
    if (consumed) *consumed = dec.bytes_used();
    if (!ok) return fail(EVXG_ERROR_INVALID_RESOURCE, "evxg_unserialize_slice: not a slice of this format");
    if (dec.bytes_used() > len) return fail(EVXG_ERROR_INVALID_RESOURCE, "evxg_unserialize_slice: slice truncated");
    return EVXG_SUCCESS;
}

}  // extern "C"
