// evxg_filters.cu -- frame-level kernels of the EVX3 encoder pipeline on sm_100a:
// RGB24 -> YUV 4:2:0 conversion, in-loop deblocking and SAO (RDO, merge and
// raster-order application).
//
// Reference: src/video/convert.cpp:11-160, src/video/deblock.cpp:14-305,
// src/video/sao.cpp:13-594 (luma-only merge branch, EVX_ENABLE_SAO_CHROMA_MERGE 0).
#include "evxg_device.cuh"

namespace evxg {

// ------------------------------------------------------------ conversion
// One thread per 2x2 pixel quad of the visible (cropped) frame; padding rows
// and columns of the aligned source stay at their zero initialisation.
__device__ __forceinline__ void convert_body(const FrameArgs &a)
{
    const int cw = min(a.vis_w, a.W), ch = min(a.vis_h, a.H);
    const int qx = blockIdx.x * blockDim.x + threadIdx.x, qy = blockIdx.y;
    if (2 * qx >= cw || 2 * qy >= ch) return;
    const int x = 2 * qx, y = 2 * qy;
    int16_t *Y = a.src, *U = a.src + (size_t)a.W * a.H, *V = U + (size_t)(a.W / 2) * (a.H / 2);
    int16_t u = 0, v = 0;
#pragma unroll
    for (int dy = 0; dy < 2; dy++)
#pragma unroll
        for (int dx = 0; dx < 2; dx++) {
            const uint8_t *p = a.rgb + ((size_t)(y + dy) * a.vis_w + x + dx) * 3;
            const int r = p[0], g = p[1], b = p[2];
            Y[(size_t)(y + dy) * a.W + x + dx] = (int16_t)(((77 * r + 150 * g + 29 * b + 128) >> 8) + 16);
            u = (int16_t)(u + ((-43 * r - 85 * g + 128 * b + 128) / 256) + 128);
            v = (int16_t)(v + ((128 * r - 107 * g - 21 * b + 128) / 256) + 128);
        }
    U[(size_t)qy * (a.W / 2) + qx] = (int16_t)((u + 2) >> 2);
    V[(size_t)qy * (a.W / 2) + qx] = (int16_t)((v + 2) >> 2);
}
__global__ void k_convert(FrameArgs a) { convert_body(a); }
__global__ void k_convert_b(const FrameArgs *args)
{
    __shared__ FrameArgs sa;
    if (const FrameArgs *a = batch_args(args, sa)) convert_body(*a);
}

// ------------------------------------------------------------ deblocking
__constant__ int16_t c_alpha[64] = {  // deblock.cpp:14-24
    0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 2, 2, 3, 3, 4, 5, 6, 7, 8, 9, 10, 12, 14, 16, 18, 20, 22, 24, 26, 29, 32, 35,
    38, 42, 46, 50, 54, 59, 64, 70, 76, 82, 89, 96, 104, 112, 120, 128, 138, 148, 158, 170, 182, 196, 210, 224,
    240, 255, 255, 255, 255, 255, 255, 255};
__constant__ int16_t c_beta[64] = {  // deblock.cpp:26-36
    0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 3, 3, 3, 4, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8, 9, 10, 11,
    12, 13, 14, 15, 16, 17, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18,
    18, 18, 18, 18, 18, 18, 18, 18};

// Effective QP and strength of the edge between block table entries li, ri
// (deblock.cpp:58-89, :148-150); strength 0 means no filtering.
__device__ __forceinline__ void edge_params(const evxg_block_desc *bt, int li, int ri, int qoff, int &qe, int &st)
{
    const int lt = __ldg(&bt[li].block_type), rt = __ldg(&bt[ri].block_type);
    const int lq = __ldg(&bt[li].q_index), rq = __ldg(&bt[ri].q_index);
    const bool lc = lt & BT_COPY, rc = rt & BT_COPY;
    int aq;
    if (!lc && !rc) aq = (lq + rq) >> 1;
    else if (!lc) aq = lq;
    else if (!rc) aq = rq;
    else aq = 0;
    st = (lc && rc) ? 0 : ((lc ^ rc) ? 1 : (li != ri ? 2 : 1));
    qe = min(aq + qoff, MAXQ);
}

// Filter one line across an edge; e points at q0, step is the distance between samples.
__device__ __forceinline__ void filter_line(int16_t *e, int step, int qe, int st, bool luma)   // deblock.cpp:91-146
{
    const int p0 = e[-step], p1 = e[-2 * step], p2 = e[-3 * step], p3 = e[-4 * step];
    const int q0 = e[0], q1 = e[step], q2 = e[2 * step], q3 = e[3 * step];
    int qi = qe;
    if (st == 2 && qe > 0) qi = min(qe + 2, MAXQ);
    if ((int16_t)iabs32(p0 - q0) >= c_alpha[qi] || (int16_t)iabs32(p1 - p0) >= c_beta[qi] ||
        (int16_t)iabs32(q1 - q0) >= c_beta[qi])
        return;
    if (st == 2) {
        e[-step] = (int16_t)rdiv(p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1, 8);
        e[-2 * step] = (int16_t)rdiv(p2 + p1 + p0 + q0, 4);
        e[0] = (int16_t)rdiv(p1 + 2 * p0 + 2 * q0 + 2 * q1 + q2, 8);
        e[step] = (int16_t)rdiv(p0 + q0 + q1 + q2, 4);
        if (luma) {
            e[-3 * step] = (int16_t)rdiv(2 * p3 + 3 * p2 + p1 + p0 + q0, 8);
            e[2 * step] = (int16_t)rdiv(2 * q3 + 3 * q2 + q1 + q0 + p0, 8);
        }
    } else {
        e[-step] = (int16_t)rdiv(((q0 + p0) * 4) + p1 - q1, 8);
        e[0] = (int16_t)rdiv(((q0 + p0) * 4) + q1 - p1, 8);
        if (luma) {
            e[-2 * step] = (int16_t)rdiv((p2 * 4) + (p0 * 2) + (q0 * 2), 8);
            e[step] = (int16_t)rdiv((q2 * 4) + (q0 * 2) + (p0 * 2), 8);
        }
    }
}

// One CTA per plane.  The reference's order (deblock.cpp:233-272) is: row band
// 0 vertical edges; then per 8-row band j the horizontal edge at x=0 and, for
// x = 8, 16, ..., the horizontal edge (x, j) followed by the vertical edge
// (x, j).  Within a band, horizontal edges touch disjoint columns and vertical
// edge (x, j) only reads columns written by horizontal edges (x-8, j) and
// (x, j), so running all horizontal edges of the band and then all vertical
// edges gives the same samples; bands stay in order.
__device__ __forceinline__ void deblock_body(const FrameArgs &a)
{
    const int pl = blockIdx.x;
    const bool luma = pl == 0;
    const int w = luma ? a.W : a.W / 2, h = luma ? a.H : a.H / 2;
    const int mbs = luma ? 16 : 8, qoff = luma ? 0 : 2;
    int16_t *d = a.planes[a.dpb] + (pl == 0 ? 0 : (size_t)a.W * a.H + (pl - 1) * (size_t)(a.W / 2) * (a.H / 2));
    const int nv = (w / 8 - 1) * 8;
    const int tid = threadIdx.x;
    for (int j = 0; j < h; j += 8) {
        if (j > 0) {
            const int brow = (j / mbs) * a.mbw, arow = ((j - 1) / mbs) * a.mbw;
            for (int x = tid; x < w; x += blockDim.x) {
                int qe, st;
                edge_params(a.bt, x / mbs + arow, x / mbs + brow, qoff, qe, st);
                if (st) filter_line(d + (size_t)j * w + x, w, qe, st, luma);
            }
            __syncthreads();
        }
        const int brow = (j / mbs) * a.mbw;
        for (int t = tid; t < nv; t += blockDim.x) {
            const int x = ((t >> 3) + 1) * 8, y = j + (t & 7);
            int qe, st;
            edge_params(a.bt, (x - 1) / mbs + brow, x / mbs + brow, qoff, qe, st);
            if (st) filter_line(d + (size_t)y * w + x, 1, qe, st, luma);
        }
        __syncthreads();
    }
}
__global__ void __launch_bounds__(1024) k_deblock(FrameArgs a) { deblock_body(a); }
__global__ void __launch_bounds__(1024) k_deblock_b(const FrameArgs *args)
{
    __shared__ FrameArgs sa;
    if (const FrameArgs *a = batch_args(args, sa)) deblock_body(*a);
}

// ------------------------------------------------------------------ SAO
__constant__ int8_t c_eo[4][4] = {{-1, 0, 1, 0}, {0, -1, 0, 1}, {-1, -1, 1, 1}, {1, -1, -1, 1}};   // sao.cpp:20-25

__device__ __forceinline__ int sclamp(int v) { return v < 0 ? 0 : (v > 255 ? 255 : v); }
__device__ __forceinline__ int eo_cat(int p, int a, int b)   // sao.cpp:27-38
{
    const int s = ((a > p) - (a < p)) + ((b > p) - (b < p));
    return s == 2 ? 0 : s == 1 ? 1 : s == -1 ? 2 : s == -2 ? 3 : 4;
}
__device__ __forceinline__ unsigned sao_bits(const evxg_sao_params &p)   // sao.cpp:150-159
{
    if (p.type == 0) return 2;
    unsigned b = 2 + (p.type == 1 ? 2 : 5);
    for (int i = 0; i < 4; i++) b += p.offsets[i] ? 4 : 1;
    return b;
}
__device__ __forceinline__ int avg_off(int sum, int cnt)   // sao.cpp:205-207
{
    int a = (sum + (sum >= 0 ? cnt / 2 : -cnt / 2)) / cnt;
    return a > 7 ? 7 : (a < -7 ? -7 : a);
}
__device__ __forceinline__ float rd_cost64(long long ssd, float lambda, unsigned bits)
{
    return __fadd_rn(__ll2float_rn(ssd), __fmul_rn(lambda, __uint2float_rn(bits)));
}
// corrected value of pixel (x, y) under p, neighbours read from img (sao.cpp:40-97, :346-387);
// kCoherent reads through L2 only, for pixels other warps modify in the same kernel.
template <bool kCoherent = false>
__device__ __forceinline__ int ldpx(const int16_t *p) { return kCoherent ? __ldcg(p) : *p; }
template <bool kCoherent = false>
__device__ __forceinline__ int sao_px(const int16_t *img, int w, int h, int x, int y, const evxg_sao_params &p)
{
    const int v = ldpx<kCoherent>(img + (size_t)y * w + x);
    if (p.type == 2) {
        const int idx = (sclamp(v) >> 3) - p.band_position;
        return (idx >= 0 && idx < 4) ? sclamp(v + p.offsets[idx]) : v;
    }
    if (p.type == 1) {
        const int ax = x + c_eo[p.eo_class][0], ay = y + c_eo[p.eo_class][1];
        const int bx = x + c_eo[p.eo_class][2], by = y + c_eo[p.eo_class][3];
        if (ax < 0 || ax >= w || ay < 0 || ay >= h || bx < 0 || bx >= w || by < 0 || by >= h) return v;
        const int ct = eo_cat(v, ldpx<kCoherent>(img + (size_t)ay * w + ax), ldpx<kCoherent>(img + (size_t)by * w + bx));
        return ct < 4 ? sclamp(v + p.offsets[ct]) : v;
    }
    return v;
}

// Per-MB RDO of one plane block (sao.cpp:150-343); returns the parameters and
// the SSD they give.  Band and edge SSDs are assembled from per-band /
// per-category deltas, which sums the same integers as a full pass.
__device__ void sao_rdo_block(const int16_t *s, const int16_t *r, int w, int h, int x0, int y0, int n, float lambda,
                              evxg_sao_params &out, long long &out_ssd)
{
    out = evxg_sao_params{};
    long long base = 0;
    int bsum[32], bcnt[32];
    for (int k = 0; k < 32; k++) { bsum[k] = 0; bcnt[k] = 0; }
    for (int y = y0; y < y0 + n; y++)
        for (int x = x0; x < x0 + n; x++) {
            const int pv = __ldg(r + (size_t)y * w + x), sv = __ldg(s + (size_t)y * w + x);
            base += (long long)((sv - pv) * (sv - pv));
            const int b = sclamp(pv) >> 3;
            bsum[b] += sv - pv;
            bcnt[b]++;
        }
    float best = rd_cost64(base, lambda, 2u);
    long long best_ssd = base;
    // band offsets: the offset of band b does not depend on the band position
    int boff[32];
    long long bdelta[32];
    for (int k = 0; k < 32; k++) { boff[k] = bcnt[k] > 0 ? avg_off(bsum[k], bcnt[k]) : 0; bdelta[k] = 0; }
    for (int y = y0; y < y0 + n; y++)
        for (int x = x0; x < x0 + n; x++) {
            const int pv = __ldg(r + (size_t)y * w + x), sv = __ldg(s + (size_t)y * w + x);
            const int b = sclamp(pv) >> 3;
            const int cv = sclamp(pv + boff[b]);
            bdelta[b] += (long long)((sv - cv) * (sv - cv)) - (long long)((sv - pv) * (sv - pv));
        }
    for (int bp = 0; bp <= 28; bp++) {
        evxg_sao_params c{};
        c.type = 2; c.band_position = (uint8_t)bp;
        bool nz = false;
        long long ssd = base;
        for (int k = 0; k < 4; k++) {
            c.offsets[k] = (int8_t)boff[bp + k];
            nz |= boff[bp + k] != 0;
            ssd += bdelta[bp + k];
        }
        if (!nz) continue;
        const float cost = rd_cost64(ssd, lambda, sao_bits(c));
        if (cost < best) { best = cost; out = c; best_ssd = ssd; }
    }
    for (int ec = 0; ec < 4; ec++) {
        int cs[4] = {0, 0, 0, 0}, cc[4] = {0, 0, 0, 0};
        for (int y = y0; y < y0 + n; y++)
            for (int x = x0; x < x0 + n; x++) {
                const int ax = x + c_eo[ec][0], ay = y + c_eo[ec][1], bx = x + c_eo[ec][2], by = y + c_eo[ec][3];
                if (ax < 0 || ax >= w || ay < 0 || ay >= h || bx < 0 || bx >= w || by < 0 || by >= h) continue;
                const int pv = __ldg(r + (size_t)y * w + x);
                const int ct = eo_cat(pv, __ldg(r + (size_t)ay * w + ax), __ldg(r + (size_t)by * w + bx));
                if (ct < 4) { cs[ct] += __ldg(s + (size_t)y * w + x) - pv; cc[ct]++; }
            }
        evxg_sao_params c{};
        c.type = 1; c.eo_class = (uint8_t)ec;
        bool nz = false;
        for (int k = 0; k < 4; k++) { c.offsets[k] = (int8_t)(cc[k] > 0 ? avg_off(cs[k], cc[k]) : 0); nz |= c.offsets[k] != 0; }
        if (!nz) continue;
        long long ssd = base;
        for (int y = y0; y < y0 + n; y++)
            for (int x = x0; x < x0 + n; x++) {
                const int ax = x + c_eo[ec][0], ay = y + c_eo[ec][1], bx = x + c_eo[ec][2], by = y + c_eo[ec][3];
                if (ax < 0 || ax >= w || ay < 0 || ay >= h || bx < 0 || bx >= w || by < 0 || by >= h) continue;
                const int pv = __ldg(r + (size_t)y * w + x);
                const int ct = eo_cat(pv, __ldg(r + (size_t)ay * w + ax), __ldg(r + (size_t)by * w + bx));
                if (ct < 4) {
                    const int sv = __ldg(s + (size_t)y * w + x), cv = sclamp(pv + c.offsets[ct]);
                    ssd += (long long)((sv - cv) * (sv - cv)) - (long long)((sv - pv) * (sv - pv));
                }
            }
        const float cost = rd_cost64(ssd, lambda, sao_bits(c));
        if (cost < best) { best = cost; out = c; best_ssd = ssd; }
    }
    out_ssd = best_ssd;
}

// One thread per MB: own luma and chroma (U plane) parameters and the cost of
// keeping them, the starting point of the merge decision (sao.cpp:414-557).
__device__ __forceinline__ void sao_rdo_body(const FrameArgs &a)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= a.mbw * a.mbh) return;
    const int bx = m % a.mbw, by = m / a.mbw;
    const int16_t *rec = a.planes[a.dpb];
    const int cw = a.W / 2, ch = a.H / 2;
    evxg_sao_info info{};
    long long lssd, cssd;
    sao_rdo_block(a.src, rec, a.W, a.H, bx * 16, by * 16, 16, a.lambda, info.luma, lssd);
    sao_rdo_block(a.src + (size_t)a.W * a.H, rec + (size_t)a.W * a.H, cw, ch, bx * 8, by * 8, 8, a.lambda, info.chroma, cssd);
    float cur;
    if (info.luma.type == 0) cur = __fadd_rn(__ll2float_rn(lssd), __fmul_rn(a.lambda, 2.0f));
    else cur = __fadd_rn(__fsub_rn(__fadd_rn(__ll2float_rn(lssd), __fmul_rn(a.lambda, 1.0f)), __fmul_rn(a.lambda, 1.0f)),
                         __fmul_rn(a.lambda, __uint2float_rn(sao_bits(info.luma))));
    a.sao[m] = info;
    a.sao_cost[m] = cur;
}
__global__ void k_sao_rdo(FrameArgs a) { sao_rdo_body(a); }
__global__ void k_sao_rdo_b(const FrameArgs *args)
{
    __shared__ FrameArgs sa;
    if (const FrameArgs *a = batch_args(args, sa)) sao_rdo_body(*a);
}

__device__ __forceinline__ evxg_sao_params ld_params_cg(const evxg_sao_params *p)
{
    evxg_sao_params r;
    const uint8_t *b = reinterpret_cast<const uint8_t *>(p);
    uint8_t *o = reinterpret_cast<uint8_t *>(&r);
#pragma unroll
    for (int i = 0; i < 7; i++) o[i] = __ldcg(b + i);
    return r;
}

// Bounded wait of lane 0 until progress[row] >= need; returns false on abort.
__device__ bool wait_row(const FrameArgs &a, const int *progress, int row, int need)
{
    bool ok = true;
    if ((threadIdx.x & 31) == 0) {
        const unsigned long long t0 = globaltimer_ns();
        while (ld_acquire(&progress[row]) < need) {
            if (*(volatile int *)a.error) { ok = false; break; }
            if ((long long)(globaltimer_ns() - t0) > a.timeout_ns) {
                atomicCAS(a.error, 0, EVXG_ERROR_OPERATION_TIMEDOUT);
                ok = false;
                break;
            }
            __nanosleep(64);
        }
    }
    return __shfl_sync(0xffffffffu, ok, 0);
}

// ---- merge decisions (sao.cpp:559-586) ----
// One warp per MB row in a wavefront: MB (r, c) needs the final parameters of
// (r-1, c) and (r, c-1).  Merge costs read the deblocked, not yet filtered
// frame, which does not change during this kernel, so each warp prefetches
// the next MB's tile (recon rows y0-1..y0+16, columns x0-2..x0+17, and the
// source block) into registers while it waits for the row above.
constexpr int MT_W = 20, MT_H = 18;   // recon tile, 10 words per row
struct MergeTile {
    int16_t rec[MT_H * MT_W];
    int16_t src[256];
};
struct TileRegs {
    unsigned r[6], s[4];
};

__device__ __forceinline__ void tile_load(const FrameArgs &a, int c, int row, int lane, TileRegs &t)
{
    const int16_t *rec = a.planes[a.dpb];
    const int x0 = c * 16 - 2, y0 = row * 16 - 1;
#pragma unroll
    for (int i = 0; i < 6; i++) {   // 180 words of the recon tile
        const int wi = lane + 32 * i;
        if (wi < MT_H * MT_W / 2) {
            const int ty = wi / (MT_W / 2), tx = 2 * (wi % (MT_W / 2));
            const int y = min(max(y0 + ty, 0), a.H - 1), x = min(max(x0 + tx, 0), a.W - 2);
            t.r[i] = __ldg(reinterpret_cast<const unsigned *>(rec + (size_t)y * a.W + x));
        }
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {   // 128 words of the source block
        const int wi = lane + 32 * i;
        const int ty = wi >> 3, tx = 2 * (wi & 7);
        t.s[i] = __ldg(reinterpret_cast<const unsigned *>(a.src + (size_t)(row * 16 + ty) * a.W + c * 16 + tx));
    }
}
__device__ __forceinline__ void tile_store(MergeTile &m, int lane, const TileRegs &t)
{
#pragma unroll
    for (int i = 0; i < 6; i++) {
        const int wi = lane + 32 * i;
        if (wi < MT_H * MT_W / 2) reinterpret_cast<unsigned *>(m.rec)[wi] = t.r[i];
    }
#pragma unroll
    for (int i = 0; i < 4; i++) reinterpret_cast<unsigned *>(m.src)[lane + 32 * i] = t.s[i];
}
// Luma SSD of the tile's MB under p, one warp (sao.cpp:346-387 without the rate).
__device__ long long tile_sao_ssd(const FrameArgs &a, const MergeTile &m, int c, int row, int lane, const evxg_sao_params &p)
{
    const int ty = lane >> 1, tx0 = (lane & 1) * 8;
    const int y = row * 16 + ty;
    long long acc = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int tx = tx0 + i, x = c * 16 + tx;
        const int v = m.rec[(ty + 1) * MT_W + tx + 2];
        int corr = v;
        if (p.type == 2) {
            const int idx = (sclamp(v) >> 3) - p.band_position;
            if (idx >= 0 && idx < 4) corr = sclamp(v + p.offsets[idx]);
        } else if (p.type == 1) {
            const int dxa = c_eo[p.eo_class][0], dya = c_eo[p.eo_class][1], dxb = c_eo[p.eo_class][2], dyb = c_eo[p.eo_class][3];
            const int ax = x + dxa, ay = y + dya, bx = x + dxb, by = y + dyb;
            if (ax >= 0 && ax < a.W && ay >= 0 && ay < a.H && bx >= 0 && bx < a.W && by >= 0 && by < a.H) {
                const int ct = eo_cat(v, m.rec[(ty + 1 + dya) * MT_W + tx + 2 + dxa], m.rec[(ty + 1 + dyb) * MT_W + tx + 2 + dxb]);
                if (ct < 4) corr = sclamp(v + p.offsets[ct]);
            }
        }
        const int d = m.src[ty * 16 + tx] - corr;
        acc += (long long)(d * d);
    }
    return warp_sum64(acc);
}
__device__ __forceinline__ evxg_sao_info ld_info_cg(const evxg_sao_info *p)
{
    const uint4 v = __ldcg(reinterpret_cast<const uint4 *>(p));
    evxg_sao_info r;
    memcpy(&r, &v, sizeof r);
    return r;
}

// Final parameters travel between rows in one tagged 64-bit word per MB:
// 25 bits per plane (type, class, band position, four offsets + 8) and the
// frame epoch in the low byte, so a waiting row polls the word it needs.
__device__ __forceinline__ unsigned long long pack_params(const evxg_sao_params &p)
{
    unsigned long long v = (unsigned long long)p.type | ((unsigned long long)p.eo_class << 2) |
                           ((unsigned long long)p.band_position << 4);
    for (int i = 0; i < 4; i++) v |= (unsigned long long)(p.offsets[i] + 8) << (9 + 4 * i);
    return v;
}
__device__ __forceinline__ evxg_sao_params unpack_params(unsigned long long v)
{
    evxg_sao_params p;
    p.type = (uint8_t)(v & 3); p.eo_class = (uint8_t)((v >> 2) & 3); p.band_position = (uint8_t)((v >> 4) & 31);
    for (int i = 0; i < 4; i++) p.offsets[i] = (int8_t)((int)((v >> (9 + 4 * i)) & 15) - 8);
    return p;
}

__device__ __forceinline__ void sao_merge_body(const FrameArgs &a, MergeTile (&tiles)[8][2])
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned long long ep = (unsigned long long)a.epoch;
    for (;;) {
        int row = 0;
        if (lane == 0) row = atomicAdd(&a.counters[1], 1);
        row = __shfl_sync(0xffffffffu, row, 0);
        if (row >= a.mbh) return;
        TileRegs t;
        tile_load(a, 0, row, lane, t);
        tile_store(tiles[w][0], lane, t);
        evxg_sao_info own = ld_info_cg(&a.sao[row * a.mbw]);
        float own_cost = __ldcg(&a.sao_cost[row * a.mbw]);
        evxg_sao_info left{};
        for (int c = 0; c < a.mbw; c++) {
            const int m = row * a.mbw + c;
            evxg_sao_info info = own;   // own RDO parameters, prefetched
            float cur = own_cost;
            if (c + 1 < a.mbw) {        // next MB's data is in flight while this one waits
                tile_load(a, c + 1, row, lane, t);
                own = ld_info_cg(&a.sao[m + 1]);
                own_cost = __ldcg(&a.sao_cost[m + 1]);
            }
            unsigned long long above = 0;
            if (row > 0) {   // bounded wait for the final parameters of (r-1, c)
                bool ok = true;
                if (lane == 0) {
                    const unsigned long long t0 = globaltimer_ns();
                    for (;;) {
                        above = ld_acquire64(&a.sao_mail[m - a.mbw]);
                        if ((above & 0xFF) == ep) break;
                        if (*(volatile int *)a.error) { ok = false; break; }
                        if ((long long)(globaltimer_ns() - t0) > a.timeout_ns) {
                            atomicCAS(a.error, 0, EVXG_ERROR_OPERATION_TIMEDOUT);
                            ok = false;
                            break;
                        }
                    }
                }
                if (!__shfl_sync(0xffffffffu, ok, 0)) return;
                above = __shfl_sync(0xffffffffu, above, 0);
            }
            __syncwarp();
            const MergeTile &mt = tiles[w][c & 1];
            if (c > 0 && left.luma.type != 0) {
                const float mc = __fadd_rn(__ll2float_rn(tile_sao_ssd(a, mt, c, row, lane, left.luma)), __fmul_rn(a.lambda, 1.0f));
                if (mc < cur) { info.merge_left = 1; info.luma = left.luma; info.chroma = left.chroma; cur = mc; }
            }
            if (!info.merge_left && row > 0) {
                const evxg_sao_params al = unpack_params(above >> 8), ac = unpack_params(above >> 33);
                if (al.type != 0) {
                    const float mc = __fadd_rn(__ll2float_rn(tile_sao_ssd(a, mt, c, row, lane, al)), __fmul_rn(a.lambda, 1.0f));
                    if (mc < cur) { info.merge_above = 1; info.luma = al; info.chroma = ac; }
                }
            }
            left = info;
            if (lane == 0) {
                *reinterpret_cast<uint4 *>(&a.sao[m]) = *reinterpret_cast<const uint4 *>(&info);
                st_release64(&a.sao_mail[m], ep | (pack_params(info.luma) << 8) | (pack_params(info.chroma) << 33));
            }
            __syncwarp();
            if (c + 1 < a.mbw) tile_store(tiles[w][(c + 1) & 1], lane, t);
        }
    }
}
__global__ void __launch_bounds__(256) k_sao_merge(FrameArgs a)
{
    __shared__ MergeTile tiles[8][2];
    sao_merge_body(a, tiles);
}
__global__ void __launch_bounds__(256) k_sao_merge_b(const FrameArgs *args)
{
    __shared__ MergeTile tiles[8][2];
    __shared__ FrameArgs sa;
    if (const FrameArgs *a = batch_args(args, sa)) sao_merge_body(*a, tiles);
}

// ---- application (sao.cpp:99-146) ----
// The reference applies offsets MB by MB in raster order, in place: a pixel's
// edge class reads its own MB's and raster-later MBs' pixels unfiltered and
// raster-earlier MBs' pixels already filtered.  Writing F for that rule, the
// filtered frame is the unique fixed point x = F(x) (every dependency points
// to an earlier MB, so there are no cycles), and the dependency chains are a
// few pixels long: they only pass through MB borders.  k_sao_fix evaluates F
// for every pixel in parallel, in place, reading unfiltered values from the
// pristine copy a.sao_orig and earlier MBs' values from the frame itself, and
// flags any change; once a pass changes nothing the frame is exactly x = F(x).
// Passes after a quiet pass return at once; if the last pass still changed a
// pixel, k_sao_restore and k_sao_apply redo the frame in raster wavefront order.
__device__ __forceinline__ void sao_fix_body(const FrameArgs &a, int pass)
{
    if (pass > 0 && __ldcg(&a.sao_flags[pass - 1]) == 0) return;
    const int cw = a.W / 2, ch = a.H / 2;
    const size_t ny = (size_t)a.W * a.H, nc = (size_t)cw * ch;
    bool changed = false;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < ny + 2 * nc; i += (size_t)gridDim.x * blockDim.x) {
        const int pl = i < ny ? 0 : (i < ny + nc ? 1 : 2);
        const size_t k = pl == 0 ? i : (pl == 1 ? i - ny : i - ny - nc);
        const int w = pl ? cw : a.W, h = pl ? ch : a.H, n = pl ? 8 : 16;
        const int y = (int)(k / w), x = (int)(k % w);
        const int m = (y / n) * a.mbw + x / n;
        const evxg_sao_params p = pl ? a.sao[m].chroma : a.sao[m].luma;
        if (p.type == 0) continue;
        const size_t off = pl == 0 ? 0 : (pl == 1 ? ny : ny + nc);
        const int16_t *orig = a.sao_orig + off;
        int16_t *img = a.planes[a.dpb] + off;
        const int v = orig[k];
        int corr = v;
        if (p.type == 2) {
            const int idx = (sclamp(v) >> 3) - p.band_position;
            if (idx >= 0 && idx < 4) corr = sclamp(v + p.offsets[idx]);
        } else {
            const int ax = x + c_eo[p.eo_class][0], ay = y + c_eo[p.eo_class][1];
            const int bx = x + c_eo[p.eo_class][2], by = y + c_eo[p.eo_class][3];
            if (ax >= 0 && ax < w && ay >= 0 && ay < h && bx >= 0 && bx < w && by >= 0 && by < h) {
                const int ma = (ay / n) * a.mbw + ax / n, mb = (by / n) * a.mbw + bx / n;
                const size_t ka = (size_t)ay * w + ax, kb = (size_t)by * w + bx;
                const int va = ma < m ? __ldcg(img + ka) : orig[ka];
                const int vb = mb < m ? __ldcg(img + kb) : orig[kb];
                const int ct = eo_cat(v, va, vb);
                if (ct < 4) corr = sclamp(v + p.offsets[ct]);
            }
        }
        if (__ldcg(img + k) != corr) {
            img[k] = (int16_t)corr;
            changed = true;
        }
    }
    if (__any_sync(0xffffffffu, changed) && (threadIdx.x & 31) == 0) atomicOr(&a.sao_flags[pass], 1);
}
__global__ void __launch_bounds__(256) k_sao_fix(FrameArgs a, int pass) { sao_fix_body(a, pass); }
__global__ void __launch_bounds__(256) k_sao_fix_b(const FrameArgs *args, int pass)
{
    __shared__ FrameArgs sa;
    if (const FrameArgs *a = batch_args(args, sa)) sao_fix_body(*a, pass);
}

// Fallback when the fixed point was not reached within the pass budget:
// restore the unfiltered frame, then the raster wavefront below.
__device__ __forceinline__ void sao_restore_body(const FrameArgs &a, int last_pass)
{
    if (__ldcg(&a.sao_flags[last_pass]) == 0) return;
    const size_t n = (size_t)a.W * a.H + 2 * (size_t)(a.W / 2) * (a.H / 2);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        a.planes[a.dpb][i] = a.sao_orig[i];
}
__global__ void k_sao_restore(FrameArgs a, int last_pass) { sao_restore_body(a, last_pass); }
__global__ void k_sao_restore_b(const FrameArgs *args, int last_pass)
{
    __shared__ FrameArgs sa;
    if (const FrameArgs *a = batch_args(args, sa)) sao_restore_body(*a, last_pass);
}

// In-place application in raster order, one warp per MB row: MB (r, c) runs
// after (r-1, c+1) and before anything of row r+1 at columns >= c-1.  Runs
// only when the fixed-point passes did not converge.
__device__ __forceinline__ void sao_apply_body(const FrameArgs &a, int last_pass)
{
    if (__ldcg(&a.sao_flags[last_pass]) == 0) return;

    const int lane = threadIdx.x & 31;
    int *progress = a.progress + 2 * a.mbh;
    int16_t *Y = a.planes[a.dpb], *U = Y + (size_t)a.W * a.H, *V = U + (size_t)(a.W / 2) * (a.H / 2);
    const int cw = a.W / 2, ch = a.H / 2;
    for (;;) {
        int row = 0;
        if (lane == 0) row = atomicAdd(&a.counters[2], 1);
        row = __shfl_sync(0xffffffffu, row, 0);
        if (row >= a.mbh) return;
        for (int c = 0; c < a.mbw; c++) {
            if (row > 0 && !wait_row(a, progress, row - 1, min(c + 1, a.mbw - 1))) return;
            const int m = row * a.mbw + c;
            const evxg_sao_params lp = ld_params_cg(&a.sao[m].luma), cp = ld_params_cg(&a.sao[m].chroma);
            int nv[8], cu[2], cv[2];
            const int y = row * 16 + (lane >> 1), x0 = c * 16 + (lane & 1) * 8;
            if (lp.type) for (int i = 0; i < 8; i++) nv[i] = sao_px<true>(Y, a.W, a.H, x0 + i, y, lp);
            const int cy = row * 8 + (lane >> 2), cx0 = c * 8 + (lane & 3) * 2;
            if (cp.type)
                for (int i = 0; i < 2; i++) {
                    cu[i] = sao_px<true>(U, cw, ch, cx0 + i, cy, cp);
                    cv[i] = sao_px<true>(V, cw, ch, cx0 + i, cy, cp);
                }
            __syncwarp();
            if (lp.type) for (int i = 0; i < 8; i++) Y[(size_t)y * a.W + x0 + i] = (int16_t)nv[i];
            if (cp.type)
                for (int i = 0; i < 2; i++) {
                    U[(size_t)cy * cw + cx0 + i] = (int16_t)cu[i];
                    V[(size_t)cy * cw + cx0 + i] = (int16_t)cv[i];
                }
            __threadfence();
            __syncwarp();
            if (lane == 0) st_release(&progress[row], c);
            __syncwarp();
        }
    }
}
__global__ void k_sao_apply(FrameArgs a, int last_pass) { sao_apply_body(a, last_pass); }
__global__ void k_sao_apply_b(const FrameArgs *args, int last_pass)
{
    __shared__ FrameArgs sa;
    if (const FrameArgs *a = batch_args(args, sa)) sao_apply_body(*a, last_pass);
}

// ------------------------------------------- batched-tick bookkeeping
// In a batched tick these kernels do, for every stream with a frame, what
// the single path does with copies and memsets around its kernels.
__device__ __forceinline__ void copy_words(int *to, const int *from, size_t n, size_t t, size_t step)
{
    for (size_t i = t; i < n; i += step) to[i] = __ldg(from + i);
}
// Before the frame: the serializer's snapshot of the previous table
// (encode.cpp:985-998 serializes before the update), wavefront progress words
// to -1, row counters and SAO pass flags to 0.
__global__ void k_tick_prep_b(const FrameArgs *args, int sao_passes)
{
    __shared__ FrameArgs sa;
    const FrameArgs *a = batch_args(args, sa);
    if (!a) return;
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x, step = (size_t)gridDim.x * blockDim.x;
    const size_t nblk = (size_t)a->mbw * a->mbh;
    copy_words(reinterpret_cast<int *>(a->prev_ser), reinterpret_cast<const int *>(a->prev_tab), nblk * 7, t, step);
    for (size_t i = t; i < 3 * (size_t)a->mbh; i += step) a->progress[i] = -1;
    if (t < 4) a->counters[t] = 0;
    if (t < (size_t)sao_passes) a->sao_flags[t] = 0;
}
// After deblocking: the pristine copy the SAO fixed-point passes read.
__global__ void k_sao_copy_b(const FrameArgs *args)
{
    __shared__ FrameArgs sa;
    const FrameArgs *a = batch_args(args, sa);
    if (!a) return;
    const uint4 *from = reinterpret_cast<const uint4 *>(a->planes[a->dpb]);
    uint4 *to = reinterpret_cast<uint4 *>(a->sao_orig);
    const size_t n = a->plane_elems / 8;   // plane sets are whole 16-byte chunks (16-aligned sizes)
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        to[i] = __ldcg(from + i);
}
// After the frame: the temporal predictor table of the next P frame is this
// frame's table, except after B frames (encode.cpp:990-998).
__global__ void k_tick_post_b(const FrameArgs *args)
{
    __shared__ FrameArgs sa;
    const FrameArgs *a = batch_args(args, sa);
    if (!a || a->type == EVXG_FRAME_BIDIR) return;
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x, step = (size_t)gridDim.x * blockDim.x;
    copy_words(reinterpret_cast<int *>(a->prev_tab), reinterpret_cast<const int *>(a->bt), (size_t)a->mbw * a->mbh * 7, t, step);
}

}  // namespace evxg
