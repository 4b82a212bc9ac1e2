// evxg_filters.cu -- frame-level kernels of the EVX3 encoder pipeline on sm_100a:
// RGB24 -> YUV 4:2:0 conversion, in-loop deblocking and SAO (RDO, merge and
// raster-order application).
//
// Reference: src/video/convert.cpp:11-160, src/video/deblock.cpp:14-305,
// src/video/sao.cpp:13-594 (luma-only merge branch, EVX_ENABLE_SAO_CHROMA_MERGE 0).
#include "evxg_internal.cuh"

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

// Filter one line across an edge (deblock.cpp:91-146); tap(k) is the sample
// k places from q0 (p0 = tap(-1), q0 = tap(0)).
template <class Tap>
__device__ __forceinline__ void filter_taps(Tap tap, int qe, int st, bool luma)
{
    const int p0 = tap(-1), p1 = tap(-2), p2 = tap(-3), p3 = tap(-4);
    const int q0 = tap(0), q1 = tap(1), q2 = tap(2), q3 = tap(3);
    int qi = qe;
    if (st == 2 && qe > 0) qi = min(qe + 2, MAXQ);
    if ((int16_t)iabs32(p0 - q0) >= c_alpha[qi] || (int16_t)iabs32(p1 - p0) >= c_beta[qi] ||
        (int16_t)iabs32(q1 - q0) >= c_beta[qi])
        return;
    if (st == 2) {
        tap(-1) = (int16_t)rdiv(p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1, 8);
        tap(-2) = (int16_t)rdiv(p2 + p1 + p0 + q0, 4);
        tap(0) = (int16_t)rdiv(p1 + 2 * p0 + 2 * q0 + 2 * q1 + q2, 8);
        tap(1) = (int16_t)rdiv(p0 + q0 + q1 + q2, 4);
        if (luma) {
            tap(-3) = (int16_t)rdiv(2 * p3 + 3 * p2 + p1 + p0 + q0, 8);
            tap(2) = (int16_t)rdiv(2 * q3 + 3 * q2 + q1 + q0 + p0, 8);
        }
    } else {
        tap(-1) = (int16_t)rdiv(((q0 + p0) * 4) + p1 - q1, 8);
        tap(0) = (int16_t)rdiv(((q0 + p0) * 4) + q1 - p1, 8);
        if (luma) {
            tap(-2) = (int16_t)rdiv((p2 * 4) + (p0 * 2) + (q0 * 2), 8);
            tap(1) = (int16_t)rdiv((q2 * 4) + (q0 * 2) + (p0 * 2), 8);
        }
    }
}
// e points at q0, step is the distance between samples.
__device__ __forceinline__ void filter_line(int16_t *e, int step, int qe, int st, bool luma)
{
    filter_taps([&](int k) -> int16_t & { return e[k * step]; }, qe, st, luma);
}

// One CTA per plane.  The reference's order (deblock.cpp:233-272) is: row band
// 0 vertical edges; then per 8-row band j the horizontal edge at x=0 and, for
// x = 8, 16, ..., the horizontal edge (x, j) followed by the vertical edge
// (x, j).  Within a band, horizontal edges touch disjoint columns and vertical
// edge (x, j) only reads columns written by horizontal edges (x-8, j) and
// (x, j), so running all horizontal edges of the band and then all vertical
// edges gives the same samples; bands stay in order.
__device__ __forceinline__ void deblock_body(const FrameArgs &a, int pl)
{
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
// The same order on eight column strips per plane, one CTA each, in one
// cluster.  A strip keeps its columns of the plane in a circular window of
// DB_SLOTS rows in shared memory; the next band's rows are read into
// registers while the current band is filtered, and a row goes back to memory
// once no later edge touches it -- after band j every row up to j+4 is final
// (later horizontal edges start at row j+8-3, vertical ones at row j+8).  The
// slots the next band takes held rows written back at least a band ago.
// Horizontal edges touch only their own columns.  A strip owns the vertical
// edges at its columns; the first of them reads and writes the four columns
// left of the strip, which live in the window of the strip that holds them,
// through distributed shared memory.  Cluster barriers give the band's order:
// every strip's horizontal edges, then every strip's vertical edges, then the
// next band.
constexpr int DB_SLOTS = 24, DB_STRIPS = 8, DB_THREADS = 256;
constexpr int DB_MAXW = 2048;   // widest strip (columns) that goes through shared memory
__device__ __forceinline__ int db_slot(int r) { return (r + DB_SLOTS) % DB_SLOTS; }
__host__ __device__ __forceinline__ int db_x0(int w, int s) { return ((s * (w / 8)) / DB_STRIPS) * 8; }
__host__ __device__ __forceinline__ bool deblock_fits(int W) { return db_x0(W, 1) <= DB_MAXW && W - db_x0(W, DB_STRIPS - 1) <= DB_MAXW; }
size_t deblock_shared_bytes(int W)   // the luma plane has the widest strips
{
    int wmax = 0;
    for (int s = 0; s < DB_STRIPS; s++) wmax = max(wmax, (s + 1 < DB_STRIPS ? db_x0(W, s + 1) : W) - db_x0(W, s));
    return deblock_fits(W) ? (size_t)DB_SLOTS * wmax * sizeof(int16_t) : 0;
}
__device__ __forceinline__ unsigned db_rank()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void db_cluster_barrier()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ int16_t *db_peer(int16_t *p, unsigned rank)
{
    int16_t *r;
    asm volatile("mapa.u64 %0, %1, %2;" : "=l"(r) : "l"(p), "r"(rank));
    return r;
}
// Deblocking beside the macroblock pass (a.db_wait): before a strip reads
// plane rows up to y, its thread 0 waits (bounded) until the wavefront has
// finished the macroblock row holding y -- rows finish in order.  After a
// wait that gave up (error word set) the strip stops waiting but keeps
// step with its cluster's barriers, so every CTA still reaches its end.
__device__ void db_wait(const FrameArgs &a, int y, int mbs, bool &live)
{
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        int ok = live;
        const int r = min(y / mbs, a.mbh - 1);
        if (ok) {
            const unsigned long long t0 = globaltimer_ns();
            while (ld_acquire(&a.progress[r]) < a.mbw - 1) {
                if (*(volatile int *)a.error || (long long)(globaltimer_ns() - t0) > a.timeout_ns) {
                    atomicCAS(a.error, 0, EVXG_ERROR_OPERATION_TIMEDOUT);
                    ok = 0;
                    break;
                }
                __nanosleep(128);
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    live = s_ok != 0;
    __syncthreads();   // s_ok is rewritten by the next wait
}
__device__ void deblock_strip_body(const FrameArgs &a, int16_t *buf)
{
    const int pl = blockIdx.x / DB_STRIPS, sid = (int)db_rank();
    const bool luma = pl == 0;
    const int w = luma ? a.W : a.W / 2, h = luma ? a.H : a.H / 2;
    const int mbs = luma ? 16 : 8, qoff = luma ? 0 : 2;
    const size_t poff = pl == 0 ? 0 : (size_t)a.W * a.H + (pl - 1) * (size_t)(a.W / 2) * (a.H / 2);
    const int16_t *d = a.planes[a.dpb] + poff;           // reconstruction read
    int16_t *o = (a.db_out ? a.db_out : a.planes[a.dpb]) + poff;   // filtered rows written
    bool live = true;
    const int xs = db_x0(w, sid), xe = sid + 1 < DB_STRIPS ? db_x0(w, sid + 1) : w;
    const int sw = xe - xs, cpr = sw / 8;   // strip width, 16-byte chunks per strip row
    // the strip holding columns xs-4 .. xs-1 (strips are multiples of 8 wide; empty ones hold nothing)
    int ls = sid - 1;
    while (ls >= 0 && db_x0(w, ls) >= xs) ls--;
    int16_t *lbuf = nullptr;
    int lw = 0, lx = 0;
    if (ls >= 0 && sw > 0) {
        lx = db_x0(w, ls);
        lw = db_x0(w, ls + 1) - lx;
        lbuf = db_peer(buf, (unsigned)ls);
    }
    const int nvx = sw / 8 - (xs == 0 ? 1 : 0);   // vertical edges owned: x = xs (if > 0), xs + 8, ...
    const int xv0 = xs == 0 ? 8 : xs;
    const int tid = threadIdx.x, nt = blockDim.x;
    if (a.db_wait) db_wait(a, min(7, h - 1), mbs, live);
    for (int i = tid; i < 8 * cpr; i += nt) {   // band 0
        const int r = i / cpr, c = i % cpr;
        *reinterpret_cast<uint4 *>(buf + db_slot(r) * sw + 8 * c) = __ldcg(reinterpret_cast<const uint4 *>(d + (size_t)r * w + xs + 8 * c));
    }
    db_cluster_barrier();
    int written = 0;   // rows [0, written) of the strip are back in the slot
    for (int j = 0; j < h; j += 8) {
        const bool more = j + 8 < h;
        if (more && a.db_wait) db_wait(a, min(j + 15, h - 1), mbs, live);
        constexpr int PF = DB_MAXW / DB_THREADS;   // next band: at most 8 rows x 256 chunks
        uint4 pf[PF];
#pragma unroll
        for (int k = 0; k < PF; k++) {
            const int i = tid + k * nt;
            if (more && i < 8 * cpr)
                pf[k] = __ldcg(reinterpret_cast<const uint4 *>(d + (size_t)(j + 8 + i / cpr) * w + xs + 8 * (i % cpr)));
        }
        if (j > 0) {   // horizontal edges at row j, own columns
            const int brow = (j / mbs) * a.mbw, arow = ((j - 1) / mbs) * a.mbw;
            int ro[8];
#pragma unroll
            for (int k = 0; k < 8; k++) ro[k] = db_slot(j - 4 + k) * sw;
            for (int c = tid; c < sw; c += nt) {
                const int x = xs + c;
                int qe, st;
                edge_params(a.bt, x / mbs + arow, x / mbs + brow, qoff, qe, st);
                if (st) filter_taps([&](int k) -> int16_t & { return buf[ro[k + 4] + c]; }, qe, st, luma);
            }
            db_cluster_barrier();
        }
        const int brow = (j / mbs) * a.mbw;
        for (int t = tid; t < nvx * 8; t += nt) {   // vertical edges of the band, own
            const int x = xv0 + (t >> 3) * 8, y = j + (t & 7), c = x - xs;
            int qe, st;
            edge_params(a.bt, (x - 1) / mbs + brow, x / mbs + brow, qoff, qe, st);
            if (!st) continue;
            int16_t *row = buf + db_slot(y) * sw;
            if (c >= 4) {
                filter_line(row + c, 1, qe, st, luma);
            } else {   // the strip's first edge: its left taps are in the strip holding them
                int16_t *lrow = lbuf + db_slot(y) * lw + (xs - lx);
                filter_taps([&](int k) -> int16_t & { return k < 0 ? lrow[k] : row[c + k]; }, qe, st, luma);
            }
        }
        db_cluster_barrier();
        const int upto = more ? j + 5 : h;
        for (int i = tid; i < (upto - written) * cpr; i += nt) {
            const int r = written + i / cpr, c = i % cpr;
            *reinterpret_cast<uint4 *>(o + (size_t)r * w + xs + 8 * c) = *reinterpret_cast<const uint4 *>(buf + db_slot(r) * sw + 8 * c);
        }
        written = upto;
#pragma unroll
        for (int k = 0; k < PF; k++) {
            const int i = tid + k * nt;
            if (more && i < 8 * cpr) *reinterpret_cast<uint4 *>(buf + db_slot(j + 8 + i / cpr) * sw + 8 * (i % cpr)) = pf[k];
        }
        __syncthreads();
    }
    db_cluster_barrier();   // no strip leaves while a neighbour may still use its window
}
__global__ void __cluster_dims__(DB_STRIPS, 1, 1) __launch_bounds__(DB_THREADS) k_deblock(FrameArgs a)
{
    extern __shared__ __align__(16) int16_t db_smem[];
    if (deblock_fits(a.W)) {
        deblock_strip_body(a, db_smem);
    } else if (blockIdx.x % DB_STRIPS == 0) {   // very wide planes: one CTA per plane, in place in memory
        deblock_body(a, blockIdx.x / DB_STRIPS);
    }
}
__global__ void __cluster_dims__(DB_STRIPS, 1, 1) __launch_bounds__(DB_THREADS) k_deblock_b(const FrameArgs *args)
{
    extern __shared__ __align__(16) int16_t db_smem[];
    __shared__ FrameArgs sa;
    const FrameArgs *a = batch_args(args, sa);   // a cluster is one stream and plane: active or not for all its CTAs
    if (!a) return;
    if (deblock_fits(a->W)) deblock_strip_body(*a, db_smem);
    else if (blockIdx.x % DB_STRIPS == 0) deblock_body(*a, blockIdx.x / DB_STRIPS);
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

// Per-warp scratch of the SAO RDO.
struct SaoScratch {
    int bsum[32], bcnt[32], boff[32];
    unsigned long long bdelta[32];   // signed sums, two's complement
};

// Per-MB RDO of one N x N plane block (sao.cpp:150-343) on one warp; returns
// the parameters and the SSD they give.  Lane l holds N*N/32 consecutive
// pixels of one row and the recon samples around them.  The candidates are
// costed independently (no SAO, band offsets at positions 0..28, edge
// offsets of classes 0..3) and the reference's loop -- take a candidate when
// it is strictly cheaper than the best so far -- picks the first candidate of
// that order whose cost is the minimum, which a (cost, index) argmin finds.
// All sums are of integers, so regrouping them changes nothing.  With stats
// set (luma), the band and edge-category sums and counts, the SSD without SAO
// and the out-of-range flag are stored for the merge costs (kSaoStatEntries).
template <int N>
__device__ void sao_rdo_warp(const int16_t *s, const int16_t *r, int w, int h, int x0, int y0, float lambda, int lane,
                             SaoScratch &sc, evxg_sao_params &out, long long &out_ssd, int2 *stats = nullptr)
{
    constexpr int P = N * N / 32;   // pixels per lane: 8 (luma) or 2 (chroma)
    const int y = y0 + lane * P / N, xs = x0 + (lane * P) % N;
    int pv[P], sv[P], nb[3][P + 2];
#pragma unroll
    for (int i = 0; i < P; i++) {
        pv[i] = __ldg(r + (size_t)y * w + xs + i);
        sv[i] = __ldg(s + (size_t)y * w + xs + i);
    }
#pragma unroll
    for (int dy = 0; dy < 3; dy++)
#pragma unroll
        for (int dx = 0; dx < P + 2; dx++) {
            const int yy = y - 1 + dy, xx = xs - 1 + dx;
            nb[dy][dx] = (yy >= 0 && yy < h && xx >= 0 && xx < w) ? __ldg(r + (size_t)yy * w + xx) : 0;
        }
    sc.bsum[lane] = 0; sc.bcnt[lane] = 0; sc.bdelta[lane] = 0;
    __syncwarp();
    long long base = 0;
#pragma unroll
    for (int i = 0; i < P; i++) {
        const int d = sv[i] - pv[i], b = sclamp(pv[i]) >> 3;
        base += (long long)(d * d);
        atomicAdd(&sc.bsum[b], d);
        atomicAdd(&sc.bcnt[b], 1);
    }
    base = warp_sum64(base);
    __syncwarp();
    if (stats) {   // band b's samples lie in [8b, 8b+7]: only bands 0 and 31 need their extremes
        bool out = false;
        int mn0 = 255, mx31 = 0;
#pragma unroll
        for (int i = 0; i < P; i++) {
            out |= pv[i] < 0 || pv[i] > 255;
            const int b = sclamp(pv[i]) >> 3;
            if (b == 0) mn0 = min(mn0, pv[i]);
            if (b == 31) mx31 = max(mx31, pv[i]);
        }
        out = __any_sync(0xffffffffu, out);
        mn0 = __reduce_min_sync(0xffffffffu, mn0);
        mx31 = __reduce_max_sync(0xffffffffu, mx31);
        const int lo = lane == 0 ? mn0 : 8 * lane, hi = lane == 31 ? mx31 : 8 * lane + 7;
        stats[lane] = make_int2(sc.bsum[lane], sc.bcnt[lane] | (lo & 255) << 9 | (hi & 255) << 17);
        if (lane == 0) stats[48] = make_int2((int)base, out ? 1 : 0);
    }
    // band offsets: lane b owns band b (its offset does not depend on the band position)
    sc.boff[lane] = sc.bcnt[lane] > 0 ? avg_off(sc.bsum[lane], sc.bcnt[lane]) : 0;
    __syncwarp();
#pragma unroll
    for (int i = 0; i < P; i++) {
        const int d = sv[i] - pv[i], b = sclamp(pv[i]) >> 3, cv = sclamp(pv[i] + sc.boff[b]), e = sv[i] - cv;
        atomicAdd(&sc.bdelta[b], (unsigned long long)((long long)(e * e) - (long long)(d * d)));
    }
    __syncwarp();
    // candidate costs; index 0 = no SAO, 1 + bp = band position bp, 30 + ec = edge class ec
    float cost = __int_as_float(0x7f800000);   // +inf: not a candidate
    int idx = 64;
    long long ssd_c = 0;
    if (lane <= 28) {
        evxg_sao_params c{};
        c.type = 2; c.band_position = (uint8_t)lane;
        bool nz = false;
        long long ssd = base;
        for (int k = 0; k < 4; k++) {
            c.offsets[k] = (int8_t)sc.boff[lane + k];
            nz |= sc.boff[lane + k] != 0;
            ssd += (long long)sc.bdelta[lane + k];
        }
        if (nz) { cost = rd_cost64(ssd, lambda, sao_bits(c)); idx = 1 + lane; ssd_c = ssd; }
    }
    if (lane == 31) { cost = rd_cost64(base, lambda, 2u); idx = 0; ssd_c = base; }
    // edge classes: category sums per class, reduced over the warp
    int cs[4][4], cc[4][4];
#pragma unroll
    for (int ec = 0; ec < 4; ec++)
#pragma unroll
        for (int k = 0; k < 4; k++) { cs[ec][k] = 0; cc[ec][k] = 0; }
    int cat[4][P];
#pragma unroll
    for (int ec = 0; ec < 4; ec++)
#pragma unroll
        for (int i = 0; i < P; i++) {
            // c_eo as compile-time constants, so the neighbourhood stays in registers
            constexpr int kEo[4][4] = {{-1, 0, 1, 0}, {0, -1, 0, 1}, {-1, -1, 1, 1}, {1, -1, -1, 1}};
            const int dxa = kEo[ec][0], dya = kEo[ec][1], dxb = kEo[ec][2], dyb = kEo[ec][3];
            const int x = xs + i, ax = x + dxa, ay = y + dya, bx = x + dxb, by = y + dyb;
            int ct = 4;
            if (!(ax < 0 || ax >= w || ay < 0 || ay >= h || bx < 0 || bx >= w || by < 0 || by >= h))
                ct = eo_cat(pv[i], nb[1 + dya][1 + i + dxa], nb[1 + dyb][1 + i + dxb]);
            cat[ec][i] = ct;
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (ct == k) { cs[ec][k] += sv[i] - pv[i]; cc[ec][k]++; }
        }
#pragma unroll
    for (int ec = 0; ec < 4; ec++)
#pragma unroll
        for (int k = 0; k < 4; k++) { cs[ec][k] = warp_sum(cs[ec][k]); cc[ec][k] = warp_sum(cc[ec][k]); }
    if (stats) {   // each category's sum, count and sample range
        int2 e = make_int2(0, 0);
#pragma unroll
        for (int ec = 0; ec < 4; ec++)
#pragma unroll
            for (int k = 0; k < 4; k++) {
                int mn = 255, mx = 0;
#pragma unroll
                for (int i = 0; i < P; i++)
                    if (cat[ec][i] == k) { mn = min(mn, pv[i]); mx = max(mx, pv[i]); }
                mn = __reduce_min_sync(0xffffffffu, mn);
                mx = __reduce_max_sync(0xffffffffu, mx);
                if (lane == 4 * ec + k) e = make_int2(cs[ec][k], cc[ec][k] | (mn & 255) << 9 | (mx & 255) << 17);
            }
        if (lane < 16) stats[32 + lane] = e;
    }
    long long eo_ssd[4];
    bool eo_nz[4];
    int off[4][4];
#pragma unroll
    for (int ec = 0; ec < 4; ec++) {
        eo_nz[ec] = false;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            off[ec][k] = cc[ec][k] > 0 ? avg_off(cs[ec][k], cc[ec][k]) : 0;
            eo_nz[ec] |= off[ec][k] != 0;
        }
        long long dl = 0;
#pragma unroll
        for (int i = 0; i < P; i++) {
            const int ct = cat[ec][i];
            if (ct < 4) {
                int o = 0;
#pragma unroll
                for (int k = 0; k < 4; k++) o = ct == k ? off[ec][k] : o;
                const int d = sv[i] - pv[i], e = sv[i] - sclamp(pv[i] + o);
                dl += (long long)(e * e) - (long long)(d * d);
            }
        }
        eo_ssd[ec] = base + warp_sum64(dl);
    }
    // argmin over (cost, index): bands / none on their lanes, then the four edge classes
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const float c2 = __shfl_xor_sync(0xffffffffu, cost, o);
        const int i2 = __shfl_xor_sync(0xffffffffu, idx, o);
        const long long s2 = __shfl_xor_sync(0xffffffffu, ssd_c, o);
        if (c2 < cost || (c2 == cost && i2 < idx)) { cost = c2; idx = i2; ssd_c = s2; }
    }
#pragma unroll
    for (int ec = 0; ec < 4; ec++) {   // edge candidates come after every band candidate
        if (!eo_nz[ec]) continue;
        evxg_sao_params c{};
        c.type = 1; c.eo_class = (uint8_t)ec;
        for (int k = 0; k < 4; k++) c.offsets[k] = (int8_t)off[ec][k];
        const float ce = rd_cost64(eo_ssd[ec], lambda, sao_bits(c));
        if (ce < cost) { cost = ce; idx = 30 + ec; ssd_c = eo_ssd[ec]; }
    }
    out = evxg_sao_params{};
    if (idx >= 30) {
        out.type = 1; out.eo_class = (uint8_t)(idx - 30);
        for (int k = 0; k < 4; k++) out.offsets[k] = (int8_t)off[idx - 30][k];
    } else if (idx >= 1) {
        out.type = 2; out.band_position = (uint8_t)(idx - 1);
        for (int k = 0; k < 4; k++) out.offsets[k] = (int8_t)sc.boff[idx - 1 + k];
    }
    out_ssd = ssd_c;
    __syncwarp();
}

// One warp per MB: own luma and chroma (U plane) parameters and the cost of
// keeping them, the starting point of the merge decision (sao.cpp:414-557),
// stored with the luma statistics in the MB's record (kSaoStatEntries).
__device__ __forceinline__ void sao_rdo_body(const FrameArgs &a, SaoScratch *scratch)
{
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    const int m = blockIdx.x * (blockDim.x >> 5) + wi;
    if (m >= a.mbw * a.mbh) return;
    const int bx = m % a.mbw, by = m / a.mbw;
    const int16_t *rec = a.planes[a.dpb];
    const int cw = a.W / 2, ch = a.H / 2;
    evxg_sao_info info{};
    long long lssd, cssd;
    sao_rdo_warp<16>(a.src, rec, a.W, a.H, bx * 16, by * 16, a.lambda, lane, scratch[wi], info.luma, lssd,
                     a.sao_stats + (size_t)m * kSaoStatEntries);
    sao_rdo_warp<8>(a.src + (size_t)a.W * a.H, rec + (size_t)a.W * a.H, cw, ch, bx * 8, by * 8, a.lambda, lane, scratch[wi],
                    info.chroma, cssd);
    if (lane == 0) {
        float cur;
        if (info.luma.type == 0) cur = __fadd_rn(__ll2float_rn(lssd), __fmul_rn(a.lambda, 2.0f));
        else cur = __fadd_rn(__fsub_rn(__fadd_rn(__ll2float_rn(lssd), __fmul_rn(a.lambda, 1.0f)), __fmul_rn(a.lambda, 1.0f)),
                             __fmul_rn(a.lambda, __uint2float_rn(sao_bits(info.luma))));
        int2 *r = a.sao_stats + (size_t)m * kSaoStatEntries;
        uint4 w;
        memcpy(&w, &info, sizeof w);
        r[49] = make_int2(__float_as_int(cur), 0);
        *reinterpret_cast<uint4 *>(r + 50) = w;
    }
}
constexpr int SAO_RDO_WARPS = 8;   // MBs per block of the RDO kernels
__global__ void __launch_bounds__(32 * SAO_RDO_WARPS) k_sao_rdo(FrameArgs a)
{
    __shared__ SaoScratch sc[SAO_RDO_WARPS];
    sao_rdo_body(a, sc);
}
__global__ void __launch_bounds__(32 * SAO_RDO_WARPS) k_sao_rdo_b(const FrameArgs *args)
{
    __shared__ SaoScratch sc[SAO_RDO_WARPS];
    __shared__ FrameArgs sa;
    if (const FrameArgs *a = batch_args(args, sa)) sao_rdo_body(*a, sc);
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
// (r-1, c) and (r, c-1).  A merge cost is the luma SSD of the MB under the
// neighbour's parameters plus one bit: from the band and edge-category sums
// k_sao_rdo stored for the MB, or, when those parameters would clamp one of
// the MB's samples, from its tile of the deblocked, not yet filtered frame
// (recon rows y0-1..y0+16, columns x0-2..x0+17, and the source block).
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
// Luma SSD of the tile's MB under p, one warp (sao.cpp:346-387 without the
// rate).  The parameters are unpacked into registers and the band / edge
// branch is taken once per call, not per pixel.
__device__ __forceinline__ int pick4(int k, int o0, int o1, int o2, int o3) { return k == 0 ? o0 : k == 1 ? o1 : k == 2 ? o2 : o3; }
__device__ __forceinline__ long long tile_sao_ssd(int W, int H, const MergeTile &m, int c, int row, int lane,
                                                  evxg_sao_params p)
{
    const int ty = lane >> 1, tx0 = (lane & 1) * 8;
    const int y = row * 16 + ty, x0 = c * 16 + tx0;
    const int o0 = p.offsets[0], o1 = p.offsets[1], o2 = p.offsets[2], o3 = p.offsets[3];
    const int16_t *rr = m.rec + (ty + 1) * MT_W + tx0 + 2;
    const int16_t *sr = m.src + ty * 16 + tx0;
    long long acc = 0;
    if (p.type == 2) {
        const int bp = p.band_position;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int v = rr[i], idx = (sclamp(v) >> 3) - bp;
            const int corr = (idx >= 0 && idx < 4) ? sclamp(v + pick4(idx, o0, o1, o2, o3)) : v;
            const int d = sr[i] - corr;
            acc += (long long)(d * d);
        }
    } else if (p.type == 1) {
        const int ec = p.eo_class;
        const int dxa = ec == 1 ? 0 : (ec == 3 ? 1 : -1), dya = ec == 0 ? 0 : -1;   // c_eo (sao.cpp:20-25)
        const int dxb = -dxa, dyb = -dya;
        const bool rows_ok = y + dya >= 0 && y + dya < H && y + dyb >= 0 && y + dyb < H;
        const int da = dya * MT_W + dxa, db = dyb * MT_W + dxb;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int v = rr[i], x = x0 + i;
            int corr = v;
            if (rows_ok && x + dxa >= 0 && x + dxa < W && x + dxb >= 0 && x + dxb < W) {
                const int ct = eo_cat(v, rr[i + da], rr[i + db]);
                if (ct < 4) corr = sclamp(v + pick4(ct, o0, o1, o2, o3));
            }
            const int d = sr[i] - corr;
            acc += (long long)(d * d);
        }
    } else {
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int d = sr[i] - rr[i];
            acc += (long long)(d * d);
        }
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

// Merge wavefront on one cluster of MERGE_CTAS CTAs per frame: CTA k takes
// the k-th block of rpc = ceil(rows / MERGE_CTAS) consecutive rows, one warp
// per row (a warp takes a second row of its block if the block has more rows
// than warps).  The final parameters of MB (r-1, c) reach row r through an
// epoch-tagged word in shared memory -- an aligned 64-bit store, with no
// fence: the parameters are the word -- and at a block boundary the last
// row stores its words straight into the next CTA's shared memory, so no
// hand-over goes through global memory.  Frames whose words would not fit
// use a.sao_mail for every row.  A CTA's dynamic shared memory holds one
// tile per warp, then one four-record ring per warp, then the words.
constexpr int MERGE_CTAS = kMergeCtas, MERGE_WARPS = kMergeThreads / 32;
constexpr int MERGE_RING = 4;   // MB records in a warp's ring: the one decided and three in flight
constexpr size_t MERGE_WARP_BYTES = sizeof(MergeTile) + MERGE_RING * kSaoStatEntries * sizeof(int2);
constexpr size_t MERGE_SMEM_MAX = 200 * 1024 - MERGE_WARPS * MERGE_WARP_BYTES;   // hand-over words
__host__ __device__ __forceinline__ int merge_rpc(int mbh) { return (mbh + MERGE_CTAS - 1) / MERGE_CTAS; }
__host__ __device__ __forceinline__ size_t merge_words_bytes(int mbw, int mbh) { return (size_t)(merge_rpc(mbh) + 1) * mbw * 8; }
__host__ __device__ __forceinline__ bool merge_words_fit(int mbw, int mbh) { return merge_words_bytes(mbw, mbh) <= MERGE_SMEM_MAX; }
size_t merge_shared_bytes(int mbw, int mbh)   // dynamic shared memory of the merge kernels
{
    return MERGE_WARPS * MERGE_WARP_BYTES + (merge_words_fit(mbw, mbh) ? merge_words_bytes(mbw, mbh) : 0);
}

// Bounded wait of the whole warp for a tagged word: every lane reads the same
// address, so each poll gives all lanes one value and the warp stays
// converged.  The shared-memory form polls cheaply and looks at the error
// word and the clock every 256 polls.
template <bool kShared>
__device__ __forceinline__ bool wait_word(const FrameArgs &a, const unsigned long long *p, unsigned long long ep,
                                          unsigned long long &v)
{
    unsigned long long t0 = 0;
    for (unsigned it = 0;; it++) {
        v = kShared ? *(const volatile unsigned long long *)p : ld_acquire64(p);
        if (__all_sync(0xffffffffu, (v & 0xFF) == ep)) return true;
        if (kShared && (it & 255) != 255) continue;
        bool stop = *(volatile int *)a.error != 0;
        const unsigned long long now = globaltimer_ns();
        if (!t0) {
            t0 = now;
        } else if ((long long)(now - t0) > a.timeout_ns) {
            atomicCAS(a.error, 0, EVXG_ERROR_OPERATION_TIMEDOUT);
            stop = true;
        }
        if (__any_sync(0xffffffffu, stop)) return false;
    }
}

// The record of MB m (kSaoStatEntries, 26 x 16 bytes) into a ring slot, by
// lanes 0..25; one commit group per MB, issued by the whole warp.
__device__ __forceinline__ void merge_fetch(const FrameArgs &a, int2 *slot, int m, int lane)
{
    if (lane < kSaoStatEntries / 2) cp_async16(slot + 2 * lane, a.sao_stats + (size_t)m * kSaoStatEntries + 2 * lane);
}

// Luma SSD of an MB under p from its record r (read alike by every lane): a
// corrected sample v + o adds o^2 - 2 o (s - v) to the SSD without SAO,
// exactly, unless v + o leaves [0, 255], where the correction clamps
// (sao.cpp:40-97); false then, read from the sample ranges of p's entries.
// Every term and the sum stay below 2^24 (256 samples, |s - v| <= 255).
__device__ __forceinline__ bool stat_ssd(const int2 *r, const evxg_sao_params &p, int &ssd)
{
    const bool bo = p.type == 2;
    const int first = bo ? p.band_position : 32 + 4 * p.eo_class, end = bo ? 32 : 48;
    const int2 h = r[48];
    int acc = h.x;
    bool exact = h.y == 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int e = first + k;
        if (e < end) {
            const int2 v = r[e];
            const int o = p.offsets[k], cnt = v.y & 511, lo = (v.y >> 9) & 255, hi = (v.y >> 17) & 255;
            if (cnt) {
                acc += cnt * o * o - 2 * o * v.x;
                exact &= lo + o >= 0 && hi + o <= 255;
            }
        }
    }
    ssd = acc;
    return exact;
}

// One row of merge decisions (sao.cpp:559-586) by one warp, all lanes in
// step; false once a wait gave up.  With shared words: above = this CTA's
// word row i (row i-1 of the block, or for i = 0 the previous block's last
// row), own = word row i+1, and next (if not null) the next CTA's word row
// 0.  The records of the next three MBs are in flight into the ring while one
// MB is decided; a cost the statistics cannot give exactly is taken on the
// MB's tile, loaded then (at most once per MB).
__device__ bool merge_row(const FrameArgs &a, MergeTile &tile, int2 *ring, unsigned long long *words,
                          unsigned long long *next, int i, int row)
{
    const int lane = threadIdx.x & 31;
    const unsigned long long ep = (unsigned long long)a.epoch;
    const int m0 = row * a.mbw;
    for (int k = 0; k < MERGE_RING - 1; k++) {
        if (k < a.mbw) merge_fetch(a, ring + k * kSaoStatEntries, m0 + k, lane);
        cp_async_commit();
    }
    evxg_sao_info left{};
    for (int c = 0; c < a.mbw; c++) {
        const int m = m0 + c;
        if (c + MERGE_RING - 1 < a.mbw)   // into the slot MB c-1 used
            merge_fetch(a, ring + ((c + MERGE_RING - 1) % MERGE_RING) * kSaoStatEntries, m + MERGE_RING - 1, lane);
        cp_async_commit();
        cp_async_wait_group<MERGE_RING - 1>();   // MB c's group has landed
        __syncwarp();
        const int2 *r = ring + (c % MERGE_RING) * kSaoStatEntries;
        evxg_sao_info info;
        const uint4 own = *reinterpret_cast<const uint4 *>(r + 50);
        memcpy(&info, &own, sizeof info);
        float cur = __int_as_float(r[49].x);
        bool have_tile = false;
        auto cost = [&](const evxg_sao_params &p) {   // luma SSD of this MB under p, plus one bit
            int ssd;
            if (stat_ssd(r, p, ssd)) return __fadd_rn(__int2float_rn(ssd), __fmul_rn(a.lambda, 1.0f));
            if (!have_tile) {
                TileRegs t;
                tile_load(a, c, row, lane, t);
                __syncwarp();
                tile_store(tile, lane, t);
                __syncwarp();
                have_tile = true;
            }
            return __fadd_rn(__ll2float_rn(tile_sao_ssd(a.W, a.H, tile, c, row, lane, p)), __fmul_rn(a.lambda, 1.0f));
        };
        // The merge-left cost needs only this row's previous MB: it is computed
        // before the wait for the row above, off the wavefront's critical path.
        const bool try_left = c > 0 && left.luma.type != 0;
        const float mc_left = try_left ? cost(left.luma) : 0.0f;
        unsigned long long above = 0;
        if (row > 0) {   // bounded wait for the final parameters of (r-1, c)
            const bool ok = words ? wait_word<true>(a, &words[i * a.mbw + c], ep, above)
                                  : wait_word<false>(a, &a.sao_mail[m - a.mbw], ep, above);
            if (!ok) {
                cp_async_wait_all();   // no copy left in flight into the ring
                return false;
            }
        }
        if (try_left && mc_left < cur) { info.merge_left = 1; info.luma = left.luma; info.chroma = left.chroma; cur = mc_left; }
        if (!info.merge_left && row > 0) {
            const evxg_sao_params al = unpack_params(above >> 8), ac = unpack_params(above >> 33);
            if (al.type != 0 && cost(al) < cur) { info.merge_above = 1; info.luma = al; info.chroma = ac; }
        }
        left = info;
        // every lane stores the same value to the same address: one store each
        const unsigned long long word = ep | (pack_params(info.luma) << 8) | (pack_params(info.chroma) << 33);
        uint4 fin;
        memcpy(&fin, &info, sizeof fin);
        *reinterpret_cast<uint4 *>(&a.sao[m]) = fin;
        if (words) {
            *(volatile unsigned long long *)&words[(i + 1) * a.mbw + c] = word;
            if (next) *(volatile unsigned long long *)&next[c] = word;
        } else {
            st_release64(&a.sao_mail[m], word);
        }
        __syncwarp();
    }
    cp_async_wait_all();
    return true;
}

__device__ __forceinline__ unsigned merge_rank()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void merge_cluster_barrier()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
template <class T>
__device__ __forceinline__ T *merge_peer(T *p, unsigned rank)
{
    T *r;
    asm volatile("mapa.u64 %0, %1, %2;" : "=l"(r) : "l"(p), "r"(rank));
    return r;
}

// Every CTA reaches both cluster barriers: the first makes every CTA's words
// zero (epoch 0 never matches) before a peer may write into them, the last
// keeps every CTA alive while a peer may still write into it.
__device__ __forceinline__ void sao_merge_body(const FrameArgs &a, unsigned char *dsm)
{
    const unsigned k = merge_rank();
    const int w = threadIdx.x >> 5;
    const int rpc = merge_rpc(a.mbh), r0 = (int)k * rpc, rows = max(0, min(rpc, a.mbh - r0));
    MergeTile *tiles = reinterpret_cast<MergeTile *>(dsm);
    int2 *rings = reinterpret_cast<int2 *>(dsm + MERGE_WARPS * sizeof(MergeTile));
    unsigned long long *words =
        merge_words_fit(a.mbw, a.mbh) ? reinterpret_cast<unsigned long long *>(dsm + MERGE_WARPS * MERGE_WARP_BYTES) : nullptr;
    if (words)
        for (int e = threadIdx.x; e < (rpc + 1) * a.mbw; e += blockDim.x) words[e] = 0;
    merge_cluster_barrier();
    unsigned long long *next = nullptr;
    if (words && r0 + rpc < a.mbh) next = merge_peer(words, k + 1);   // the next block's word row 0
    bool alive = true;
    for (int i = w; i < rows && alive; i += MERGE_WARPS)
        alive = merge_row(a, tiles[w], rings + w * MERGE_RING * kSaoStatEntries, words, i == rpc - 1 ? next : nullptr, i, r0 + i);
    merge_cluster_barrier();
}
__global__ void __cluster_dims__(MERGE_CTAS, 1, 1) __launch_bounds__(32 * MERGE_WARPS, 1) k_sao_merge(FrameArgs a)
{
    extern __shared__ __align__(16) unsigned char merge_smem[];
    sao_merge_body(a, merge_smem);
}
__global__ void __cluster_dims__(MERGE_CTAS, 1, 1) __launch_bounds__(32 * MERGE_WARPS, 1) k_sao_merge_b(const FrameArgs *args)
{
    extern __shared__ __align__(16) unsigned char merge_smem[];
    __shared__ FrameArgs sa;
    const FrameArgs *a = batch_args(args, sa);   // a cluster is one stream: active or not for all its CTAs
    if (a) sao_merge_body(*a, merge_smem);
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
// In the first pass one work item is 8 consecutive samples of a row (always
// inside one MB: MBs are 16 luma / 8 chroma samples wide), read and written
// as 16-byte chunks; the item's row and column come from one 32-bit division.
// After it, band offsets and every sample whose edge neighbours lie in its
// own MB or raster-later ones are final: neighbours are one sample away, so
// only a sample on its MB's top row or left column can read a raster-earlier
// MB, and the later passes evaluate those samples of edge-offset MBs alone
// (luma 16 + 15, chroma 8 + 7 per MB and plane), one thread each.
// Edge-offset value of sample (x, y) of MB m, unfiltered value v.
__device__ __forceinline__ int sao_fix_sample(const FrameArgs &a, const evxg_sao_params &p, const int16_t *orig,
                                              const int16_t *img, int w, int h, int sh, int m, int x, int y, int v)
{
    const int ax = x + c_eo[p.eo_class][0], ay = y + c_eo[p.eo_class][1];
    const int bx = x + c_eo[p.eo_class][2], by = y + c_eo[p.eo_class][3];
    if (ax < 0 || ax >= w || ay < 0 || ay >= h || bx < 0 || bx >= w || by < 0 || by >= h) return v;
    const int ma = (ay >> sh) * a.mbw + (ax >> sh), mb = (by >> sh) * a.mbw + (bx >> sh);
    const size_t ka = (size_t)ay * w + ax, kb = (size_t)by * w + bx;
    const int va = ma < m ? __ldcg(img + ka) : orig[ka];
    const int vb = mb < m ? __ldcg(img + kb) : orig[kb];
    const int ct = eo_cat(v, va, vb);
    return ct < 4 ? sclamp(v + p.offsets[ct]) : v;
}
__device__ __forceinline__ void sao_fix_border(const FrameArgs &a, int pass)
{
    constexpr int kLuma = 31, kChroma = 15, kPer = kLuma + 2 * kChroma;
    const int cw = a.W / 2, ch = a.H / 2;
    const size_t ny = (size_t)a.W * a.H, nc = (size_t)cw * ch;
    bool changed = false;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.mbw * a.mbh * kPer; i += gridDim.x * blockDim.x) {
        const int m = i / kPer, s = i - m * kPer;
        const int pl = s < kLuma ? 0 : (s < kLuma + kChroma ? 1 : 2);
        const evxg_sao_params p = pl ? a.sao[m].chroma : a.sao[m].luma;
        if (p.type != 1) continue;
        const int t = pl == 0 ? s : (pl == 1 ? s - kLuma : s - kLuma - kChroma);
        const int n = pl ? 8 : 16, sh = pl ? 3 : 4, w = pl ? cw : a.W, h = pl ? ch : a.H;
        const int x0 = (m % a.mbw) * n, y0 = (m / a.mbw) * n;
        const int x = t < n ? x0 + t : x0, y = t < n ? y0 : y0 + t - n + 1;   // top row, then the left column
        const size_t off = pl == 0 ? 0 : (pl == 1 ? ny : ny + nc);
        int16_t *img = a.planes[a.dpb] + off;
        const int16_t *orig = a.sao_orig + off;
        const size_t k = (size_t)y * w + x;
        const int corr = sao_fix_sample(a, p, orig, img, w, h, sh, m, x, y, orig[k]);
        if (__ldcg(img + k) != corr) {   // the sample is this thread's alone
            img[k] = (int16_t)corr;
            changed = true;
        }
    }
    if (__any_sync(0xffffffffu, changed) && (threadIdx.x & 31) == 0) atomicOr(&a.sao_flags[pass], 1);
}
__device__ __forceinline__ void sao_fix_body(const FrameArgs &a, int pass)
{
    if (pass > 0 && __ldcg(&a.sao_flags[pass - 1]) == 0) return;
    if (pass > 0) {
        sao_fix_border(a, pass);
        return;
    }
    const int cw = a.W / 2, ch = a.H / 2;
    const int ly = a.H * (a.W / 8), lc = ch * (cw / 8);   // items per plane
    const size_t ny = (size_t)a.W * a.H, nc = (size_t)cw * ch;
    bool changed = false;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ly + 2 * lc; i += gridDim.x * blockDim.x) {
        const int pl = i < ly ? 0 : (i < ly + lc ? 1 : 2);
        const int j = pl == 0 ? i : (pl == 1 ? i - ly : i - ly - lc);
        const int w = pl ? cw : a.W, h = pl ? ch : a.H, sh = pl ? 3 : 4;   // MB size 8 / 16 = 1 << sh
        const int cpr = w / 8, y = j / cpr, x0 = (j - y * cpr) * 8;
        const int m = (y >> sh) * a.mbw + (x0 >> sh);
        const evxg_sao_params p = pl ? a.sao[m].chroma : a.sao[m].luma;
        if (p.type == 0) continue;
        const size_t off = pl == 0 ? 0 : (pl == 1 ? ny : ny + nc);
        const int16_t *orig = a.sao_orig + off;
        int16_t *img = a.planes[a.dpb] + off;
        const size_t k0 = (size_t)y * w + x0;
        uint4 ov = *reinterpret_cast<const uint4 *>(orig + k0), iv = __ldcg(reinterpret_cast<const uint4 *>(img + k0));
        const int16_t *o8 = reinterpret_cast<const int16_t *>(&ov);
        int16_t *i8 = reinterpret_cast<int16_t *>(&iv);
        bool any = false;
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const int x = x0 + e, v = o8[e];
            int corr = v;
            if (p.type == 2) {
                const int idx = (sclamp(v) >> 3) - p.band_position;
                if (idx >= 0 && idx < 4) corr = sclamp(v + p.offsets[idx]);
            } else {
                corr = sao_fix_sample(a, p, orig, img, w, h, sh, m, x, y, v);
            }
            if (i8[e] != corr) { i8[e] = (int16_t)corr; any = true; }
        }
        if (any) {   // the item's samples are this thread's alone
            *reinterpret_cast<uint4 *>(img + k0) = iv;
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
