// evxg_device.cuh -- device-side constants and exact-integer helpers shared by
// the EVX3 encoder kernels (sm_100a).  Every helper keeps the reference's C
// semantics: truncating division, int16 stores that wrap, int32 products that
// wrap, IEEE single precision with round-to-nearest and no FMA contraction.
#pragma once
#include <cstdint>
#include <climits>
#include <cuda_runtime.h>
#include "evxg.h"

namespace evxg {

// Block-type bits (reference src/video/types.h:63-91).
constexpr int BT_INTRA = 1, BT_MOTION = 2, BT_COPY = 4;
constexpr int INTRA_DEFAULT = 1, INTER_MOTION_DELTA = 2;
constexpr int MODE_NONE = 7;
constexpr int SAD_THRESHOLD = 8192;   // motion.cpp:24
constexpr int SEARCH_RADIUS = 16;     // motion.cpp:29
constexpr int MAXQ = 63;              // quantize.h:42 (levels - 1)

// Search window in shared memory: a 16x16 block anywhere within +-31 px of a
// base position, plus the 6-tap overshoot (-3 .. +18), clamped to the frame
// the way interp.cpp:8-14 clamps its samples.
// The window's left edge is rounded down to a multiple of 8 samples so rows
// are copied as aligned 16-byte chunks; a chunk is then either entirely
// inside the plane or entirely outside it (plane widths are multiples of 8).
constexpr int WL_ROWS = 84;           // luma rows:  base-34 .. base+49
constexpr int WL = 104;               // luma row stride: 13 chunks cover base-41 .. base+62 (stride avoids 4-way bank conflicts)
constexpr int WC_ROWS = 48;           // chroma rows: (base>>1)-19 .. +28
constexpr int WC = 56;                // chroma row stride: 7 chunks
constexpr int WL_OFF = 34, WC_OFF = 19;

__device__ __forceinline__ int rdiv(int n, int d)   // rounded_div, evx_math.h:228-236
{
    return (((n < 0) != (d < 0)) ? n - d / 2 : n + d / 2) / d;   // one division: select the numerator first
}
__device__ __forceinline__ int lg2u(unsigned v) { return v ? 31 - __clz((int)v) : 0; }  // evx_math.h:69-113
__device__ __forceinline__ int req_bits8(int x) { return lg2u((unsigned)(x & 255)) + 1; }  // required_bits((uint8)x)
__device__ __forceinline__ int iabs32(int v) { return v == INT_MIN ? INT_MAX : (v < 0 ? -v : v); }
__device__ __forceinline__ int16_t iabs16(int16_t v) { return v == INT16_MIN ? (int16_t)INT16_MAX : (int16_t)(v < 0 ? -v : v); }
__device__ __forceinline__ int16_t sgn16(int16_t v) { return (int16_t)((v > 0) - (v < 0)); }
__device__ __forceinline__ int wmul(int a, int b) { return (int)((unsigned)a * (unsigned)b); }
__device__ __forceinline__ int16_t tap6(int a, int b, int c, int d, int e, int f)   // interp.cpp:18-41
{
    return (int16_t)((a - 5 * b + 20 * c + 20 * d - 5 * e + f + 16) >> 5);
}
// cost = (float)a + lambda * (float)b, in that operation order.
__device__ __forceinline__ float rd_cost(int a, float lambda, unsigned b)
{
    return __fadd_rn(__int2float_rn(a), __fmul_rn(lambda, __uint2float_rn(b)));
}

// Whole-warp integer sum / max (wrapping sum: the order does not matter).
__device__ __forceinline__ int warp_sum(int v) { return __reduce_add_sync(0xffffffffu, v); }
__device__ __forceinline__ int warp_max(int v) { return __reduce_max_sync(0xffffffffu, v); }
__device__ __forceinline__ long long warp_sum64(long long v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// acquire / release on a progress word (gpu scope)
__device__ __forceinline__ int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int *p, int v)
{
    asm volatile("st.release.gpu.global.s32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release64(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.release.gpu.global.u64 [%0], %1;" :: "l"(p), "l"(v) : "memory");
}
// 16-byte asynchronous copies global -> shared, in commit groups.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// The SAO RDO's results for one MB, read by the merge: entries 0..31 are the
// luma bands, 32..47 the luma edge categories (class * 4 + category), each as
// (sum of source - recon, count | lowest recon sample << 9 | highest << 17);
// entry 48 is the luma SSD without SAO and a flag set when a recon sample
// lies outside [0, 255]; 49 the cost of the MB's own parameters (float bits);
// 50..51 those parameters (evxg_sao_info).  416 bytes, a multiple of 16.
constexpr int kSaoStatEntries = 52;

// Per-frame parameters shared by all kernels of one encode step.
struct FrameArgs {
    int W, H, mbw, mbh;          // aligned context size and MB grid
    int vis_w, vis_h;            // visible RGB size
    int type, quality, dpb, ref_fwd, ref_bwd;
    // P frames: the references searched, nearest first.  With B frames one,
    // the frame's forward slot; without them (EVX_ENABLE_B_FRAMES 0) the slots
    // at offsets 1 .. EVX_REFERENCE_FRAME_COUNT-1 from the frame index
    // (encode.cpp:211-247), whose descriptors name the offset and which pay a
    // distance bias (ip_mode).
    int nref, ref_slot[3], ip_mode;
    float lambda;
    int16_t *planes[4];          // DPB plane sets
    int16_t *src;                // converted source plane set
    int16_t *lev;                // quantised level plane set (persistent)
    evxg_block_desc *bt;         // block table of this frame
    const evxg_block_desc *prev; // temporal MV predictor table (P frames), else null
    evxg_sao_info *sao;          // final SAO table
    int2 *sao_stats;             // per MB: kSaoStatEntries entries of RDO results for the merge
    int16_t *sao_orig;           // deblocked, not yet SAO-filtered copy of the destination slot
    int *sao_flags;              // per fixed-point pass: 1 if the pass changed a pixel
    unsigned long long *sao_mail;// per MB: final SAO parameters of this frame, tagged with epoch
    int epoch;                   // 1..255, differs from the previous frame's
    const uint8_t *rgb;          // device RGB24 input
    int *progress;               // per-MB-row progress words (wavefronts)
    int *counters;               // [0] next MB row, [1] next SAO merge row, [2] next SAO apply row
    int *error;                  // device error word (0 = ok)
    long long timeout_ns;        // bound on every spin-wait
    int active;                  // batched launches: 0 = this stream has no frame in the tick
    // batched bookkeeping (the single path does these with copies and memsets)
    evxg_block_desc *prev_tab;   // temporal predictor table (the frame's update target)
    evxg_block_desc *prev_ser;   // snapshot of it for the serializer
    size_t plane_elems;          // samples in one plane set
    // deblocking beside the macroblock pass: filtered rows go to db_out
    // (else in place), each band once the wavefront has finished its rows
    int16_t *db_out;
    int db_wait;
};

// Batched launches: blockIdx.z selects the stream; its parameters are copied
// into shared memory once per block.  Returns null for a stream without a
// frame in this tick (the whole block then returns).
__device__ __forceinline__ const FrameArgs *batch_args(const FrameArgs *args, FrameArgs &sa)
{
    if (threadIdx.x == 0 && threadIdx.y == 0) sa = args[blockIdx.z];
    __syncthreads();
    return sa.active ? &sa : nullptr;
}

}  // namespace evxg
