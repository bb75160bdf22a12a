// Tensor-core (tcgen05) spike x weight convolution with BF16-split weights.
//
// Implicit GEMM: D[m, n] = sum_k A[m, k] * W[n, k] with
//   m = (image, oy, ox) over N*OH*OW output positions (N folds batch, time),
//   k = a receptive-field tap (ky, kx) and input channel c,
//   A[m, k] = spike u8 of the receptive field (exact in BF16).
// Each F32 weight is split into BF16 terms w = h + m (+ l) (h = bf16(w),
// m = bf16(w - h), l = bf16(w - h - m)); every term gets its own FP32
// accumulator in tensor memory, so each partial sum stays exact for weights
// in [2^-6, 1]; the terms are added once in FP64 and rounded once to F32.
// BF16X3 therefore reproduces the exactly rounded potential; BF16X2 (hi+lo)
// is within 2^-18 relative.
//
// Two A layouts:
//  * channels-last (Cin >= 8): the spikes are first transposed to
//    [N, H, W, Cpad] u8 (Cpad = Cin rounded up to 8) and k = tap * Cpad + c,
//    so every 8-wide K chunk of a row is one 8-byte load;
//  * channel-major (Cin < 8): k = c * KH*KW + tap (the reference's order),
//    gathered element by element (keeps K small for 1-2 input channels).
//
// CTA (persistent, 256 threads) per 128-row M tile and N tile walks K in
// 64-wide blocks through a two-stage shared-memory ring: thread 0 starts a
// bulk copy (TMA engine, no multicast) of the pre-split weight block, stored
// in global memory in the K-major no-swizzle canonical layout, while all
// threads gather the A block; thread 0 then issues the tcgen05.mma
// instructions (M=128, N=n_tile, K=16) and commits them to the stage's
// mbarrier.  The epilogue reads the accumulators with tcgen05.ld.  Every
// mbarrier wait is bounded: on timeout the kernel records an error in the
// device status word (spk_device_status) and leaves.
#include <algorithm>
#include <type_traits>

#include "conv_tc.cuh"
#include "tc_ptx.cuh"

#include <cuda_bf16.h>

namespace spk
{
static __device__ int g_tc_status;
// Rows (one pixel at one step) whose channel decision the FP32 bound could
// not certify and that were recomputed with FP64 sums.
static __device__ unsigned long long g_rechecks;
// Rows of the search path that the term sums could not decide and that
// were recomputed as the oracle does (search_fix_kernel).
static __device__ unsigned long long g_recomputes;

namespace
{
using namespace tc;

constexpr int BM = 128, BK = 64;
constexpr uint32_t kMaxProbes = 1u << 22;
constexpr int kMaxKBlocks = 128;  // K up to 8192
// entries per block of a row-list compaction
constexpr int kCompactShift = 11, kCompactItems = 1 << kCompactShift;

// Division of any 32-bit n by an invariant d >= 1 (Granlund and Montgomery,
// "Division by Invariant Integers using Multiplication", PLDI 1994, fig. 4.1):
// with l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1,
// n / d = (t + ((n - t) >> min(l, 1))) >> max(l - 1, 0), t = umulhi(m, n).
// sh packs the two shifts (low byte, next byte).
struct DivMagic
{
    uint32_t m, sh;
};

inline DivMagic div_magic(uint32_t d)
{
    int l = 0;
    while (l < 32 && (uint64_t(1) << l) < d) ++l;
    const uint64_t m = ((uint64_t(1) << 32) * ((uint64_t(1) << l) - d)) / d + 1;
    return DivMagic{uint32_t(m), uint32_t(l < 1 ? l : 1) | (uint32_t(l > 1 ? l - 1 : 0) << 8)};
}

__device__ __forceinline__ uint32_t div_by(uint32_t n, uint32_t m, uint32_t sh)
{
    const uint32_t t = __umulhi(n, m);
    return (t + ((n - t) >> (sh & 0xFFu))) >> (sh >> 8);
}

struct TcParams
{
    const uint8_t *in;  // channel-major input, or its channels-last copy
    const uint8_t *wimg;
    float *out;
    int64_t M, tiles, img_stride, ohw;
    // gather strides: element address = base + iy * rs + ix * ps + c * cs
    // (base = image, or sample + step * ts in the fused (pixel, time) layout)
    int64_t rs, ps, cs, ts;
    int cin, h, w, cout, kh, kw, oh, ow, sy, sx, top, left;
    int kblocks, n_tile, n_tiles, nsplit, cpad, nhwc;
    uint32_t tmem_cols, idesc;
    int stages, nacc;
    // fused spiking epilogue (kFused): rows are (pixel, t) with t fastest
    int T, tp_log2, pp, lp_log2;
    int64_t npix;
    float thr, thv, inh_thr, fire_thr, wta_thr;
    uint8_t *spikes;    // [B, T, Cout, OH, OW]
    uint8_t *pooled;    // [B, T, Cout, POH, POW] or null: spikes pooled over pky x pkx windows
    int pky, pkx, poh, pow_;
    int4 *records;      // [B * OH * OW]: (winning channel, first step, value bits, 0)
    unsigned *mins, *maxs;  // [B] order-preserving encodings
    // fused producers: `in` is the first-spike map [B, H, W, Cp]; when *flag
    // is set the input was not cumulative 0/1 spikes and rows are gathered
    // from `raw` [B, T, Cin, H, W] instead
    const uint8_t *raw;
    const int *flag;
    // several networks in one launch (snet null: one network): network of
    // each sample, each network's threshold, byte stride between the
    // networks' weight images.  No tile holds pixels of two networks.
    const int32_t *snet;
    const float *net_thr;
    int64_t wimg_stride;
    // set by the weight split when some weight is negative (then the fused
    // epilogue takes its general argmax)
    int *negw;
    // kTimes: output times [B, Cout, OH, OW]
    float *tout;
    // kSearch (the lean first-crossing search, see search_epilogue): round 0
    // takes every pixel at step T - 1, round 1 the (pixel, step) entries of
    // list_in, round 2 the (pixel, winner) entries of list_in at step T - 1
    int round, wta;
    const int2 *list_in;
    const int *count_in;
    int2 *list_out, *final_list;  // list_out: each row's next entry at the row's index
    int *list_bc;                 // per compaction block of list_out, its entries with a step (added by the writers)
    int *tile_ctr;                // search: tickets of the tiles after each CTA's first (zeroed; null: static)
    uint32_t ohw_m, ohw_sh, ow_m, ow_sh;  // division by ohw and ow: div_magic's multiplier and shifts
    int *final_count;
    int4 *fix_list;  // rows left for the exact recompute: (pixel, step, row index, winner)
    int *fix_count;
    int4 *val_list;  // rows whose winner is decided but not its value: (pixel, step, row index, winner)
    int *val_count;
    int4 *state;     // per pixel: (lo | hi << 8 | winner << 16, value, winner at T-1, value at T-1)
    const float *echan;     // per channel bound of |oracle potential - exact term sum|
    const float *cscale;    // per channel 2^(e - 32): the value of one unit of the term total
    const unsigned *sinfo;  // [0] largest echan (bits), [1] largest channel exponent + 128
    int kreal;              // real K (taps x input channels)
    int r0_list;            // round 0 takes the (pixel, T - 1) entries of list_in (bound pre-filter ran)
    int nparts;             // channel parts of n_tile per tile (search)
    const uint8_t *tlo;     // search: per pixel, the first step the bound allows a spike at (null: 0)
    // kFused: leave at once when the search path ran (no negative weight and
    // cumulative 0/1 input; these are the words of negw and flag)
    int skip_when_lean;
};

// kTimes: the fused (pixel, time) rows with an epilogue that writes each
// neuron's first step above threshold (F32 time, T = never).
constexpr int kPotentials = 0, kFused = 1, kTimes = 2, kSearch = 3;
// Base-256 digits per weight of the search kernels' 8-bit split.
constexpr int kSearchTerms = 4;

__device__ __forceinline__ unsigned order_enc(float f)
{
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float order_dec(unsigned e)
{
    return __uint_as_float((e & 0x80000000u) ? (e & 0x7FFFFFFFu) : ~e);
}

__device__ __forceinline__ uint32_t bf16_of_byte(uint32_t b)
{
    // exact: float(b) for b < 256 has at most 8 significant bits
    return __float_as_uint(__uint_as_float(0x4B000000u | b) - 8388608.0f) >> 16;
}

__device__ __forceinline__ uint4 bf16x8_of_bytes(uint2 v)
{
    uint4 r;
    if (((v.x | v.y) & 0xFEFEFEFEu) == 0)
    {
        // spikes: every byte is 0 or 1, and bf16(1) = 0x3F80 (two per word)
        r.x = __byte_perm(v.x, 0, 0x7170) * 0x3F80u;
        r.y = __byte_perm(v.x, 0, 0x7372) * 0x3F80u;
        r.z = __byte_perm(v.y, 0, 0x7170) * 0x3F80u;
        r.w = __byte_perm(v.y, 0, 0x7372) * 0x3F80u;
        return r;
    }
    r.x = bf16_of_byte(v.x & 0xFF) | (bf16_of_byte((v.x >> 8) & 0xFF) << 16);
    r.y = bf16_of_byte((v.x >> 16) & 0xFF) | (bf16_of_byte(v.x >> 24) << 16);
    r.z = bf16_of_byte(v.y & 0xFF) | (bf16_of_byte((v.y >> 8) & 0xFF) << 16);
    r.w = bf16_of_byte((v.y >> 16) & 0xFF) | (bf16_of_byte(v.y >> 24) << 16);
    return r;
}

// [N, C, H, W] -> [N, H, W, Cpad] (zero-filled pad channels), 8 channels per thread.
__global__ void to_channels_last_kernel(const uint8_t *__restrict__ in, uint2 *__restrict__ out, int64_t n, int c,
                                        int64_t hw, int cpad)
{
    const int groups = cpad / 8;
    const int64_t total = n * hw * groups;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x)
    {
        const int g = int(i % groups);
        const int64_t px = (i / groups) % hw, img = i / (int64_t(groups) * hw);
        const uint8_t *src = in + img * c * hw + px;
        uint32_t lo = 0, hi = 0;
#pragma unroll
        for (int e = 0; e < 8; ++e)
        {
            const int ch = g * 8 + e;
            const uint32_t v = ch < c ? src[int64_t(ch) * hw] : 0u;
            if (e < 4)
                lo |= v << (8 * e);
            else
                hi |= v << (8 * (e - 4));
        }
        out[i] = make_uint2(lo, hi);
    }
}

// Weight images: [n_tiles][kblocks][nsplit][n_tile x 64] BF16 in the K-major
// no-swizzle layout (8-row groups of 1024 B, 8 K-chunks of 128 B, 16 B per
// row), K ordered as the A operand.  One thread per (tile, block, row, chunk).
__global__ void split_weights_kernel(const float *__restrict__ kernel, uint4 *__restrict__ wimg, int cout, int cin,
                                     int taps, int nhwc, int cpad, int kblocks, int n_tile, int n_tiles, int nsplit,
                                     int64_t wimg_stride16, int *negw)
{
    // blockIdx.y: network (kernels [N, Cout, Cin, KH, KW], images wimg_stride16 uint4 apart)
    kernel += int64_t(blockIdx.y) * cout * cin * taps;
    wimg += int64_t(blockIdx.y) * wimg_stride16;
    const int64_t total = int64_t(n_tiles) * kblocks * n_tile * 8;
    const int kreal = nhwc ? taps * cpad : taps * cin;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x)
    {
        const int kc = int(i % 8);
        const int nl = int((i / 8) % n_tile);
        const int kb = int((i / (8 * n_tile)) % kblocks);
        const int nt = int(i / (int64_t(8) * n_tile * kblocks));
        const int n = nt * n_tile + nl;
        uint32_t parts[3][4];
#pragma unroll
        for (int e = 0; e < 8; e += 2)
        {
            uint32_t bits[2][3];
#pragma unroll
            for (int q = 0; q < 2; ++q)
            {
                const int k = kb * BK + kc * 8 + e + q;
                float wv = 0.f;
                if (n < cout && k < kreal)
                {
                    int c, tap;
                    if (nhwc)
                        tap = k / cpad, c = k % cpad;
                    else
                        c = k / taps, tap = k % taps;
                    if (c < cin) wv = kernel[(int64_t(n) * cin + c) * taps + tap];
                }
                if (negw != nullptr && !(wv >= 0.f)) atomicOr(negw, 1);
                const __nv_bfloat16 h = __float2bfloat16_rn(wv);
                const float r1 = __fsub_rn(wv, __bfloat162float(h));
                const __nv_bfloat16 m = __float2bfloat16_rn(r1);
                const float r2 = __fsub_rn(r1, __bfloat162float(m));
                const __nv_bfloat16 l = __float2bfloat16_rn(r2);
                bits[q][0] = __bfloat16_as_ushort(h), bits[q][1] = __bfloat16_as_ushort(m);
                bits[q][2] = __bfloat16_as_ushort(l);
            }
#pragma unroll
            for (int p = 0; p < 3; ++p) parts[p][e / 2] = bits[0][p] | (bits[1][p] << 16);
        }
        const int64_t block = (int64_t(nt) * kblocks + kb) * nsplit;
        for (int p = 0; p < nsplit; ++p)
        {
            const int64_t idx = (block + p) * (int64_t(n_tile) * 8) + (nl / 8) * 64 + kc * 8 + (nl % 8);
            wimg[idx] = make_uint4(parts[p][0], parts[p][1], parts[p][2], parts[p][3]);
        }
    }
}

__device__ __forceinline__ bool wait_bounded(uint64_t *bar, uint32_t parity)
{
    for (uint32_t i = 0; i < kMaxProbes; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    atomicExch(&g_tc_status, 1);
    return false;
}

__device__ __forceinline__ void arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// 8-byte asynchronous global -> shared copy (both addresses 8-byte aligned),
// completed for the issuing thread by cp_async_wait_all.
__device__ __forceinline__ void cp_async8(void *dst, const void *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Bulk (non-tensor) global -> shared copy completing on `bar`; both addresses
// 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// 16 consecutive accumulator columns of this warp's 32 rows, the BF16 terms
// added in FP64 and rounded once to F32.  Warp-uniform (tcgen05.ld is .sync).
__device__ __forceinline__ void load_exact16(uint32_t lane_base, int c0, int n_tile, int nsplit, float (&v)[16])
{
    uint32_t r0[16], r1[16], r2[16];
    tmem_ld16(lane_base + uint32_t(c0), r0);
    tmem_ld16(lane_base + uint32_t(n_tile + c0), r1);
    if (nsplit == 3) tmem_ld16(lane_base + uint32_t(2 * n_tile + c0), r2);
    tmem_ld_wait();
#pragma unroll
    for (int j = 0; j < 16; ++j)
    {
        double acc = double(__uint_as_float(r0[j])) + double(__uint_as_float(r1[j]));
        if (nsplit == 3) acc += double(__uint_as_float(r2[j]));
        v[j] = float(acc);
    }
}

// Fused spiking epilogue of one tile of PP pixels x TP steps, with every
// output channel of a pixel in this CTA's tensor memory.  Restates, for the
// pipeline  out = inhibit(threshold(conv(x), thr, thv), inh_thr);
// spikes = fire(out, fire_thr); convwta(out, r, k, wta_thr):
//   threshold  cpu/fire.cpp:41-51     x <= thr -> thv
//   inhibit    cpu/inhibit.cpp:41-121 first-max channel per step, winner taken
//              at step T - max(#steps whose max > inh_thr, 1), others x * 0
//   fire       cpu/fire.cpp:67-82     x > fire_thr
//   WTA key    cpu/wta.cpp:45-64      first step with x > wta_thr, its value
// With fire_thr, wta_thr >= 0 only the winning channel of a pixel can spike or
// hold a WTA key, so each pixel yields one record (channel, first step,
// value) and the per-sample min / max of the inhibited potentials.  Run by
// warps 0-3, one (pixel, step) row per thread; `acc` is the accumulator base.
// Fast first-max state of one row (see row_argmax).
struct FastMax
{
    float r1 = -INFINITY, r2 = -INFINITY, amax = 0.f, dmin = INFINITY;
    int a1 = -1, b1 = INT_MAX;
};

constexpr int kEpiChunk = 8;  // accumulator columns per tensor-memory load

// Lean first-max state (non-negative weights, value <= threshold): the
// largest potential (first index) and the runner-up over all channels.
struct LeanMax
{
    float r1 = -INFINITY, r2 = -INFINITY;
    int a1 = -1;
};

__device__ __forceinline__ void merge_lean(LeanMax &s, const LeanMax &o)
{
    const bool take = o.r1 > s.r1 || (o.r1 == s.r1 && o.a1 >= 0 && (s.a1 < 0 || o.a1 < s.a1));
    s.r2 = fmaxf(fmaxf(s.r2, o.r2), take ? s.r1 : o.r1);
    s.r1 = take ? o.r1 : s.r1;
    s.a1 = take ? o.a1 : s.a1;
}

// Merge the state of another set of channels into s: the larger maximum
// wins, ties going to the lower channel; the loser's maximum competes for
// the runner-up.
__device__ __forceinline__ void merge_fast(FastMax &s, const FastMax &o)
{
    const bool take = o.r1 > s.r1 || (o.r1 == s.r1 && o.a1 >= 0 && (s.a1 < 0 || o.a1 < s.a1));
    s.r2 = fmaxf(fmaxf(s.r2, o.r2), take ? s.r1 : o.r1);
    s.r1 = take ? o.r1 : s.r1;
    s.a1 = take ? o.a1 : s.a1;
    s.amax = fmaxf(s.amax, o.amax);
    s.dmin = fminf(s.dmin, o.dmin);
    s.b1 = min(s.b1, o.b1);
}

template <int NS>
__device__ __forceinline__ void tmem_chunk(uint32_t lane_base, int c0, int n_tile, uint32_t (&q)[3][kEpiChunk])
{
    tmem_ld8(lane_base + uint32_t(c0), q[0]);
    tmem_ld8(lane_base + uint32_t(n_tile + c0), q[1]);
    if (NS == 3) tmem_ld8(lane_base + uint32_t(2 * n_tile + c0), q[2]);
}

template <int NS>
__device__ __forceinline__ void tmem_chunk_wait(uint32_t (&q)[3][kEpiChunk])
{
    tmem_ld_wait8(q[0]);
    tmem_ld_wait8(q[1]);
    if (NS == 3) tmem_ld_wait8(q[2]);
}

// One chunk of columns: f = (h + m) + l in FP32, the largest above-threshold
// value (first index on ties) and the runner-up, the first below-threshold
// channel, the largest |h| + |m| + |l| and the closest distance to the
// threshold.  Branch-free.
template <int NS>
__device__ __forceinline__ void fast_chunk(const TcParams &P, float thr, const uint32_t (&q)[3][kEpiChunk], int c0,
                                           FastMax &st)
{
#pragma unroll
    for (int j = 0; j < kEpiChunk; ++j)
    {
        const int c = c0 + j;
        const float h = __uint_as_float(q[0][j]), m = __uint_as_float(q[1][j]);
        const float l = NS == 3 ? __uint_as_float(q[2][j]) : 0.f;
        const float f = __fadd_rn(__fadd_rn(h, m), l);
        const float a = __fadd_rn(__fadd_rn(fabsf(h), fabsf(m)), fabsf(l));
        const bool valid = c < P.cout;
        const bool real = valid && f > thr;
        const bool gt = real && f > st.r1;
        st.amax = valid ? fmaxf(st.amax, a) : st.amax;
        st.dmin = valid ? fminf(st.dmin, fabsf(__fsub_rn(f, thr))) : st.dmin;
        st.r2 = gt ? st.r1 : (real ? fmaxf(st.r2, f) : st.r2);
        st.r1 = gt ? f : st.r1;
        st.a1 = gt ? c : st.a1;
        st.b1 = (valid && !real) ? min(st.b1, c) : st.b1;
    }
}

// The lean chunk: f = (h + m) + l and the running first max / runner-up;
// channels past Cout (padding) never win.
template <int NS>
__device__ __forceinline__ void lean_chunk(const TcParams &P, const uint32_t (&q)[3][kEpiChunk], int c0, LeanMax &st)
{
    const int lim = P.cout - c0;
#pragma unroll
    for (int j = 0; j < kEpiChunk; ++j)
    {
        const float h = __uint_as_float(q[0][j]), m = __uint_as_float(q[1][j]);
        const float l = NS == 3 ? __uint_as_float(q[2][j]) : 0.f;
        float f = __fadd_rn(__fadd_rn(h, m), l);
        f = j < lim ? f : -INFINITY;
        const bool gt = f > st.r1;
        st.r2 = gt ? st.r1 : fmaxf(st.r2, f);
        st.r1 = gt ? f : st.r1;
        st.a1 = gt ? c0 + j : st.a1;
    }
}

// Thresholded first-max channel of one row, exactly as with the FP64-summed
// potentials.  Fast pass: the BF16 terms are added in FP32, f = (h + m) + l,
// which is within 3.01 * 2^-24 * (|h| + |m| + |l|) of the exactly rounded
// potential; with tol = 2^-21 times the row's largest such sum, every
// decision is certain unless some potential is within tol of the threshold,
// the two largest above-threshold values are within 2 tol, or the largest is
// within tol of the below-threshold value or of the inhibition threshold.
// Such rows (rare) are redone with FP64 sums.  Tensor-memory loads of the
// next chunk are in flight while a chunk is processed; even and odd chunks
// keep separate states (two independent dependency chains), merged at the end.
template <int NS>
__device__ __forceinline__ void row_argmax(const TcParams &P, float thr, bool lean, uint32_t lane_base, bool row_ok,
                                           int &am, float &xam)
{
    constexpr int W = kEpiChunk;
    uint32_t qa[3][W], qb[3][W];
    bool unsure;
    tmem_chunk<NS>(lane_base, 0, P.n_tile, qa);
    if (lean)
    {
        // Non-negative weights: every BF16 term of a channel has |m|, |l| <=
        // 2^-7.9 h, so |h| + |m| + |l| <= 1.0625 f and 1.0625 * max(r1, 0)
        // bounds the row's term sums.  With value <= threshold a channel at or
        // below the threshold never beats one above it, so only the maximum,
        // its runner-up and the two thresholds decide (no per-channel checks).
        LeanMax st, st2;
        for (int c0 = 0; c0 < P.n_tile; c0 += 2 * W)
        {
            tmem_chunk_wait<NS>(qa);
            tmem_chunk<NS>(lane_base, c0 + W, P.n_tile, qb);
            lean_chunk<NS>(P, qa, c0, st);
            tmem_chunk_wait<NS>(qb);
            if (c0 + 2 * W < P.n_tile) tmem_chunk<NS>(lane_base, c0 + 2 * W, P.n_tile, qa);
            lean_chunk<NS>(P, qb, c0 + W, st2);
        }
        merge_lean(st, st2);
        const float tol = __fmaf_rn(1.0625f * fmaxf(st.r1, 0.f), 0x1p-21f, 0x1p-140f);
        const bool real = st.r1 > thr;
        unsure = fabsf(__fsub_rn(st.r1, thr)) <= tol;
        if (real) unsure |= __fsub_rn(st.r1, st.r2) <= 2.f * tol || fabsf(__fsub_rn(st.r1, P.inh_thr)) <= tol;
        am = real ? st.a1 : 0;
        xam = real ? st.r1 : P.thv;
    }
    else
    {
        FastMax st, st2;
        for (int c0 = 0; c0 < P.n_tile; c0 += 2 * W)
        {
            // n_tile is a multiple of 16 = 2 W: both halves exist
            tmem_chunk_wait<NS>(qa);
            tmem_chunk<NS>(lane_base, c0 + W, P.n_tile, qb);
            fast_chunk<NS>(P, thr, qa, c0, st);
            tmem_chunk_wait<NS>(qb);
            if (c0 + 2 * W < P.n_tile) tmem_chunk<NS>(lane_base, c0 + 2 * W, P.n_tile, qa);
            fast_chunk<NS>(P, thr, qb, c0 + W, st2);
        }
        merge_fast(st, st2);
        const float tol = __fmaf_rn(st.amax, 0x1p-21f, 0x1p-140f);
        unsure = st.dmin <= tol;
        const bool has_real = st.a1 >= 0, has_low = st.b1 != INT_MAX;
        if (has_real && has_low) unsure |= fabsf(__fsub_rn(st.r1, P.thv)) <= tol;
        const bool real_wins = has_real && (!has_low || st.r1 > P.thv);
        if (real_wins) unsure |= __fsub_rn(st.r1, st.r2) <= 2.f * tol || fabsf(__fsub_rn(st.r1, P.inh_thr)) <= tol;
        am = real_wins ? st.a1 : st.b1;
        xam = real_wins ? st.r1 : P.thv;
    }
    const unsigned redo = __ballot_sync(0xffffffffu, unsure && row_ok);
    if (redo)
    {
        if ((threadIdx.x & 31) == 0) atomicAdd(&g_rechecks, (unsigned long long)__popc(redo));
        // exact pass: FP64 sums rounded once to F32 (warp-uniform tcgen05.ld)
        float mx = 0.f;
        int ae = 0;
        for (int c0 = 0; c0 < P.n_tile; c0 += 16)
        {
            float v[16];
            load_exact16(lane_base, c0, P.n_tile, NS, v);
#pragma unroll
            for (int j = 0; j < 16; ++j)
            {
                const int c = c0 + j;
                const float x = (v[j] <= thr) ? P.thv : v[j];
                if (c == 0)
                    mx = x;
                else if (c < P.cout && x > mx)
                    mx = x, ae = c;
            }
        }
        if (unsure) am = ae, xam = mx;
    }
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// `release` (the accumulator's empty barrier) is arrived at as soon as the
// last tensor-memory load of the tile has completed, so the next tile's MMAs
// overlap the stores below.
template <int NS>
__device__ void fused_epilogue(const TcParams &P, float thr, uint32_t acc, bool row_ok, int tstep, int64_t sample,
                               int64_t pix, uint64_t *release)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int TP = 1 << P.tp_log2, T = P.T, C = P.cout;
    const uint32_t lane_base = acc + (uint32_t((warp & 3) * 32) << 16);
    // thresholded first-max channel of this (pixel, step)
    float mx;
    int am;
    // lean argmax: no negative weight and value <= threshold (uniform)
    const bool lean = !*P.negw && P.thv <= thr;
    row_argmax<NS>(P, thr, lean, lane_base, row_ok, am, mx);
    const int base = (lane >> P.tp_log2) << P.tp_log2;  // first lane of this pixel
    const unsigned grp = (TP == 32) ? 0xffffffffu : (((1u << TP) - 1u) << base);
    const unsigned above = __ballot_sync(0xffffffffu, row_ok && mx > P.inh_thr) & grp;
    const int n = __popc(above);
    const int ts = T - (n > 1 ? n : 1);
    const int win = __shfl_sync(0xffffffffu, am, base + ts);
    // exact value of the winning channel at this step: reload only the column
    // chunks that hold the warp's winners
    // (up to two 8-column chunks per round trip)
    uint32_t pieces[3] = {0, 0, 0};
    unsigned pending = 0xffffffffu;
    while (pending)
    {
        const int ca = (__shfl_sync(0xffffffffu, win, __ffs(pending) - 1) >> 3) << 3;
        const bool ma = (win >> 3) == (ca >> 3);
        const unsigned rest = pending & ~__ballot_sync(0xffffffffu, ma);
        const bool two = rest != 0;
        const int cb = two ? (__shfl_sync(0xffffffffu, win, __ffs(rest) - 1) >> 3) << 3 : ca;
        const bool mb = two && (win >> 3) == (cb >> 3);
        uint32_t qa[3][kEpiChunk], qb[3][kEpiChunk];
        tmem_chunk<NS>(lane_base, ca, P.n_tile, qa);
        if (two) tmem_chunk<NS>(lane_base, cb, P.n_tile, qb);
        tmem_chunk_wait<NS>(qa);
        if (two) tmem_chunk_wait<NS>(qb);
#pragma unroll
        for (int j = 0; j < kEpiChunk; ++j)
        {
            if (ma && ca + j == win)
            {
                pieces[0] = qa[0][j], pieces[1] = qa[1][j];
                if (NS == 3) pieces[2] = qa[2][j];
            }
            if (mb && cb + j == win)
            {
                pieces[0] = qb[0][j], pieces[1] = qb[1][j];
                if (NS == 3) pieces[2] = qb[2][j];
            }
        }
        pending &= ~__ballot_sync(0xffffffffu, ma || mb);
    }
    tc_fence_before();
    mbar_arrive(release);
    double accv = double(__uint_as_float(pieces[0])) + double(__uint_as_float(pieces[1]));
    if (NS == 3) accv += double(__uint_as_float(pieces[2]));
    const float raw = float(accv);
    const float vw = (raw <= thr) ? P.thv : raw;
    // spike of the winning channel (the spike tensor was zero-filled first)
    if (row_ok && vw > P.fire_thr)
    {
        P.spikes[((sample * T + tstep) * C + win) * P.ohw + pix] = 1;
        if (P.pooled)
        {
            // max of 0/1 spikes over the window: any spike marks the cell
            // (several pixels may store the same 1)
            const int oy = int(pix / P.ow), ox = int(pix - int64_t(oy) * P.ow);
            const int py = oy / P.pky, px = ox / P.pkx;
            if (py < P.poh && px < P.pow_)
                P.pooled[((sample * T + tstep) * C + win) * int64_t(P.poh) * P.pow_ + py * P.pow_ + px] = 1;
        }
    }
    if (P.records == nullptr) return;  // no WTA on this call (uniform)
    // WTA record: first step whose inhibited value exceeds wta_thr
    const unsigned keyed = __ballot_sync(0xffffffffu, row_ok && vw > P.wta_thr) & grp;
    const int first_lane = keyed ? __ffs(keyed) - 1 : base;
    const float first_v = __shfl_sync(0xffffffffu, vw, first_lane);
    const bool pixel_ok = __shfl_sync(0xffffffffu, row_ok ? 1 : 0, base) != 0;
    if (lane == base && pixel_ok)
        P.records[sample * P.ohw + pix] = make_int4(win, keyed ? first_lane - base : T, __float_as_int(first_v), 0);
    // per-sample min / max of the inhibited values: the winner's value, and a
    // zero from every losing channel when there is more than one channel
    float rmin = vw, rmax = vw;
    if (C > 1)
    {
        rmin = (0.f < rmin) ? 0.f : rmin;
        rmax = (rmax < 0.f) ? 0.f : rmax;
    }
    const unsigned okm = __ballot_sync(0xffffffffu, row_ok);
    if (okm == 0) return;
    const int src = __ffs(okm) - 1;
    const int key = row_ok ? int(sample) : -1;
    const int k0 = __shfl_sync(0xffffffffu, key, src);
    if (__all_sync(0xffffffffu, !row_ok || key == k0))
    {
        const unsigned emin = __reduce_min_sync(0xffffffffu, row_ok ? order_enc(rmin) : 0xFFFFFFFFu);
        const unsigned emax = __reduce_max_sync(0xffffffffu, row_ok ? order_enc(rmax) : 0u);
        if (lane == src)
        {
            atomicMin(P.mins + sample, emin);
            atomicMax(P.maxs + sample, emax);
        }
        return;
    }
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const unsigned emin = __reduce_min_sync(peers, order_enc(rmin));
    const unsigned emax = __reduce_max_sync(peers, order_enc(rmax));
    if (row_ok && lane == __ffs(peers) - 1)
    {
        atomicMin(P.mins + sample, emin);
        atomicMax(P.maxs + sample, emax);
    }
}

// First-spike epilogue (kTimes) of one tile of PP pixels x TP steps: per
// (row, channel) the potential is the FP64 sum of the BF16 terms rounded once
// to F32 (the value the op-by-op conv writes), a spike is potential > thr
// (cpu/fire.cpp:67-82), and a neuron's time is its first spiking step, T
// when none (cpu/time.cpp:40-58).  A warp's ballot per channel finds it for
// the rows it holds; pixels spread over several warps (TP > 32) take the
// minimum of the warps' candidates through shared memory (double-buffered by
// tile parity; `tbar`, an mbarrier of the 128 epilogue threads, completes
// once per tile and its wait is bounded like every other).
template <int NS>
__device__ void times_epilogue(const TcParams &P, uint32_t acc, bool row_ok, int64_t mt, uint64_t *release,
                               int *s_cand, uint32_t j, uint64_t *tbar)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int TP = 1 << P.tp_log2;
    const uint32_t lane_base = acc + (uint32_t((warp & 3) * 32) << 16);
    const bool split = TP > 32;
    int *cand = s_cand + int(j & 1) * 4 * P.n_tile + warp * P.n_tile;
    const int gsz = split ? 32 : TP, base = (lane / gsz) * gsz;
    const unsigned gmask = gsz == 32 ? 0xffffffffu : (((1u << gsz) - 1u) << base);
    // (sample, pixel) of this lane's group (TP <= 32: a whole pixel)
    const uint32_t gp = uint32_t(mt) * uint32_t(P.pp) + uint32_t((warp * 32 + base) >> P.tp_log2);
    const bool pix_ok = int64_t(gp) < P.npix;
    const uint32_t smp = gp / uint32_t(P.ohw), pix = gp - smp * uint32_t(P.ohw);
    const int t_lane0 = (warp * 32) & (TP - 1);
    for (int c0 = 0; c0 < P.n_tile; c0 += kEpiChunk)
    {
        uint32_t q[3][kEpiChunk];
        tmem_chunk<NS>(lane_base, c0, P.n_tile, q);
        tmem_chunk_wait<NS>(q);
#pragma unroll
        for (int e = 0; e < kEpiChunk; ++e)
        {
            const int c = c0 + e;
            double v = double(__uint_as_float(q[0][e])) + double(__uint_as_float(q[1][e]));
            if (NS == 3) v += double(__uint_as_float(q[2][e]));
            const bool spike = row_ok && c < P.cout && float(v) > P.thr;
            const unsigned bal = __ballot_sync(0xffffffffu, spike) & gmask;
            if (split)
            {
                if (lane == 0) cand[c] = bal ? t_lane0 + __ffs(bal) - 1 : P.T;
            }
            else if (lane == base && pix_ok && c < P.cout)
                P.tout[(int64_t(smp) * P.cout + c) * P.ohw + pix] = float(bal ? __ffs(bal) - 1 - base : P.T);
        }
    }
    tc_fence_before();
    mbar_arrive(release);
    if (!split) return;
    mbar_arrive(tbar);
    if (!wait_bounded(tbar, j & 1)) return;
    const int wpp = TP / 32;  // warps per pixel
    const int *cb = s_cand + int(j & 1) * 4 * P.n_tile;
    for (int i = tid; i < P.pp * P.cout; i += 128)
    {
        const int pl = i / P.cout, c = i - pl * P.cout;
        const uint32_t g = uint32_t(mt) * uint32_t(P.pp) + uint32_t(pl);
        if (int64_t(g) >= P.npix) continue;
        int t = P.T;
        for (int w = pl * wpp; w < pl * wpp + wpp; ++w) t = min(t, cb[w * P.n_tile + c]);
        const uint32_t sm = g / uint32_t(P.ohw), px = g - sm * uint32_t(P.ohw);
        P.tout[(int64_t(sm) * P.cout + c) * P.ohw + px] = float(t);
    }
}

// Row of a tile: (image for the A gather, sample, step, output pixel).
struct RowInfo
{
    bool ok;
    int64_t img, sample, pix;
    int tstep, iy0, ix0;
};

template <int MODE>
__device__ __forceinline__ RowInfo row_info(const TcParams &P, int64_t mt, int row)
{
    RowInfo r{};
    if constexpr (MODE == kPotentials)
    {
        const int64_t m = mt * BM + row;
        r.ok = m < P.M;
        if (r.ok) r.img = m / P.ohw, r.pix = m % P.ohw;
    }
    else
    {
        // row = (pixel in tile) * TP + t: all steps of a pixel in one warp;
        // pixel indexes fit in 32 bits (checked on the host)
        r.tstep = row & ((1 << P.tp_log2) - 1);
        const uint32_t gp = uint32_t(mt) * uint32_t(P.pp) + uint32_t(row >> P.tp_log2);
        r.ok = r.tstep < P.T && int64_t(gp) < P.npix;
        if (r.ok)
        {
            const uint32_t ohw = uint32_t(P.ohw), smp = gp / ohw, pix = gp - smp * ohw;
            r.sample = smp, r.pix = pix, r.img = int64_t(smp) * P.T + r.tstep;
            const int oy = int(pix / uint32_t(P.ow)), ox = int(pix) - oy * P.ow;
            r.iy0 = oy * P.sy - P.top;
            r.ix0 = ox * P.sx - P.left;
        }
        return r;
    }
    if (r.ok)
    {
        const int oy = int(r.pix / P.ow), ox = int(r.pix % P.ow);
        r.iy0 = oy * P.sy - P.top;
        r.ix0 = ox * P.sx - P.left;
    }
    return r;
}

// Raw bytes of four 8-wide K chunks of one A row (loads in flight until used).
struct Gathered
{
    uint2 v[4];
};

template <typename RI>
__device__ __forceinline__ void gather_load(const TcParams &P, const int4 *tab, const RI &r, const uint8_t *ib, int kb,
                                            int c_lo, Gathered &g)
{
    if (P.nhwc)
    {
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            const int4 t = tab[kb * 8 + c_lo + j];
            const int iy = r.iy0 + t.x, ix = r.ix0 + t.y;
            g.v[j] = make_uint2(0, 0);
            if (r.ok && t.w && iy >= 0 && iy < P.h && ix >= 0 && ix < P.w)
                g.v[j] = *reinterpret_cast<const uint2 *>(ib + int64_t(iy) * P.rs + int64_t(ix) * P.ps + t.z);
        }
    }
    else
    {
        const int64_t rowoff = int64_t(r.iy0) * P.rs + int64_t(r.ix0) * P.ps;
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            uint32_t w[2] = {0, 0};
#pragma unroll
            for (int e = 0; e < 8; ++e)
            {
                const int4 t = tab[kb * BK + (c_lo + j) * 8 + e];
                const int iy = r.iy0 + t.y, ix = r.ix0 + t.z;
                uint32_t b8 = 0;
                if (r.ok && t.w && iy >= 0 && iy < P.h && ix >= 0 && ix < P.w) b8 = ib[rowoff + t.x];
                w[e >> 2] |= b8 << (8 * (e & 3));
            }
            g.v[j] = make_uint2(w[0], w[1]);
        }
    }
}

__device__ __forceinline__ void gather_store(const TcParams &, const Gathered &g, unsigned char *a, int c_lo)
{
#pragma unroll
    for (int j = 0; j < 4; ++j) *reinterpret_cast<uint4 *>(a + (c_lo + j) * 128) = bf16x8_of_bytes(g.v[j]);
}

// ---- fused producers ---------------------------------------------------------
// A rows (pixel, t) of a fused tile from the first-spike map: a unit (pixel,
// 8-wide K chunk, R consecutive steps) loads the chunk's 8 first-spike bytes
// once (one 8-byte load channels-last, or 8 byte gathers when Cin < 8) and
// writes R rows of BF16 {0, 1}.  K order and table entries (c, ky, kx,
// valid) as the weight image.
struct FusedPixel
{
    bool ok;
    int64_t sample;
    int iy0, ix0;
};

// Table slot of K element (kb, kc, i) of the fused producers: the 8 lanes of
// a quarter warp read chunks kc = 0..7 of the same K block at once, so the
// chunks of a block sit in 8 different 16-byte bank groups (kc * (8 kblocks
// + 1) is kc mod 8).
__device__ __forceinline__ int ftab(int kblocks, int kb, int kc, int i)
{
    return kc * (8 * kblocks + 1) + i * kblocks + kb;
}

__device__ __forceinline__ FusedPixel fused_pixel(const TcParams &P, int64_t mt, int pl)
{
    // pixel indexes fit in 32 bits (checked on the host): 32-bit divisions
    FusedPixel u{};
    const uint32_t gp = uint32_t(mt) * uint32_t(P.pp) + uint32_t(pl);
    u.ok = int64_t(gp) < P.npix;
    if (u.ok)
    {
        const uint32_t ohw = uint32_t(P.ohw), smp = gp / ohw, pix = gp - smp * ohw;
        u.sample = smp;
        const int oy = int(pix / uint32_t(P.ow)), ox = int(pix) - oy * P.ow;
        u.iy0 = oy * P.sy - P.top;
        u.ix0 = ox * P.sx - P.left;
    }
    return u;
}

// First-spike bytes of K chunk (kb, kc) for a pixel; 0xFF = never.
__device__ __forceinline__ uint2 fst_chunk(const TcParams &P, const int4 *tab, const FusedPixel &u, int kb, int kc)
{
    if (!u.ok) return make_uint2(~0u, ~0u);
    const uint8_t *base = P.in + u.sample * P.img_stride;
    if (P.nhwc)
    {
        const int4 e = tab[ftab(P.kblocks, kb, kc, 0)];
        const int iy = u.iy0 + e.y, ix = u.ix0 + e.z;
        if (e.w && iy >= 0 && iy < P.h && ix >= 0 && ix < P.w)
            return *reinterpret_cast<const uint2 *>(base + (int64_t(iy) * P.w + ix) * P.cpad + e.x);
        return make_uint2(~0u, ~0u);
    }
    uint32_t w[2] = {0, 0};
#pragma unroll
    for (int i = 0; i < 8; ++i)
    {
        const int4 e = tab[ftab(P.kblocks, kb, kc, i)];
        const int iy = u.iy0 + e.y, ix = u.ix0 + e.z;
        uint32_t b = 0xFF;
        if (e.w && iy >= 0 && iy < P.h && ix >= 0 && ix < P.w) b = base[(int64_t(iy) * P.w + ix) * P.cin + e.x];
        w[i >> 2] |= b << (8 * (i & 3));
    }
    return make_uint2(w[0], w[1]);
}

__device__ __forceinline__ unsigned char *a_row_chunk(unsigned char *sA, int r, int kc)
{
    return sA + (r >> 3) * 1024 + (r & 7) * 16 + kc * 128;
}

// Rows t0 .. t0+R-1: byte b of the chunk is 1 where first-spike[b] <= t.
// (f | 0x80) - (t + 1) keeps bit 7 of a byte iff f > t, with no borrow
// between bytes since t + 1 <= 32.
// `rot` rotates the order of the R rows so that the 8 lanes of a quarter
// warp store to 8 different 16-byte bank groups.
__device__ __forceinline__ void store_fst_rows(unsigned char *sA, int row0, int t0, int R, int kc, uint2 f, int rot)
{
    const uint32_t lo = f.x | 0x80808080u, hi = f.y | 0x80808080u;
    for (int i0 = 0; i0 < R; ++i0)
    {
        const int i = (i0 + rot) & (R - 1);
        const uint32_t tt = uint32_t(t0 + i + 1) * 0x01010101u;
        const uint32_t sl = (~(lo - tt) >> 7) & 0x01010101u, sh = (~(hi - tt) >> 7) & 0x01010101u;
        uint4 v;
        v.x = __byte_perm(sl, 0, 0x7170) * 0x3F80u;
        v.y = __byte_perm(sl, 0, 0x7372) * 0x3F80u;
        v.z = __byte_perm(sh, 0, 0x7170) * 0x3F80u;
        v.w = __byte_perm(sh, 0, 0x7372) * 0x3F80u;
        *reinterpret_cast<uint4 *>(a_row_chunk(sA, row0 + i, kc)) = v;
    }
}

// Fallback rows gathered from the spikes themselves (any u8 values).
__device__ __forceinline__ void store_raw_rows(const TcParams &P, const int4 *tab, const FusedPixel &u,
                                               unsigned char *sA, int row0, int t0, int R, int kb, int kc)
{
    for (int i = 0; i < R; ++i)
    {
        const int t = t0 + i;
        uint32_t w[2] = {0, 0};
        if (u.ok && t < P.T)
        {
            const uint8_t *base = P.raw + (u.sample * P.T + t) * int64_t(P.cin) * P.h * P.w;
            for (int e8 = 0; e8 < 8; ++e8)
            {
                const int4 e = tab[ftab(P.kblocks, kb, kc, e8)];
                const int iy = u.iy0 + e.y, ix = u.ix0 + e.z;
                uint32_t b = 0;
                if (e.w && iy >= 0 && iy < P.h && ix >= 0 && ix < P.w)
                    b = base[(int64_t(e.x) * P.h + iy) * P.w + ix];
                w[e8 >> 2] |= b << (8 * (e8 & 3));
            }
        }
        *reinterpret_cast<uint4 *>(a_row_chunk(sA, row0 + i, kc)) = bf16x8_of_bytes(make_uint2(w[0], w[1]));
    }
}

// Fused producer loop of thread p (0..255) with NU unit slots (units per
// thread: 1 when a unit covers 4 steps, up to 4 for T <= 2).
template <int NU>
__device__ __forceinline__ void fused_producer(const TcParams &P, const int4 *tab, unsigned char *smem,
                                               uint64_t *full_bar, uint64_t *empty_bar, int S, int stage_bytes,
                                               int a_bytes, int b_bytes, int p)
{
    const int TP = 1 << P.tp_log2, R = TP < 4 ? TP : 4, G = TP / R;
    const int units = P.pp * 8 * G;  // 1024 / R
    const bool raw = *P.flag != 0;
    int upl[NU], ukc[NU], ug[NU];
#pragma unroll
    for (int i = 0; i < NU; ++i)
    {
        const int q = p + i * 256;
        ug[i] = q % G, ukc[i] = (q / G) & 7, upl[i] = q / (G * 8);
    }
    uint32_t it = 0;
    bool failed = false;
    for (int64_t tile = blockIdx.x; tile < P.tiles && !failed; tile += gridDim.x)
    {
        FusedPixel fu[NU];
#pragma unroll
        for (int i = 0; i < NU; ++i)
            if (p + i * 256 < units) fu[i] = fused_pixel(P, tile, upl[i]);
        const uint8_t *wbase = P.wimg;
        if (P.snet) wbase += P.snet[(uint32_t(tile) * uint32_t(P.pp)) / uint32_t(P.ohw)] * P.wimg_stride;
        for (int kb = 0; kb < P.kblocks; ++kb, ++it)
        {
            // the loads are in flight while waiting for the stage
            uint2 f[NU];
            if (!raw)
#pragma unroll
                for (int i = 0; i < NU; ++i)
                    if (p + i * 256 < units) f[i] = fst_chunk(P, tab, fu[i], kb, ukc[i]);
            const int s = int(it % uint32_t(S));
            const uint32_t u = it / uint32_t(S);
            if (u > 0 && !wait_bounded(&empty_bar[s], (u - 1) & 1))
            {
                failed = true;
                break;
            }
            unsigned char *sA = smem + s * stage_bytes;
            if (p == 0)
            {
                arrive_expect_tx(&full_bar[s], uint32_t(b_bytes));
                bulk_g2s(sA + a_bytes, wbase + int64_t(kb) * b_bytes, uint32_t(b_bytes), &full_bar[s]);
            }
#pragma unroll
            for (int i = 0; i < NU; ++i)
                if (p + i * 256 < units)
                {
                    const int row0 = upl[i] * TP + ug[i] * R, t0 = ug[i] * R;
                    if (raw)
                        store_raw_rows(P, tab, fu[i], sA, row0, t0, R, kb, ukc[i]);
                    else
                        store_fst_rows(sA, row0, t0, R, ukc[i], f[i], (ug[i] >> 1) + 2 * (ukc[i] & 1));
                }
            fence_proxy_async_smem();
            mbar_arrive(&full_bar[s]);
        }
    }
}

// ---- lean first-crossing search (kSearch) ------------------------------------
// With no negative weight and cumulative 0/1 input spikes every potential
// V_c(t) is non-decreasing in t.  When the thresholds satisfy
// value <= inhibit, fire, WTA thresholds <= threshold, each of those tests on
// the thresholded potential is the test V_c(t) > threshold, so one output
// pixel is fixed by t0, the first step at which some channel exceeds the
// threshold, and by w, the first channel of largest potential at t0
// (cpu/inhibit.cpp:41-121 takes the winner at step T - #steps above):
//   spikes   channel w from t0 to T - 1, nothing else (cpu/fire.cpp:67-82);
//   record   (w, t0, V_w(t0)), the WTA key of cpu/wta.cpp:53-62;
//   min/max  0 from the losing channels, `value` below the threshold, and
//            V_w(T - 1) as the sample's largest inhibited potential.
// A pixel with nothing above the threshold at T - 1 never fires (record
// (0, T, value)).  The search evaluates one (pixel, step) row per pixel and
// round: round 0 every pixel at T - 1, then a bisection of (lo, hi] over the
// crossing pixels, then (with WTA) V_w(T - 1) where w is not also the
// largest channel at T - 1.  ceil(log2 T) + 2 rows at most per crossing
// pixel against T for the dense layer.
//
// Every decision is the oracle's: the potential of a row is the F32 rounding
// of the FP64 sum of its products in (channel, ky, kx) order.  The weights
// are split on fixed per-channel grids (fixed_split_kernel), so each
// tensor-memory sum is exact and their total r_q is within echan[c] of the
// oracle's FP64 sum.  Tier 1 adds the terms in FP32 and decides when the
// rigorous bound 3.125 * 2^-24 |f| + c0 separates the largest potential from
// the threshold and from the runner-up by more than an ulp; the winner's
// value is then r_q rounded once, kept when r_q +- echan stays inside that
// float's rounding interval.  Tier 2 (rows tier 1 leaves open) does the same
// for every channel of the row and decides on the exact values, with the
// possible neighbours of each uncertified one.  Rows still open go to
// search_fix_kernel, which recomputes them as the oracle does.
template <int NS>
__device__ __forceinline__ void s_chunk(uint32_t lane_base, int c0, int n_tile, uint32_t (&q)[NS][kEpiChunk])
{
#pragma unroll
    for (int j = 0; j < NS; ++j) tmem_ld8(lane_base + uint32_t(j * n_tile + c0), q[j]);
}

template <int NS>
__device__ __forceinline__ void s_chunk_wait(uint32_t (&q)[NS][kEpiChunk])
{
#pragma unroll
    for (int j = 0; j < NS; ++j) tmem_ld_wait8(q[j]);
}

// Exact term total of a column: the NS 32-bit accumulators hold sums of
// base-256 digit products, so the total is an integer below 2^46.
template <int NS>
__device__ __forceinline__ uint64_t s_total(const uint32_t (&q)[NS][kEpiChunk], int j)
{
    uint64_t r = 0;
#pragma unroll
    for (int i = 0; i < NS; ++i) r = (r << 8) + uint64_t(q[i][j]);
    return r;
}

// The floats a potential within E of the exact S (= R * scale) can round to:
// [lo, hi] = [RN(S - E), RN(S + E)] (RN is monotone); lo == hi: P is the
// oracle's value.  E == 0: the term total is the oracle's FP64 sum itself.
__device__ __forceinline__ void s_round(double S, float E, float &P, float &lo, float &hi)
{
    P = float(S);
    if (E == 0.f)
    {
        lo = hi = P;
        return;
    }
    lo = float(__dsub_rd(S, double(E)));
    hi = float(__dadd_ru(S, double(E)));
}

// Exact term total of column `col` of this lane's row (col < 0: none), the
// warp's columns fetched one 8-column chunk at a time.  Warp-uniform.
template <int NS>
__device__ __forceinline__ uint64_t s_reload(uint32_t lane_base, int n_tile, int col)
{
    uint64_t R = 0;
    unsigned pending = __ballot_sync(0xffffffffu, col >= 0);
    while (pending)
    {
        const int c0 = (__shfl_sync(0xffffffffu, col, __ffs(pending) - 1) >> 3) << 3;
        uint32_t q[NS][kEpiChunk];
        s_chunk<NS>(lane_base, c0, n_tile, q);
        s_chunk_wait<NS>(q);
        const bool mine = col >= 0 && (col >> 3) == (c0 >> 3);
        const int jj = col - c0;
#pragma unroll
        for (int j = 0; j < kEpiChunk; ++j) R = (mine && jj == j) ? s_total<NS>(q, j) : R;
        pending &= ~__ballot_sync(0xffffffffu, mine);
    }
    return R;
}

// Tier 2: every channel of the row from its exact total.  dec: 0 open, 1 no
// channel above thr, 2 crossing with winner a (first of the largest) of value v.
template <int NS>
__device__ __forceinline__ void s_tier2(const TcParams &P, uint32_t lane_base, float thr, int &dec, int &a, float &v,
                                        const float *scale, const float *bound)
{
    float mlo = -INFINITY, hmax = -INFINITY, hun = -INFINITY, vs = -INFINITY;
    int as = -1;
    for (int c0 = 0; c0 < P.n_tile; c0 += kEpiChunk)
    {
        uint32_t q[NS][kEpiChunk];
        s_chunk<NS>(lane_base, c0, P.n_tile, q);
        s_chunk_wait<NS>(q);
#pragma unroll
        for (int j = 0; j < kEpiChunk; ++j)
        {
            const int c = c0 + j;
            const bool real = c < P.cout;
            float pc, lo, hi;
            const double S = double(s_total<NS>(q, j)) * double(real ? scale[c] : 0.f);
            s_round(S, real ? bound[c] : 0.f, pc, lo, hi);
            if (!real) lo = hi = pc = -INFINITY;
            mlo = fmaxf(mlo, lo);
            hmax = fmaxf(hmax, hi);
            const bool exact = lo == hi;
            const bool better = exact && pc > vs;
            vs = better ? pc : vs;
            as = better ? c : as;
            hun = exact ? hun : fmaxf(hun, hi);
        }
    }
    dec = 0;
    if (mlo > thr)
    {
        // the winner is among the channels that can reach mlo: decided when
        // all of them are exact
        if (hun < mlo && as >= 0) dec = 2, a = as, v = vs;
    }
    else if (hmax <= thr)
        dec = 1;
}

// The largest float any channel of value P (its exact total within the
// rounding cell of P) can round to when the oracle's sum is within E of it.
__device__ __forceinline__ float s_upper(float P, float E)
{
    const double up = double(P) + 0.5 * (double(nextafterf(P, INFINITY)) - double(P));
    return float(__dadd_ru(up, double(E)));
}

// What a decided row does to its pixel (shared by the epilogue and the exact
// recompute).  Returns the list entries to append and the sample maximum to
// raise.
struct SearchAct
{
    bool next = false, fin = false, max = false, thv = false;
    int2 next_e, fin_e;
    float maxv = 0.f;
};

__device__ __forceinline__ int4 s_pack(int lo, int hi, int w, float v, int at, float vt)
{
    return make_int4((lo & 0xFF) | ((hi & 0xFF) << 8) | (w << 16), __float_as_int(v), at, __float_as_int(vt));
}

__device__ __forceinline__ SearchAct search_act(const TcParams &P, int round, int pix, int t, int dec, int a,
                                                float v, int4 s)
{
    SearchAct r;
    const int T = P.T;
    if (round == 2)
    {
        r.max = true, r.maxv = v;
        return r;
    }
    int lo, hi, w, at;
    float vh, vt;
    if (round == 0)
    {
        if (dec == 1)
        {
            P.records[pix] = make_int4(0, T, __float_as_int(P.thv), 0);
            r.thv = true;
            return r;
        }
        lo = (P.tlo ? int(P.tlo[pix]) : 0) - 1, hi = T - 1, w = a, vh = v, at = a, vt = v;
    }
    else
    {
        lo = int(int8_t(s.x & 0xFF)), hi = int(int8_t((s.x >> 8) & 0xFF)), w = s.x >> 16;
        vh = __int_as_float(s.y), at = s.z, vt = __int_as_float(s.w);
        if (dec == 2)
            hi = t, w = a, vh = v;
        else
            lo = t;
    }
    if (hi - lo > 1)
    {
        P.state[pix] = s_pack(lo, hi, w, vh, at, vt);
        r.next = true, r.next_e = make_int2(pix, (lo + hi) >> 1);
        return r;
    }
    // t0 = hi: the pixel is settled
    P.records[pix] = make_int4(w, hi, __float_as_int(vh), 0);
    if (P.wta)
    {
        r.thv = hi > 0;
        if (w == at)
            r.max = true, r.maxv = vt;
        else
            r.fin = true, r.fin_e = make_int2(pix, w);
    }
    return r;
}

// A row's next-round entry (valid: it has a step) counted into its
// compaction block, one atomic per block a warp's entries fall in.  Every
// lane of the warp calls it.
__device__ __forceinline__ void list_count_warp(int *bc, int idx, bool valid)
{
    const int key = valid ? (idx >> kCompactShift) : -1;
    const unsigned grp = __match_any_sync(0xffffffffu, key);
    if (valid && int(threadIdx.x & 31) == __ffs(int(grp)) - 1) atomicAdd(bc + key, __popc(grp));
}

__device__ __forceinline__ void s_extremes(const TcParams &P, int pix, const SearchAct &r)
{
    const int smp = int(div_by(uint32_t(pix), P.ohw_m, P.ohw_sh));
    if (r.max) atomicMax(P.maxs + smp, order_enc(r.maxv));
    if (r.thv && P.thv != 0.f)
    {
        atomicMin(P.mins + smp, order_enc(P.thv));
        atomicMax(P.maxs + smp, order_enc(P.thv));
    }
}

// Search epilogue of one row per thread (warps 0-3).  `emax` is the largest
// channel bound.  Tier 1 scans the row: each channel's exact total R, its
// float P = RN(R) * 2^(e - 32) (exact scaling by the channel's power of two),
// the three largest (first index first).  The winner's value and, when the
// runner-up is within two ulps, the runner-up's, are certified against their
// channel bounds; nothing else can change a decision unless the third value
// comes that close too.
// Running state of a row's scan over the channel parts of a tile: the three
// largest potentials, the channels of the first two and their term totals
// (r1 also carries the winner's total in the last round).
struct SearchScan
{
    float p1 = -INFINITY, p2 = -INFINITY, p3 = -INFINITY;
    int a1 = -1, a2 = -1;
    uint64_t r1 = 0, r2 = 0;
};

template <int NS>
__device__ void search_epilogue(const TcParams &P, uint32_t acc, bool ok, int pix, int t, int aux, int4 pstate,
                                uint64_t *release, float emax, const float *scale, const float *bound, int idx,
                                int part, SearchScan &sc)
{
    const int warp = threadIdx.x >> 5;
    const uint32_t lane_base = acc + (uint32_t((warp & 3) * 32) << 16);
    const float thr = P.thr;
    const bool last = part == P.nparts - 1;
    const int cg = part * P.n_tile;  // first channel of this part
    int dec = 0, a = -1;
    float v = 0.f;
    if (P.round == 2)
    {
        const int col = (ok && aux >= cg && aux < cg + P.n_tile) ? aux - cg : -1;
        const uint64_t R = s_reload<NS>(lane_base, P.n_tile, col);
        if (col >= 0) sc.r1 = R;
        tc_fence_before();
        mbar_arrive(release);
        if (!last) return;
        if (ok)
        {
            float lo, hi;
            s_round(double(sc.r1) * double(scale[aux]), bound[aux], v, lo, hi);
            dec = lo == hi ? 2 : 3;
            a = aux;
        }
    }
    else
    {
        float &p1 = sc.p1, &p2 = sc.p2, &p3 = sc.p3;
        int &a1 = sc.a1, &a2 = sc.a2;
        uint64_t &r1 = sc.r1, &r2 = sc.r2;
        for (int cb = 0; cb < P.n_tile; cb += kEpiChunk)
        {
            uint32_t q[NS][kEpiChunk];
            s_chunk<NS>(lane_base, cb, P.n_tile, q);
            s_chunk_wait<NS>(q);
            const int lim = P.cout - cg - cb;
#pragma unroll
            for (int j = 0; j < kEpiChunk; ++j)
            {
                const uint64_t R = s_total<NS>(q, j);
                const int c = cg + cb + j;
                const float pv = j < lim ? __ll2float_rn((long long)R) * scale[c] : -INFINITY;
                const bool g1 = pv > p1, g2 = !g1 && pv > p2, g3 = !g1 && !g2 && pv > p3;
                p3 = g1 || g2 ? p2 : (g3 ? pv : p3);
                p2 = g1 ? p1 : (g2 ? pv : p2);
                a2 = g1 ? a1 : (g2 ? c : a2);
                r2 = g1 ? r1 : (g2 ? R : r2);
                p1 = g1 ? pv : p1;
                a1 = g1 ? c : a1;
                r1 = g1 ? R : r1;
            }
        }
        if (!last)
        {
            tc_fence_before();
            mbar_arrive(release);
            return;
        }
        int d1 = 0;  // tier-1 decision: 0 open, 1 below, 2 winner decided (value certified or not)
        bool vexact = false;
        if (ok)
        {
            if (s_upper(p1, emax) <= thr)
                d1 = 1;  // no channel's value can round above the threshold
            else
            {
                float pa, lo1, hi1;
                s_round(double(r1) * double(scale[a1]), bound[a1], pa, lo1, hi1);
                const float near = nextafterf(nextafterf(p1, -INFINITY), -INFINITY);
                if (lo1 > thr && !(p3 >= near && s_upper(p3, emax) >= lo1))
                {
                    bool win = true;
                    if (p2 >= near && s_upper(p2, emax) >= lo1)
                    {
                        float pb, lo2, hi2;
                        s_round(double(r2) * double(scale[a2]), bound[a2], pb, lo2, hi2);
                        // both exact: the larger wins, ties to the lower index (a1)
                        win = lo1 > hi2 || (lo1 == hi1 && lo2 == hi2 && pa >= pb);
                    }
                    if (win) d1 = 2, vexact = lo1 == hi1, v = pa;
                }
            }
        }
        int d2 = 0, a2t = -1;
        float v2 = 0.f;
        const unsigned open1 = __ballot_sync(0xffffffffu, ok && d1 == 0);
        // tier 2 reads every channel from tensor memory: one part only (with
        // several, the row goes to the exact recompute)
        if (open1 && P.nparts == 1)
        {
            if ((threadIdx.x & 31) == 0) atomicAdd(&g_rechecks, (unsigned long long)__popc(open1));
            s_tier2<NS>(P, lane_base, thr, d2, a2t, v2, scale, bound);
        }
        tc_fence_before();
        mbar_arrive(release);
        if (ok)
        {
            if (d1 == 1)
                dec = 1;
            else if (d1 == 2)
                a = a1, dec = vexact ? 2 : 3;
            else
                dec = d2, a = a2t, v = v2;
        }
    }
    // dec 3: the winner a is decided, its value is left to the exact sum
    SearchAct r;
    if (ok && (dec == 1 || dec == 2)) r = search_act(P, P.round, pix, t, dec, a, v, pstate);
    // a decided row writes its pixel's entry of the next round at its own
    // index (the next step, or -1 when the pixel is settled; a compaction
    // keeps the list in pixel order); rows left open are written by the
    // exact recompute.  The rarer lists take one atomic per warp each, all
    // in flight at once.
    if (ok && P.round != 2 && (dec == 1 || dec == 2)) P.list_out[idx] = r.next ? r.next_e : make_int2(pix, -1);
    if (P.round != 2) list_count_warp(P.list_bc, idx, ok && (dec == 1 || dec == 2) && r.next);
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const bool wf = ok && dec == 0, wv = ok && dec == 3;
    const unsigned mf = __ballot_sync(0xffffffffu, wf), mv = __ballot_sync(0xffffffffu, wv);
    const unsigned mi = __ballot_sync(0xffffffffu, r.fin);
    int bf = 0, bv = 0, bi = 0;
    if (lane == 0)
    {
        if (mf) bf = atomicAdd(P.fix_count, __popc(mf));
        if (mv) bv = atomicAdd(P.val_count, __popc(mv));
        if (mi) bi = atomicAdd(P.final_count, __popc(mi));
    }
    bf = __shfl_sync(0xffffffffu, bf, 0) + __popc(mf & below);
    bv = __shfl_sync(0xffffffffu, bv, 0) + __popc(mv & below);
    bi = __shfl_sync(0xffffffffu, bi, 0) + __popc(mi & below);
    if (wf) P.fix_list[bf] = make_int4(pix, t, idx, aux);
    if (wv) P.val_list[bv] = make_int4(pix, t, idx, a);
    if (r.fin) P.final_list[bi] = r.fin_e;
    if (P.wta)
    {
        // the sample maxima: one atomic per sample among the warp's lanes
        const int smp = ok ? pix / int(P.ohw) : -1;
        const bool has = ok && r.max;
        const unsigned key = has ? unsigned(smp) : 0xFFFFFFFFu;
        const unsigned peers = __match_any_sync(0xffffffffu, key);
        const unsigned enc = has ? order_enc(r.maxv) : 0u;
        const unsigned best = __reduce_max_sync(peers, enc);
        if (has && lane == __ffs(peers) - 1) atomicMax(P.maxs + smp, best);
        if (ok && r.thv && P.thv != 0.f)
        {
            atomicMin(P.mins + smp, order_enc(P.thv));
            atomicMax(P.maxs + smp, order_enc(P.thv));
        }
    }
}

// A search row's pixel in three words: byte offset of its sample's
// first-spike map (-1: no row), receptive-field origin (iy0, ix0) packed as
// two 16-bit fields, and its step.  The search operands are 8-bit and
// channels-last: a 16-byte chunk of a row is two 8-channel groups, each 8
// bytes of the first-spike map (0xFF: outside the input).

// Bytes 1 where the first-spike byte f <= t, else 0; tt = (t + 1) * 0x01010101
// ((f | 0x80) - (t + 1) keeps bit 7 iff f > t, no borrow between bytes).
__device__ __forceinline__ uint32_t spike_bytes(uint32_t f, uint32_t tt)
{
    return (~((f | 0x80808080u) - tt) >> 7) & 0x01010101u;
}

// 8-channel group g of a search row (tab entry: first channel, ky, kx,
// valid); 0xFF bytes outside the input.
__device__ __forceinline__ uint2 fst_group(const TcParams &P, const int4 *tab, int base, int yx, int g)
{
    if (base < 0) return make_uint2(~0u, ~0u);
    const int iy0 = int(uint32_t(yx) >> 16) - 32768, ix0 = int(uint32_t(yx) & 0xFFFFu) - 32768;
    const int4 e = tab[g];
    const int iy = iy0 + e.y, ix = ix0 + e.z;
    if (e.w && iy >= 0 && iy < P.h && ix >= 0 && ix < P.w)
        return __ldg(reinterpret_cast<const uint2 *>(P.in + base + (iy * P.w + ix) * P.cpad + e.x));
    return make_uint2(~0u, ~0u);
}

// The list entries of the rows a thread with kc == 0 covers in `tile`, copied
// into `buf` (128 entries, by row) asynchronously.
template <int NU>
__device__ __forceinline__ void entry_prefetch(const TcParams &P, int2 *buf, int64_t tile, int row0, int rs,
                                               int64_t nrows)
{
#pragma unroll
    for (int i = 0; i < NU; ++i)
    {
        const int64_t idx = tile * BM + row0 + rs * i;
        if (idx < nrows) cp_async8(buf + row0 + rs * i, P.list_in + idx);
    }
    cp_async_commit();
}

// Search producers: a thread builds NU (row, 16-byte chunk) units of every K
// block (128 U8 elements), one row each at that row's own step.  Unit i of
// thread p is row (p & 7) + 8 (p >> 6) + (1024 / NU / 8) i and chunk
// (p >> 3) & 7, so the 8 lanes of a quarter warp take 8 consecutive rows of
// one chunk (distinct 16-byte bank groups).  The gathers of a step are issued
// before the wait for its stage, all in flight together.  (Copying them into
// the stage with 8-byte cp.async and converting in place one step later
// measured slower: the per-copy issue cost outweighed the deeper pipeline.)
// In rounds with a row list the threads with kc == 0
// (together one per row) fetch the next tile's list entries into shared
// memory (cp.async) while the current tile is built, so their latency leaves
// the per-tile chain; every producer thread reads them after an mbarrier of
// the NT producers (two buffers, by tile parity).
template <int NU>
__device__ __forceinline__ void search_producer(const TcParams &P, const int4 *tab, unsigned char *smem,
                                                uint64_t *full_bar, uint64_t *empty_bar, int S, int stage_bytes,
                                                int a_bytes, int b_bytes, int p, int64_t nrows, int64_t ntiles,
                                                int2 *s_ent, uint64_t *ent_bar, int *s_tiles, uint64_t *tq_bar)
{
    constexpr int NT = 1024 / NU, RS = NT / 8;  // producer threads; row step between a thread's units
    const int row0 = (p & 7) + 8 * (p >> 6), kc = (p >> 3) & 7;
    if (int64_t(blockIdx.x) >= ntiles) return;
    const bool listed = !(P.round == 0 && !P.r0_list);
    const bool dyn = P.tile_ctr != nullptr;
    int ticket = 0;  // (thread 0) the claimed ticket of the tile after the next one
    if (p == 0)
    {
        s_tiles[0] = int(blockIdx.x);
        mbar_arrive(&tq_bar[0]);
        if (dyn) ticket = atomicAdd(P.tile_ctr, 1);
    }
    if (listed && kc == 0) entry_prefetch<NU>(P, s_ent, blockIdx.x, row0, RS, nrows);
    int ss = 0;  // the stage ring: slot and pass of the next K block
    uint32_t su = 0;
    int64_t tile = blockIdx.x;
    for (uint32_t k = 0;; ++k)
    {
        const int cb = int(k & 1);
        // thread 0 publishes the tile after this one in the ring (-1: none)
        if (p == 0)
        {
            const int64_t nt = dyn ? int64_t(gridDim.x) + ticket : tile + gridDim.x;
            s_tiles[(k + 1) & 15] = nt < ntiles ? int(nt) : -1;
            mbar_arrive(&tq_bar[(k + 1) & 15]);
        }
        if (listed && kc == 0) cp_async_wait_all();
        mbar_arrive(&ent_bar[cb]);
        if (!wait_bounded(&ent_bar[cb], (k >> 1) & 1)) return;
        // every thread has read the other entry buffer (the previous tile's)
        // and sees the next tile
        const int next = s_tiles[(k + 1) & 15];
        if (p == 0 && dyn && next >= 0) ticket = atomicAdd(P.tile_ctr, 1);
        if (listed && kc == 0 && next >= 0) entry_prefetch<NU>(P, s_ent + (cb ^ 1) * BM, next, row0, RS, nrows);
        int ubase[NU], uyx[NU];
        uint32_t utt[NU];
#pragma unroll
        for (int i = 0; i < NU; ++i)
        {
            const int64_t idx = tile * BM + row0 + RS * i;
            ubase[i] = -1, uyx[i] = 0, utt[i] = 0x01010101u;
            if (idx < nrows)
            {
                int2 e = make_int2(int(idx), P.T - 1);
                if (listed)
                {
                    e = s_ent[cb * BM + row0 + RS * i];
                    if (P.round != 1) e.y = P.T - 1;
                }
                const uint32_t smp = div_by(uint32_t(e.x), P.ohw_m, P.ohw_sh);
                const uint32_t pix = uint32_t(e.x) - smp * uint32_t(P.ohw);
                const int oy = int(div_by(pix, P.ow_m, P.ow_sh)), ox = int(pix) - oy * P.ow;
                ubase[i] = int(int64_t(smp) * P.img_stride);
                uyx[i] = int((uint32_t(oy * P.sy - P.top + 32768) << 16) | uint32_t(ox * P.sx - P.left + 32768));
                utt[i] = uint32_t(e.y + 1) * 0x01010101u;
            }
        }
        for (int part = 0; part < P.nparts; ++part)
            for (int kb = 0; kb < P.kblocks; ++kb)
            {
                uint2 fa[NU], fb[NU];
#pragma unroll
                for (int i = 0; i < NU; ++i)
                {
                    fa[i] = fst_group(P, tab, ubase[i], uyx[i], kb * 16 + 2 * kc);
                    fb[i] = fst_group(P, tab, ubase[i], uyx[i], kb * 16 + 2 * kc + 1);
                }
                const int s = ss;
                if (su > 0 && !wait_bounded(&empty_bar[s], (su - 1) & 1)) return;
                unsigned char *sA = smem + s * stage_bytes;
                if (p == 0)
                {
                    arrive_expect_tx(&full_bar[s], uint32_t(b_bytes));
                    bulk_g2s(sA + a_bytes, P.wimg + (int64_t(part) * P.kblocks + kb) * b_bytes, uint32_t(b_bytes),
                             &full_bar[s]);
                }
#pragma unroll
                for (int i = 0; i < NU; ++i)
                    *reinterpret_cast<uint4 *>(a_row_chunk(sA, row0 + RS * i, kc)) =
                        make_uint4(spike_bytes(fa[i].x, utt[i]), spike_bytes(fa[i].y, utt[i]),
                                   spike_bytes(fb[i].x, utt[i]), spike_bytes(fb[i].y, utt[i]));
                fence_proxy_async_smem();
                mbar_arrive(&full_bar[s]);
                if (++ss == S) ss = 0, ++su;
            }
        if (next < 0) break;
        tile = next;
    }
}

// Warp-specialised persistent kernel (416 threads):
//   warps 4-11 producers: per K block, wait for a free stage, bulk-copy the
//              weight block (thread 128) and gather half an A row each;
//   warp 12    one thread issues the tcgen05.mma of every stage into one of
//              (up to) two tensor-memory accumulators and commits;
//   warps 0-3  epilogue: read the accumulator of a finished tile (one row per
//              thread) while the next tile is being multiplied.
// Stage ring: full[s] (256 producer arrivals + the weight bytes), empty[s]
// (MMA commit); accumulators: acc_full[a] (MMA commit), acc_empty[a] (128
// epilogue arrivals).  Every wait is bounded; a timeout raises the device
// status word and makes every role leave.
//
// The search kernel (kSearch) runs with 4 producer warps (288 threads) so
// that two CTAs fit on an SM where their tensor memory allows: its
// per-tile work is latency-bound, and a second CTA hides those latencies.
constexpr int kWsThreads = 416, kSearchThreads = 288, kMaxStages = 6;

template <int MODE, int NPW>
__device__ __forceinline__ void conv_ws_body(const TcParams &P)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t full_bar[kMaxStages], empty_bar[kMaxStages], accf_bar[2], acce_bar[2], tim_bar,
        ent_bar[2], tq_bar[16];
    // search: the CTA's tiles in order (slot k & 15 holds its k-th tile, -1
    // after the last), each published by a producer arrival on tq_bar
    __shared__ int s_tiles[16];
    __shared__ uint32_t tmem_slot;

    // the search kernels run only on the lean path, the dense fused kernel
    // only off it (both words are set before the launch; uniform exit)
    if constexpr (MODE == kSearch)
    {
        if (*P.negw || *P.flag) return;
    }
    if constexpr (MODE == kFused)
    {
        if (P.skip_when_lean && !*P.negw && !*P.flag) return;
    }
    int64_t nrows = 0, ntiles = P.tiles;
    if constexpr (MODE == kSearch)
    {
        nrows = (P.round == 0 && !P.r0_list) ? P.npix : int64_t(*P.count_in);
        ntiles = ceil_div(nrows, BM);
    }
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int S = P.stages, nacc = P.nacc;
    const int a_bytes = BM * BK * 2;
    const int b_bytes = P.nsplit * P.n_tile * BK * 2;
    const int stage_bytes = a_bytes + b_bytes;
    int4 *tab = reinterpret_cast<int4 *>(smem + S * stage_bytes);
    const int taps = P.kh * P.kw;
    // search: the channels' scales and bounds, staged after the table
    const int nch = MODE == kSearch ? P.nparts * P.n_tile : P.n_tile;  // channels of the tables
    float *s_scale = reinterpret_cast<float *>(tab + P.kblocks * 16), *s_bound = s_scale + nch;
    // search: two buffers of the next tile's list entries (128 each)
    int2 *s_ent = reinterpret_cast<int2 *>(s_bound + nch + ((16 - ((2 * nch) & 15)) & 15));
    if constexpr (MODE == kSearch)
    {
        // per 8-element group of a 128-element K block (channels-last, 8-bit
        // operands): (first channel, ky, kx, valid)
        for (int g = tid; g < P.kblocks * 16; g += blockDim.x)
        {
            const int k = g * 8, tap = k / P.cpad, c = k % P.cpad;
            tab[g] = make_int4(c, tap / P.kw, tap % P.kw, (tap < taps && c < P.cin) ? 1 : 0);
        }
        for (int c = tid; c < nch; c += blockDim.x) s_scale[c] = P.cscale[c], s_bound[c] = P.echan[c];
    }
    else if constexpr (MODE != kPotentials)
    {
        // per K element: (channel, ky, kx, valid) in the weight image's order
        for (int k = tid; k < P.kblocks * BK; k += blockDim.x)
        {
            int c, tap;
            if (P.nhwc)
                tap = k / P.cpad, c = k % P.cpad;
            else
                c = k / taps, tap = k % taps;
            tab[ftab(P.kblocks, k / BK, (k / 8) % 8, k % 8)] =
                make_int4(c, tap / P.kw, tap % P.kw, (tap < taps && c < P.cin) ? 1 : 0);
        }
    }
    else if (P.nhwc)
    {
        const int groups = P.cpad / 8;
        for (int q = tid; q < P.kblocks * 8; q += blockDim.x)
        {
            const int tap = q / groups, g = q % groups;
            tab[q] = make_int4(tap / P.kw, tap % P.kw, g * 8, tap < taps ? 1 : 0);
        }
    }
    else
    {
        for (int k = tid; k < P.kblocks * BK; k += blockDim.x)
        {
            const int c = k / taps, tap = k % taps, ky = tap / P.kw, kx = tap % P.kw;
            tab[k] = make_int4(int(c * P.cs + ky * P.rs + kx * P.ps), ky, kx, c < P.cin ? 1 : 0);
        }
    }
    if (tid == 0)
    {
        for (int s = 0; s < S; ++s)
            mbar_init(&full_bar[s], 1 + 32 * NPW), mbar_init(&empty_bar[s], 1);
        for (int a = 0; a < 2; ++a) mbar_init(&accf_bar[a], 1), mbar_init(&acce_bar[a], 128);
        mbar_init(&tim_bar, 128);
        for (int b = 0; b < 2; ++b) mbar_init(&ent_bar[b], 32 * NPW);
        for (int q = 0; q < 16; ++q) mbar_init(&tq_bar[q], 1);
        fence_mbar_init();
    }
    if (warp == 0)
    {
        tmem_alloc(&tmem_slot, P.tmem_cols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    const int acc_cols = P.nsplit * P.n_tile;

    constexpr int kMmaWarp = 4 + NPW;
    if (MODE == kSearch && warp >= 4 && warp < kMmaWarp)
        search_producer<1024 / (32 * NPW)>(P, tab, smem, full_bar, empty_bar, S, stage_bytes, a_bytes, b_bytes,
                                           tid - 128, nrows, ntiles, s_ent, ent_bar, s_tiles, tq_bar);
    else if (MODE != kPotentials && MODE != kSearch && warp >= 4 && warp < kMmaWarp)
    {
        // ---------------- fused producers (8 warps) ----------------
        if (P.tp_log2 >= 2)
            fused_producer<1>(P, tab, smem, full_bar, empty_bar, S, stage_bytes, a_bytes, b_bytes, tid - 128);
        else
            fused_producer<4>(P, tab, smem, full_bar, empty_bar, S, stage_bytes, a_bytes, b_bytes, tid - 128);
    }
    else if (MODE == kPotentials && warp >= 4 && warp < kMmaWarp)
    {
        // ---------------- producers (8 warps) ----------------
        // Thread p gathers K chunks c_lo..c_lo+3 of row prow.  The loads of the
        // next K block are issued before waiting for a free stage, so the
        // gather latency overlaps the wait and the previous block's stores.
        const int p = tid - 128;
        const int prow = p & (BM - 1), c_lo = (p >> 7) * 4;
        uint32_t it = 0;
        int64_t tile = blockIdx.x;
        int kb = 0;
        if (tile < P.tiles)
        {
            RowInfo r = row_info<MODE>(P, tile / P.n_tiles, prow);
            const uint8_t *ib = (MODE == kPotentials) ? P.in + r.img * P.img_stride
                                                      : P.in + r.sample * P.img_stride + r.tstep * P.ts;
            Gathered cur;
            gather_load(P, tab, r, ib, kb, c_lo, cur);
            while (true)
            {
                // next (tile, k block) and its loads
                int64_t ntile = tile;
                int nkb = kb + 1;
                if (nkb == P.kblocks) nkb = 0, ntile += gridDim.x;
                const bool more = ntile < P.tiles;
                RowInfo nr = r;
                const uint8_t *nib = ib;
                Gathered nxt;
                if (more)
                {
                    if (ntile != tile)
                    {
                        nr = row_info<MODE>(P, ntile / P.n_tiles, prow);
                        nib = (MODE == kPotentials) ? P.in + nr.img * P.img_stride
                                                    : P.in + nr.sample * P.img_stride + nr.tstep * P.ts;
                    }
                    gather_load(P, tab, nr, nib, nkb, c_lo, nxt);
                }
                const int s = int(it % uint32_t(S));
                const uint32_t u = it / uint32_t(S);
                if (u > 0 && !wait_bounded(&empty_bar[s], (u - 1) & 1)) break;
                unsigned char *sA = smem + s * stage_bytes;
                if (p == 0)
                {
                    const int nt = int(tile % P.n_tiles);
                    arrive_expect_tx(&full_bar[s], uint32_t(b_bytes));
                    bulk_g2s(sA + a_bytes, P.wimg + (int64_t(nt) * P.kblocks + kb) * b_bytes, uint32_t(b_bytes),
                             &full_bar[s]);
                }
                gather_store(P, cur, sA + (prow >> 3) * 1024 + (prow & 7) * 16, c_lo);
                fence_proxy_async_smem();
                mbar_arrive(&full_bar[s]);
                ++it;
                if (!more) break;
                tile = ntile, kb = nkb, r = nr, ib = nib, cur = nxt;
            }
        }
    }
    else if (warp == kMmaWarp)
    {
        // ---------------- MMA issuer ----------------
        if (lane == 0)
        {
            uint32_t it = 0, j = 0, k = 0;
            bool failed = false;
            const int parts = MODE == kSearch ? P.nparts : 1;
            int64_t tile = blockIdx.x;
            // units (tile, part) in the CTA's order: the tiles stride by the
            // grid, or (search) come from the producers' ring
            for (int part = 0; tile >= 0 && tile < ntiles && !failed; ++j)
            {
                if (j > 0 && part == 0)
                {
                    // (after the last part of a tile) the next tile
                    if constexpr (MODE == kSearch)
                    {
                        if (!wait_bounded(&tq_bar[k & 15], (k >> 4) & 1)) break;
                        tile = s_tiles[k & 15];
                        if (tile < 0) break;
                    }
                    else
                    {
                        tile += gridDim.x;
                        if (tile >= ntiles) break;
                    }
                }
                if (++part == parts) part = 0, ++k;
                const int a = int(j % uint32_t(nacc));
                const uint32_t ua = j / uint32_t(nacc);
                if (ua > 0 && !wait_bounded(&acce_bar[a], (ua - 1) & 1)) break;
                tc_fence_after();
                const uint32_t d = tmem + uint32_t(a * acc_cols);
                for (int kb = 0; kb < P.kblocks; ++kb, ++it)
                {
                    const int s = int(it % uint32_t(S));
                    const uint32_t u = it / uint32_t(S);
                    if (!wait_bounded(&full_bar[s], u & 1))
                    {
                        failed = true;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a_base = smem_u32(smem + s * stage_bytes);
                    const uint32_t b_base = a_base + uint32_t(a_bytes);
                    // The split terms' weight rows are stacked in one K-major
                    // B of nsplit * n_tile rows whose accumulators are
                    // adjacent: one MMA covers up to 256 of them, so the A
                    // tile is read once per 256 columns, not once per term.
                    const int ncols = P.nsplit * P.n_tile;
                    for (int c = 0; c < ncols; c += 256)
                    {
                        const int n = ncols - c < 256 ? ncols - c : 256;
                        // the same 32-byte steps of each 128-byte row: 16
                        // BF16 or (search) 32 U8 elements per instruction
                        const uint32_t idesc = MODE == kSearch ? idesc_u8_s32(BM, n) : idesc_bf16_f32(BM, n);
#pragma unroll
                        for (int k16 = 0; k16 < BK / 16; ++k16)
                        {
                            const uint64_t ad = smem_desc(a_base + k16 * 256, 128, 1024);
                            const uint64_t bd = smem_desc(b_base + c * 128 + k16 * 256, 128, 1024);
                            if constexpr (MODE == kSearch)
                                mma_u8(d + uint32_t(c), ad, bd, idesc, (kb > 0 || k16 > 0) ? 1u : 0u);
                            else
                                mma_bf16(d + uint32_t(c), ad, bd, idesc, (kb > 0 || k16 > 0) ? 1u : 0u);
                        }
                    }
                    mma_commit(&empty_bar[s]);
                }
                if (!failed) mma_commit(&accf_bar[a]);
            }
        }
        __syncwarp();
    }
    else
    {
        // ---------------- epilogue (warps 0-3) ----------------
        // warp w reads tensor-memory lanes 32 w .. 32 w + 31 (rows of the tile)
        const int row = (warp & 3) * 32 + lane;
        // the largest channel bound (search)
        float emax = 0.f;
        if constexpr (MODE == kSearch) emax = __uint_as_float(P.sinfo[0]);
        uint32_t j = 0, k = 0;
        const int parts = MODE == kSearch ? P.nparts : 1;
        SearchScan scan;
        int64_t tile = blockIdx.x;
        // the MMA issuer's order of units (tile, part)
        for (int part = 0, nextp = 0; tile >= 0 && tile < ntiles; ++j, part = nextp)
        {
            if (j > 0 && part == 0)
            {
                if constexpr (MODE == kSearch)
                {
                    if (!wait_bounded(&tq_bar[k & 15], (k >> 4) & 1)) break;
                    tile = s_tiles[k & 15];
                    if (tile < 0) break;
                }
                else
                {
                    tile += gridDim.x;
                    if (tile >= ntiles) break;
                }
            }
            nextp = part + 1;
            if (nextp == parts) nextp = 0, ++k;
            const int a = int(j % uint32_t(nacc));
            const uint32_t ua = j / uint32_t(nacc);
            // search rows: the row's list entry and pixel state are loaded
            // before the wait, so their latency hides behind it
            bool s_ok = false;
            int2 s_e = make_int2(0, 0);
            int s_aux = 0;
            int4 s_st = make_int4(0, 0, 0, 0);
            if constexpr (MODE == kSearch)
            {
                const int64_t idx = tile * BM + row;
                s_ok = idx < nrows;
                if (s_ok)
                {
                    if (P.round == 0 && !P.r0_list)
                        s_e = make_int2(int(idx), P.T - 1);
                    else if (P.round == 0)
                        s_e = make_int2(P.list_in[idx].x, P.T - 1);
                    else
                    {
                        const int2 le = P.list_in[idx];
                        s_e = P.round == 1 ? le : make_int2(le.x, P.T - 1);
                        s_aux = le.y;
                        if (P.round == 1) s_st = P.state[le.x];
                    }
                }
            }
            if (!wait_bounded(&accf_bar[a], ua & 1)) break;
            tc_fence_after();
            const int64_t mt = tile / P.n_tiles;
            const int nt = int(tile % P.n_tiles);
            RowInfo r{};
            if constexpr (MODE != kSearch) r = row_info<MODE>(P, mt, row);
            const uint32_t acc = tmem + uint32_t(a * acc_cols);
            if constexpr (MODE == kPotentials)
            {
                const uint32_t lane_base = acc + (uint32_t((warp & 3) * 32) << 16);
                for (int c0 = 0; c0 < P.n_tile; c0 += 16)
                {
                    float v[16];
                    load_exact16(lane_base, c0, P.n_tile, P.nsplit, v);
                    if (r.ok)
                    {
#pragma unroll
                        for (int q = 0; q < 16; ++q)
                        {
                            const int n = nt * P.n_tile + c0 + q;
                            if (n < P.cout) P.out[(r.img * P.cout + n) * P.ohw + r.pix] = v[q];
                        }
                    }
                }
            }
            if constexpr (MODE == kTimes)
            {
                int *s_cand = reinterpret_cast<int *>(smem + S * stage_bytes + (P.kblocks * BK + 8) * 16);
                if (P.nsplit == 3)
                    times_epilogue<3>(P, acc, r.ok, mt, &acce_bar[a], s_cand, j, &tim_bar);
                else
                    times_epilogue<2>(P, acc, r.ok, mt, &acce_bar[a], s_cand, j, &tim_bar);
            }
            else if constexpr (MODE == kSearch)
            {
                if (part == 0) scan = SearchScan{};
                search_epilogue<kSearchTerms>(P, acc, s_ok, s_e.x, s_e.y, P.round == 2 ? s_aux : 0, s_st,
                                              &acce_bar[a], emax, s_scale, s_bound, int(tile * BM + row), part, scan);
            }
            else if constexpr (MODE == kFused)
            {
                float thr = P.thr;
                if (P.snet) thr = P.net_thr[P.snet[(uint32_t(mt) * uint32_t(P.pp)) / uint32_t(P.ohw)]];
                if (P.nsplit == 3)
                    fused_epilogue<3>(P, thr, acc, r.ok, r.tstep, r.sample, r.pix, &acce_bar[a]);
                else
                    fused_epilogue<2>(P, thr, acc, r.ok, r.tstep, r.sample, r.pix, &acce_bar[a]);
            }
            else
            {
                tc_fence_before();
                mbar_arrive(&acce_bar[a]);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
    {
        tc_fence_after();
        tmem_dealloc(tmem, P.tmem_cols);
    }
}

template <int MODE>
__global__ void __launch_bounds__(kWsThreads, 1) conv_ws_kernel(TcParams P)
{
    conv_ws_body<MODE, 8>(P);
}

// The search kernel for layers whose accumulators leave room for a second
// CTA on the SM (4 producer warps).
__global__ void __launch_bounds__(kSearchThreads, 2) search_ws_kernel(TcParams P) { conv_ws_body<kSearch, 4>(P); }

// WTA over the per-pixel records of one sample (one CTA per sample).  Keys
// follow cpu/wta.cpp:53-62 with the sample's min / max; ties resolve to the
// lowest flat index channel * H*W + pixel, as std::max_element does.
__global__ void wta_records_kernel(const int4 *__restrict__ records, const unsigned *__restrict__ mins,
                                   const unsigned *__restrict__ maxs, int hw, int w, int T, int ry, int rx, int count,
                                   int32_t *__restrict__ winners, int32_t *__restrict__ counts)
{
    extern __shared__ __align__(16) unsigned char wsm[];
    float *key = reinterpret_cast<float *>(wsm);
    int *flat = reinterpret_cast<int *>(key + hw);
    __shared__ float s_v[32];
    __shared__ int s_i[32];
    const int64_t b = blockIdx.x;
    const float mn = order_dec(mins[b]), mx = order_dec(maxs[b]);
    const float diff = __fmul_rn(__fsub_rn(mx, mn), 2.0f);
    for (int p = threadIdx.x; p < hw; p += blockDim.x)
    {
        const int4 r = records[b * hw + p];
        if (r.y < T)
        {
            key[p] = __fadd_rn(float(T - r.y - 1), __fdiv_rn(__fsub_rn(__int_as_float(r.z), mn), diff));
            flat[p] = r.x * hw + p;
        }
        else
        {
            key[p] = -INFINITY;
            flat[p] = INT_MAX;
        }
    }
    __syncthreads();
    int found = 0;
    for (int round = 0; round < count; ++round)
    {
        float bv = -INFINITY;
        int bi = INT_MAX;
        for (int p = threadIdx.x; p < hw; p += blockDim.x)
            if (key[p] > bv || (key[p] == bv && flat[p] < bi)) bv = key[p], bi = flat[p];
        for (int o = 16; o > 0; o >>= 1)
        {
            const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > bv || (ov == bv && oi < bi)) bv = ov, bi = oi;
        }
        if ((threadIdx.x & 31) == 0) s_v[threadIdx.x >> 5] = bv, s_i[threadIdx.x >> 5] = bi;
        __syncthreads();
        bv = s_v[0], bi = s_i[0];
        for (int q = 1; q < int(blockDim.x >> 5); ++q)
            if (s_v[q] > bv || (s_v[q] == bv && s_i[q] < bi)) bv = s_v[q], bi = s_i[q];
        __syncthreads();
        if (bi == INT_MAX) break;  // only sentinels left
        const int z = bi / hw, p0 = bi % hw, y = p0 / w, x = p0 % w;
        if (threadIdx.x == 0)
        {
            int32_t *e = winners + (b * count + round) * 5;
            e[0] = 0, e[1] = 0, e[2] = z, e[3] = y, e[4] = x;
        }
        for (int p = threadIdx.x; p < hw; p += blockDim.x)
        {
            const int py = p / w, px = p % w;
            const bool box = py >= y - ry && py <= y + ry && px >= x - rx && px <= x + rx;
            if (box || (flat[p] != INT_MAX && flat[p] / hw == z)) key[p] = -INFINITY, flat[p] = INT_MAX;
        }
        __syncthreads();
        ++found;
    }
    if (threadIdx.x == 0) counts[b] = found;
}

// The same selection with one warp per sample for maps of up to 32 * KPL
// pixels: lane l holds pixels l, l + 32, ... in registers, a round is a
// lane-local best and a 5-step shuffle argmax (no block barriers), and the
// suppression walks the lane's pixels with (y, x) advanced incrementally.
template <int KPL>
__global__ void __launch_bounds__(128) wta_records_warp_kernel(const int4 *__restrict__ records,
                                                               const unsigned *__restrict__ mins,
                                                               const unsigned *__restrict__ maxs, int64_t nb, int hw,
                                                               int w, int T, int ry, int rx, int count,
                                                               int32_t *__restrict__ winners,
                                                               int32_t *__restrict__ counts)
{
    const int lane = threadIdx.x & 31;
    const int64_t b = int64_t(blockIdx.x) * 4 + (threadIdx.x >> 5);
    if (b >= nb) return;  // whole warps leave together
    const float mn = order_dec(mins[b]), mx = order_dec(maxs[b]);
    const float diff = __fmul_rn(__fsub_rn(mx, mn), 2.0f);
    float key[KPL];
    int flat[KPL];
#pragma unroll
    for (int q = 0; q < KPL; ++q)
    {
        const int p = lane + 32 * q;
        key[q] = -INFINITY, flat[q] = INT_MAX;
        if (p < hw)
        {
            const int4 r = records[b * hw + p];
            if (r.y < T)
            {
                key[q] = __fadd_rn(float(T - r.y - 1), __fdiv_rn(__fsub_rn(__int_as_float(r.z), mn), diff));
                flat[q] = r.x * hw + p;
            }
        }
    }
    // each slot's (row, column), packed, for the suppression boxes
    int pyx[KPL];
    {
        int py = lane / w, px = lane - py * w;
#pragma unroll
        for (int q = 0; q < KPL; ++q)
        {
            pyx[q] = (py << 16) | px;
            px += 32;
            while (px >= w) px -= w, ++py;
        }
    }
    int found = 0;
    for (int round = 0; round < count; ++round)
    {
        float bv = -INFINITY;
        int bi = INT_MAX;
#pragma unroll
        for (int q = 0; q < KPL; ++q)
            if (key[q] > bv || (key[q] == bv && flat[q] < bi)) bv = key[q], bi = flat[q];
        for (int o = 16; o > 0; o >>= 1)
        {
            const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > bv || (ov == bv && oi < bi)) bv = ov, bi = oi;
        }
        if (bi == INT_MAX) break;  // only sentinels left (the same in every lane)
        const int z = bi / hw, p0 = bi - z * hw, y = p0 / w, x = p0 - y * w;
        if (lane == 0)
        {
            int32_t *e = winners + (b * count + round) * 5;
            e[0] = 0, e[1] = 0, e[2] = z, e[3] = y, e[4] = x;
        }
        // the winner's box (every channel) and the winner's channel leave
        const int zlo = z * hw, zhi = zlo + hw;
#pragma unroll
        for (int q = 0; q < KPL; ++q)
        {
            const int py = pyx[q] >> 16, px = pyx[q] & 0xFFFF;
            const bool box = py >= y - ry && py <= y + ry && px >= x - rx && px <= x + rx;
            if (box || (flat[q] >= zlo && flat[q] < zhi)) key[q] = -INFINITY, flat[q] = INT_MAX;
        }
        ++found;
    }
    if (lane == 0) counts[b] = found;
}

// ---- search path: weight split, exact recompute, outputs ---------------------
// Split of output channel n's weights into NS base-256 digits (one CTA per
// channel of the padded tile).  With 2^e the smallest power of two above the
// channel's largest weight (e clamped to [-94, 100]), w = 2^e sum_j d_j
// 256^-(j+1) + rem, digits d_j in [0, 255] (floor), 0 <= rem < 2^(e - 8 NS).
// A 0/1 spike times a digit is an exact 8-bit product and the tensor core's
// 32-bit integer sums are exact, so the row's term total R (an integer) times
// cscale[n] = 2^(e - 8 NS) is the potential of the digit weights exactly.
// echan[n] bounds |oracle - R cscale| for any 0/1 input: the sum of the
// remainders (zero when every weight lies on the 2^(e - 8 NS) grid) plus,
// unless the oracle's ordered FP64 sum is exact for these weights, K^2
// 2^(e-52).  Negative weights only raise *negw (the search then stands down).
// The operand layout is split_weights_kernel's, with 16 U8 elements per
// 16-byte chunk (128 per K block), K in channels-last order.
template <int NS>
__global__ void __launch_bounds__(256) fixed_split_kernel(const float *__restrict__ kernel, uint4 *__restrict__ wimg,
                                                          int cout, int cin, int taps, int cpad, int kblocks,
                                                          int n_tile, float *__restrict__ echan,
                                                          float *__restrict__ cscale, unsigned *__restrict__ sinfo,
                                                          int *__restrict__ negw, unsigned *__restrict__ wmax)
{
    __shared__ float s_mx[8];
    __shared__ double s_err[8];
    __shared__ int s_lsb[8];
    const int n = blockIdx.x, tid = threadIdx.x;
    const int kreal = taps * cpad;
    const int K = kblocks * 2 * BK;
    auto weight = [&](int k) -> float {
        if (n >= cout || k >= kreal) return 0.f;
        const int tap = k / cpad, c = k % cpad;
        return c < cin ? kernel[(int64_t(n) * cin + c) * taps + tap] : 0.f;
    };
    float mx = 0.f;
    bool neg = false;
    int lsb = INT_MAX;  // exponent of the lowest set bit of any weight
    for (int k = tid; k < K; k += blockDim.x)
    {
        const float w = weight(k);
        mx = fmaxf(mx, fabsf(w));
        neg |= !(w >= 0.f);
        if (wmax && n < cout && k < kreal && w > 0.f)
        {
            // largest weight of each input over the channels (oracle layout)
            const int tap = k / cpad, c = k % cpad;
            if (c < cin) atomicMax(wmax + c * taps + tap, __float_as_uint(w));
        }
        const uint32_t bits = __float_as_uint(w) & 0x7FFFFFFFu;
        if (bits != 0u && bits < 0x7F800000u)
        {
            const int ex = int(bits >> 23);
            const uint32_t sig = ex ? ((bits & 0x7FFFFFu) | 0x800000u) : bits;
            lsb = min(lsb, __ffs(int(sig)) - 1 + (ex ? ex : 1) - 150);
        }
    }
    for (int o = 16; o > 0; o >>= 1)
    {
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        lsb = min(lsb, __shfl_xor_sync(0xffffffffu, lsb, o));
    }
    if ((tid & 31) == 0) s_mx[tid >> 5] = mx, s_lsb[tid >> 5] = lsb;
    __syncthreads();
    mx = s_mx[0], lsb = s_lsb[0];
    for (int i = 1; i < int(blockDim.x >> 5); ++i) mx = fmaxf(mx, s_mx[i]), lsb = min(lsb, s_lsb[i]);
    int e = 0;
    if (mx > 0.f)
    {
        int ex;
        frexpf(mx, &ex);  // mx = fr 2^ex, fr in [0.5, 1): mx < 2^ex
        e = ex;
    }
    e = max(-94, min(100, e));
    double err = 0.0;
    for (int i = tid; i < kblocks * 8; i += blockDim.x)
    {
        const int kb = i / 8, kc = i % 8;
        uint32_t parts[NS][4];
#pragma unroll
        for (int j = 0; j < NS; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) parts[j][q] = 0u;
#pragma unroll
        for (int e16 = 0; e16 < 16; ++e16)
        {
            const double w = fmax(double(weight(kb * 2 * BK + kc * 16 + e16)), 0.0);
            double r = ldexp(w, -e);  // in [0, 1)
#pragma unroll
            for (int j = 0; j < NS; ++j)
            {
                const double d = floor(r * 256.0);
                r = r * 256.0 - d;
                parts[j][e16 >> 2] |= uint32_t(d) << (8 * (e16 & 3));
            }
            err += ldexp(r, e - 8 * NS);
        }
#pragma unroll
        for (int j = 0; j < NS; ++j)
        {
            // part n / n_tile of the channels, row n % n_tile within it
            const int part = n / n_tile, nl = n % n_tile;
            const int64_t idx = ((int64_t(part) * kblocks + kb) * NS + j) * (int64_t(n_tile) * 8) + (nl / 8) * 64 +
                                kc * 8 + (nl % 8);
            wimg[idx] = make_uint4(parts[j][0], parts[j][1], parts[j][2], parts[j][3]);
        }
    }
    for (int o = 16; o > 0; o >>= 1) err += __shfl_xor_sync(0xffffffffu, err, o);
    if ((tid & 31) == 0) s_err[tid >> 5] = err;
    if (neg && n < cout) atomicOr(negw, 1);
    __syncthreads();
    if (tid == 0)
    {
        err = s_err[0];
        for (int i = 1; i < int(blockDim.x >> 5); ++i) err += s_err[i];
        // the oracle's ordered FP64 sum is exact when every partial sum
        // (a multiple of 2^lsb, at most kreal 2^e) fits in 53 bits
        int lk = 0;
        while ((1 << lk) < kreal) ++lk;
        const bool exact64 = lsb == INT_MAX || e + lk - lsb <= 53;
        const double bound = err + (exact64 ? 0.0 : double(kreal) * double(kreal) * ldexp(1.0, e - 52));
        const float eb = __double2float_ru(bound);
        echan[n] = eb;
        cscale[n] = ldexpf(1.f, e - 8 * NS);
        if (n < cout)
        {
            atomicMax(sinfo + 0, __float_as_uint(eb));
            atomicMax(sinfo + 1, unsigned(e + 128));
        }
    }
}

// Per sample min / max of the inhibited potentials before the search adds to
// them: on the search path the losing channels' zeros, on the dense path the
// identities of the min / max (that kernel adds every value itself).
__global__ void search_init_kernel(unsigned *mins, unsigned *maxs, int64_t b, const int *negw, const int *flag)
{
    const bool lean = !*negw && !*flag;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < b; i += int64_t(gridDim.x) * blockDim.x)
    {
        mins[i] = lean ? order_enc(0.f) : 0xFFFFFFFFu;
        maxs[i] = lean ? order_enc(0.f) : 0u;
    }
}

// Pre-filter of round 0: with no negative weight, a pixel's potential at
// T - 1 is at most U, the sum over the inputs that fired of their largest
// weight over the channels.  A pixel with U at or below the threshold never
// fires and is settled here; the others go to round 0's list (entry
// (pixel, T - 1) at the pixel's index, -1 for settled pixels; the list is
// then compacted in pixel order).  U is summed in FP32 (non-negative terms)
// and multiplied, rounding up, by 1 + (K + 2) 2^-23, which covers the
// roundings of that sum, of the oracle's FP64 sum and of its rounding to F32.
// A CTA per sample: the sample's first-spike map becomes a 32-bit mask per
// input pixel (the channels fired by T - 1, up to 32) in shared memory, the
// per-tap channel maxima a table beside it; a thread per output pixel adds
// the maxima of its taps' set bits.  With T <= 32 it adds them into bins by
// their inputs' first steps (one bin per step and thread in shared memory):
// the running sums of the bins give U(t) for every t, U = U(T - 1), and
// t_lo, the first step whose U(t) (widened the same way) is above the
// threshold: no channel fires before t_lo, so the bisection starts from
// (t_lo - 1, T - 1].
__global__ void __launch_bounds__(256) search_bound_kernel(TcParams P, const unsigned *__restrict__ wmax, int cp,
                                                           int2 *__restrict__ list, uint8_t *__restrict__ tlo)
{
    if (*P.negw || *P.flag) return;
    extern __shared__ __align__(16) uint8_t s_bound_sm[];
    const int taps = P.kh * P.kw, kr = P.cin * taps, hw = P.h * P.w;
    // regions, each 16-byte aligned: masks [H * W], channel maxima [taps][cp],
    // (tlo) bins [T][blockDim] and the map's bytes [H * W][cp]
    const int o_w = (hw * 4 + 15) & ~15, o_acc = o_w + ((taps * cp * 4 + 15) & ~15);
    const int o_fb = o_acc + ((P.T * int(blockDim.x) * 4 + 15) & ~15);
    uint32_t *s_fired = reinterpret_cast<uint32_t *>(s_bound_sm);
    float *wm = reinterpret_cast<float *>(s_bound_sm + o_w);
    float *s_acc = reinterpret_cast<float *>(s_bound_sm + o_acc);
    uint8_t *s_fb = s_bound_sm + o_fb;
    for (int i = threadIdx.x; i < taps * cp; i += blockDim.x)
    {
        const int tap = i / cp, c = i % cp;
        wm[i] = c < P.cin ? __uint_as_float(wmax[c * taps + tap]) : 0.f;
    }
    // FP32 sum of at most kr non-negative terms: within kr 2^-24 of the exact
    // sum, itself at least the oracle's FP64 sum / (1 + kr 2^-53)
    const float widen = 1.f + float(kr + 2) * 0x1p-23f;
    const int ohw = int(P.ohw);
    const uint32_t tt = uint32_t(P.T) * 0x01010101u;
    const int64_t b = P.npix / ohw;
    const int words = cp / 8;
    for (int64_t smp = blockIdx.x; smp < b; smp += gridDim.x)
    {
        const uint8_t *fm = P.in + smp * P.img_stride;
        __syncthreads();  // the previous sample's masks are read (and the table written)
        for (int q = threadIdx.x; q < hw; q += blockDim.x)
        {
            uint32_t m = 0;
            for (int g = 0; g < words; ++g)
            {
                const uint2 f = __ldg(reinterpret_cast<const uint2 *>(fm + int64_t(q) * cp) + g);
                if (tlo) reinterpret_cast<uint2 *>(s_fb + q * cp)[g] = f;
                // 0x80 in the bytes that fired by step T - 1 (byte < T)
                const uint32_t lo = ((f.x | 0x80808080u) - tt) ^ 0x80808080u;
                const uint32_t hi = ((f.y | 0x80808080u) - tt) ^ 0x80808080u;
#pragma unroll
                for (int c = 0; c < 4; ++c)
                    m |= (((lo >> (8 * c + 7)) & 1u) << (8 * g + c)) | (((hi >> (8 * c + 7)) & 1u) << (8 * g + c + 4));
            }
            s_fired[q] = m;
        }
        __syncthreads();
        for (int p0 = 0; p0 < ohw; p0 += int(blockDim.x))
        {
            // warp-uniform trips: the candidates are counted per warp
            const int p = p0 + int(threadIdx.x);
            const int pix = int(smp * ohw) + p;
            bool cand = false;
            if (p < ohw)
            {
                const int oy = p / P.ow, ox = p - oy * P.ow;
                const int iy0 = oy * P.sy - P.top, ix0 = ox * P.sx - P.left;
                const int ky0 = max(0, -iy0), ky1 = min(P.kh, P.h - iy0);
                const int kx0 = max(0, -ix0), kx1 = min(P.kw, P.w - ix0);
                if (tlo)
                {
                    // one pass: the terms binned by their inputs' first steps
                    // (all below T); U is the sum of the bins, the same terms
                    // summed in another order (the widening covers any order)
                    float *acc = s_acc + threadIdx.x;
                    for (int t = 0; t < P.T; ++t) acc[t * blockDim.x] = 0.f;
                    for (int ky = ky0; ky < ky1; ++ky)
                        for (int kx = kx0; kx < kx1; ++kx)
                        {
                            const int q = (iy0 + ky) * P.w + ix0 + kx;
                            uint32_t m = s_fired[q];
                            const float *w = wm + (ky * P.kw + kx) * cp;
                            while (m)
                            {
                                const int c = __ffs(int(m)) - 1;
                                acc[int(s_fb[q * cp + c]) * blockDim.x] += w[c];
                                m &= m - 1u;
                            }
                        }
                    float run = 0.f;
                    int t0 = P.T - 1;  // no step below T - 1 can fire either when none passes
                    for (int t = 0; t < P.T; ++t)
                    {
                        run += acc[t * blockDim.x];
                        if (t0 == P.T - 1 && t < P.T - 1 && __fmul_ru(run, widen) > P.thr) t0 = t;
                    }
                    cand = __fmul_ru(run, widen) > P.thr;
                    if (cand) tlo[pix] = uint8_t(t0);
                }
                else
                {
                    float u = 0.f;
                    for (int ky = ky0; ky < ky1; ++ky)
                        for (int kx = kx0; kx < kx1; ++kx)
                        {
                            uint32_t m = s_fired[(iy0 + ky) * P.w + ix0 + kx];
                            const float *w = wm + (ky * P.kw + kx) * cp;
                            while (m)
                            {
                                u += w[__ffs(int(m)) - 1];
                                m &= m - 1u;
                            }
                        }
                    cand = __fmul_ru(u, widen) > P.thr;
                }
                if (!cand)
                {
                    P.records[pix] = make_int4(0, P.T, __float_as_int(P.thv), 0);
                    if (P.wta && P.thv != 0.f)
                    {
                        atomicMin(P.mins + smp, order_enc(P.thv));
                        atomicMax(P.maxs + smp, order_enc(P.thv));
                    }
                }
                list[pix] = make_int2(pix, cand ? P.T - 1 : -1);
            }
            list_count_warp(P.list_bc, pix, cand);
        }
    }
}

// Stable compaction of a row list: the entries with a step >= 0 of
// in[0 .. n) (n = *n_dev, or n_max when n_dev is null) go to out in their
// order, their number to *count_out.  The kernels that write the list also
// count its valid entries per block of kCompactItems (list_count_warp), so
// for up to kSelfPrefixBlocks blocks the compaction is one launch: each
// scatter block sums the counts before its own.  Longer lists take three:
// per-block counts, one block's exclusive scan of them, and the scatter (a
// block writes its entries from its offset, ranked by warp ballots).  The
// lists stay in pixel order, so a tile's rows lie in a few neighbouring
// images.
constexpr int kSelfPrefixBlocks = 2048;

__device__ __forceinline__ int64_t list_len(const int *n_dev, int64_t n_max) { return n_dev ? int64_t(*n_dev) : n_max; }

__global__ void __launch_bounds__(256) list_count_kernel(const int2 *__restrict__ in, const int *n_dev, int64_t n_max,
                                                         int *__restrict__ bcount, const int *negw, const int *flag)
{
    if (*negw || *flag) return;
    __shared__ int ws[8];
    const int64_t n = list_len(n_dev, n_max), b0 = int64_t(blockIdx.x) * kCompactItems;
    int c = 0;
    for (int i = threadIdx.x; i < kCompactItems; i += blockDim.x)
    {
        const int64_t j = b0 + i;
        c += (j < n && in[j].y >= 0) ? 1 : 0;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        int t = 0;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) t += ws[w];
        bcount[blockIdx.x] = t;
    }
}

// One block of 1024 threads: bcount[0 .. nb) becomes its exclusive prefix sum.
__global__ void __launch_bounds__(1024) list_scan_kernel(int *__restrict__ bcount, int nb, int *__restrict__ count_out,
                                                         const int *negw, const int *flag)
{
    if (*negw || *flag) return;
    __shared__ int ws[32];
    const int per = (nb + 1023) / 1024, lo = threadIdx.x * per, hi = min(nb, lo + per);
    int sum = 0;
    for (int i = lo; i < hi; ++i) sum += bcount[i];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = sum;
    for (int o = 1; o < 32; o <<= 1)
    {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) ws[warp] = incl;
    __syncthreads();
    if (warp == 0)
    {
        int w = ws[lane], wi = w;
        for (int o = 1; o < 32; o <<= 1)
        {
            const int v = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += v;
        }
        ws[lane] = wi - w;  // exclusive prefix of the warps
        if (lane == 31) *count_out = wi;
    }
    __syncthreads();
    int run = ws[warp] + incl - sum;
    for (int i = lo; i < hi; ++i)
    {
        const int v = bcount[i];
        bcount[i] = run;
        run += v;
    }
}

// The scatter (256 threads, kCompactItems entries a block, all loaded at
// once).  A block's offset is boff[block] (the scan's output) or, with
// self_prefix, the sum of the entry counts of the blocks before it, which the
// list's writers added to bcount: then the block holding the list's last
// entry also writes *count_out.  Every launch zeroes bzero[0 .. nbz), the
// counts of the next compaction.
__global__ void __launch_bounds__(256) list_scatter_kernel(const int2 *__restrict__ in, const int *n_dev,
                                                           int64_t n_max, const int *__restrict__ boff,
                                                           int self_prefix, int *__restrict__ count_out,
                                                           int *__restrict__ bzero, int nbz, int2 *__restrict__ out,
                                                           const int *negw, const int *flag)
{
    if (*negw || *flag) return;
    constexpr int Q = kCompactItems / 256;
    __shared__ int ws[Q][8], wsum[8];
    for (int i = int(blockIdx.x * blockDim.x + threadIdx.x); i < nbz; i += int(gridDim.x * blockDim.x)) bzero[i] = 0;
    const int64_t n = list_len(n_dev, n_max), b0 = int64_t(blockIdx.x) * kCompactItems;
    if (b0 >= n)
    {
        if (self_prefix && blockIdx.x == 0 && threadIdx.x == 0) *count_out = 0;
        return;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int2 e[Q];
    unsigned m[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        const int64_t j = b0 + q * 256 + threadIdx.x;
        e[q] = j < n ? in[j] : make_int2(0, -1);
    }
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        m[q] = __ballot_sync(0xffffffffu, e[q].y >= 0);
        if (lane == 0) ws[q][warp] = __popc(m[q]);
    }
    if (self_prefix)
    {
        int acc = 0;
        for (int i = threadIdx.x; i < int(blockIdx.x); i += 256) acc += boff[i];
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) wsum[warp] = acc;
    }
    __syncthreads();
    int off = 0;
    if (self_prefix)
    {
#pragma unroll
        for (int w = 0; w < 8; ++w) off += wsum[w];
    }
    else
        off = boff[blockIdx.x];
    const unsigned below = (1u << lane) - 1u;
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        int before = 0, total = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w)
        {
            before += w < warp ? ws[q][w] : 0;
            total += ws[q][w];
        }
        if (e[q].y >= 0) out[off + before + __popc(m[q] & below)] = e[q];
        off += total;
    }
    if (self_prefix && threadIdx.x == 0 && b0 + kCompactItems >= n) *count_out = off;
}

// Rows the search could not decide from the term sums (a potential within
// echan of a rounding boundary that matters), recomputed as the oracle does:
// per channel the FP64 sum of the F32 weights of the active inputs in
// (channel, ky, kx) order (the oracle's convolution loop), rounded once to
// F32.  One warp per row; its lanes take the output channels.
// The oracle's potential of one channel (weights wk [Cin, KH, KW]) at step t
// for the pixel whose receptive field starts at (iy0, ix0): the FP64 sum of
// the weights of the inputs that fired by t, in (channel, ky, kx) order,
// positions outside the input skipped.
// The same sum for maps of 8 padded channels and windows up to 5 x 5: the
// window's first-spike words are loaded first, all in flight together (0xFF
// bytes outside the input never fire), then summed in the same order.
__device__ __forceinline__ double oracle_sum_small(const TcParams &P, const uint8_t *fm, const float *wk, int iy0,
                                                   int ix0, int t)
{
    uint2 f[25];
#pragma unroll
    for (int ky = 0; ky < 5; ++ky)
#pragma unroll
        for (int kx = 0; kx < 5; ++kx)
        {
            const int iy = iy0 + ky, ix = ix0 + kx;
            f[ky * 5 + kx] = (ky < P.kh && kx < P.kw && iy >= 0 && iy < P.h && ix >= 0 && ix < P.w)
                                 ? __ldg(reinterpret_cast<const uint2 *>(fm + (int64_t(iy) * P.w + ix) * 8))
                                 : make_uint2(~0u, ~0u);
        }
    double acc = 0.0;
    for (int c = 0; c < P.cin; ++c)
    {
        const int sh = (c & 3) * 8;
        const float *wc = wk + c * P.kh * P.kw;
#pragma unroll
        for (int ky = 0; ky < 5; ++ky)
#pragma unroll
            for (int kx = 0; kx < 5; ++kx)
                if (ky < P.kh && kx < P.kw)
                {
                    const double wv = double(__ldg(wc + ky * P.kw + kx));
                    const uint32_t word = c < 4 ? f[ky * 5 + kx].x : f[ky * 5 + kx].y;
                    if (int((word >> sh) & 0xFFu) <= t) acc += wv;
                }
    }
    return acc;
}

__device__ __forceinline__ double oracle_sum(const TcParams &P, const uint8_t *fm, const float *wk, int iy0, int ix0,
                                             int cp, int t)
{
    if (cp == 8 && P.kh <= 5 && P.kw <= 5) return oracle_sum_small(P, fm, wk, iy0, ix0, t);
    const int ky0 = max(0, -iy0), ky1 = min(P.kh, P.h - iy0);
    const int kx0 = max(0, -ix0), kx1 = min(P.kw, P.w - ix0);
    double acc = 0.0;
    for (int c = 0; c < P.cin; ++c)
        for (int ky = ky0; ky < ky1; ++ky)
        {
            const int64_t fr = (int64_t(iy0 + ky) * P.w + ix0) * cp + c;  // index of kx = 0 (may lie outside)
            const float *wr = wk + (c * P.kh + ky) * P.kw;
#pragma unroll 4
            for (int kx = kx0; kx < kx1; ++kx)
            {
                const float wv = __ldg(wr + kx);
                if (int(__ldg(fm + fr + int64_t(kx) * cp)) <= t) acc += double(wv);
            }
        }
    return acc;
}

__global__ void __launch_bounds__(128) search_fix_kernel(TcParams P, const float *__restrict__ kernel, int cp)
{
    if (*P.negw || *P.flag) return;
    const int lane = threadIdx.x & 31;
    const int64_t nw = int64_t(gridDim.x) * (blockDim.x >> 5);
    const int taps = P.kh * P.kw;
    // rows whose winner is decided: one lane per row sums the winner's
    // products in the oracle's order
    const int nv = *P.val_count;
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < nv; q += int64_t(gridDim.x) * blockDim.x)
    {
        const int4 e = P.val_list[q];
        const int pix = e.x, t = e.y, idx = e.z, o = e.w, round = P.round;
        const int smp = pix / int(P.ohw), pp = pix - smp * int(P.ohw);
        const int oy = pp / P.ow, ox = pp - oy * P.ow;
        const int iy0 = oy * P.sy - P.top, ix0 = ox * P.sx - P.left;
        const uint8_t *fm = P.in + int64_t(smp) * P.img_stride;
        const float *wk = kernel + int64_t(o) * P.cin * taps;
        const double acc = oracle_sum(P, fm, wk, iy0, ix0, cp, t);
        atomicAdd(&g_recomputes, 1ull);
        const SearchAct r = search_act(P, round, pix, t, 2, o, float(acc), round == 1 ? P.state[pix] : int4{});
        if (round != 2) P.list_out[idx] = r.next ? r.next_e : make_int2(pix, -1);
        if (round != 2 && r.next) atomicAdd(P.list_bc + (idx >> kCompactShift), 1);
        if (r.fin) P.final_list[atomicAdd(P.final_count, 1)] = r.fin_e;
        if (P.wta) s_extremes(P, pix, r);
    }
    const int n = *P.fix_count;
    for (int64_t q = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); q < n; q += nw)
    {
        const int4 e = P.fix_list[q];
        const int pix = e.x, t = e.y, idx = e.z, aux = e.w, round = P.round;
        const int smp = pix / int(P.ohw), pp = pix - smp * int(P.ohw);
        const int oy = pp / P.ow, ox = pp - oy * P.ow;
        const int iy0 = oy * P.sy - P.top, ix0 = ox * P.sx - P.left;
        const uint8_t *fm = P.in + int64_t(smp) * P.img_stride;
        float best = -INFINITY, mine = 0.f;
        int besti = INT_MAX;
        for (int o = lane; o < P.cout; o += 32)
        {
            if (round == 2 && o != aux) continue;
            const float pv = float(oracle_sum(P, fm, kernel + int64_t(o) * P.cin * taps, iy0, ix0, cp, t));
            if (pv > best) best = pv, besti = o;
            if (o == aux) mine = pv;
        }
        // first channel of the largest potential across the lanes
        for (int off = 16; off > 0; off >>= 1)
        {
            const float ob = __shfl_xor_sync(0xffffffffu, best, off);
            const int oi = __shfl_xor_sync(0xffffffffu, besti, off);
            if (ob > best || (ob == best && oi < besti)) best = ob, besti = oi;
        }
        mine = __shfl_sync(0xffffffffu, mine, aux & 31);
        if (lane == 0)
        {
            atomicAdd(&g_recomputes, 1ull);
            int dec, a;
            float v;
            if (round == 2)
                dec = 2, a = aux, v = mine;
            else if (best > P.thr)
                dec = 2, a = besti, v = best;
            else
                dec = 1, a = -1, v = 0.f;
            const SearchAct r = search_act(P, round, pix, t, dec, a, v, round == 1 ? P.state[pix] : int4{});
            if (round != 2) P.list_out[idx] = r.next ? r.next_e : make_int2(pix, -1);
            if (round != 2 && r.next) atomicAdd(P.list_bc + (idx >> kCompactShift), 1);
            if (r.fin) P.final_list[atomicAdd(P.final_count, 1)] = r.fin_e;
            if (P.wta) s_extremes(P, pix, r);
        }
    }
}

// Per-pixel winner and first-step bytes (t0 = T: never) of maps too large to
// stage in shared memory: wbytes [npix], then tbytes [npix].
__global__ void search_codes_kernel(const int4 *__restrict__ records, uint8_t *__restrict__ codes, int64_t npix,
                                    int T, const int *negw, const int *flag)
{
    if (*negw || *flag) return;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < npix; i += int64_t(gridDim.x) * blockDim.x)
    {
        const int4 r = records[i];
        codes[i] = uint8_t(r.x);
        codes[npix + i] = uint8_t(min(r.y, T));
    }
}

// Byte-parallel tests on four pixels at once (bytes below 0x80): the bytes
// of w that equal c, and the bytes of t0 at or below t, as 0x80 flags.
__device__ __forceinline__ uint32_t bytes_eq(uint32_t w, uint32_t c4)
{
    const uint32_t x = w ^ c4;
    return ~(((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x | 0x7F7F7F7Fu);
}
__device__ __forceinline__ uint32_t bytes_le(uint32_t t0, uint32_t t4) { return ((t4 | 0x80808080u) - t0) & 0x80808080u; }

// Spikes (and pooled spikes) of the search path from the per-pixel records:
// channel w fires from step t0 on.  A CTA per sample writes its
// [T, C, OH, OW] block; per pixel the winner and first-step bytes sit in
// shared memory (or in global memory for maps above 16384 pixels).  Pooled
// spikes [T, C, POH, POW] come from a byte table of the first firing step
// per (channel, cell): a cell fires from the earliest t0 of its window's
// pixels won by that channel.  Off the search path (negative weights or
// other input) it writes zeros, which the dense kernel then fills.
//
// The block is written by (channel, pixel) slabs of one step: when a slab of
// C x HW bytes is a multiple of V (16 or 4) and a plane a multiple of 4
// pixels, a thread takes one V-byte chunk of the slab (4-pixel words, each
// inside one plane), reads its pixels' winner and first-step bytes once and
// writes that chunk for every step (T stores of one byte-parallel compare
// and mask per word); other shapes take a byte per thread.
template <int V>
__device__ __forceinline__ void write_slab_words(uint8_t *dst, int T, int C, int hw, bool lean, bool pass0,
                                                 const uint8_t *wsrc, const uint8_t *tsrc, int tstride)
{
    constexpr int NW = V / 4;
    using Vec = typename std::conditional<V == 16, uint4, uint32_t>::type;
    const int slab = C * hw, nq = slab / V;
    for (int q = threadIdx.x; q < nq; q += blockDim.x)
    {
        uint32_t eq[NW], tw[NW];
#pragma unroll
        for (int r = 0; r < NW; ++r)
        {
            const int f = V * q + 4 * r, c = f / hw, px = f - c * hw;
            if (pass0)
            {
                eq[r] = bytes_eq(*reinterpret_cast<const uint32_t *>(wsrc + px), uint32_t(c) * 0x01010101u);
                tw[r] = *reinterpret_cast<const uint32_t *>(tsrc + px);
            }
            else
            {
                eq[r] = 0x80808080u;
                tw[r] = *reinterpret_cast<const uint32_t *>(tsrc + c * tstride + px);
            }
            if (!lean) eq[r] = 0u;
        }
        Vec *d = reinterpret_cast<Vec *>(dst) + q;
        for (int t = 0; t < T; ++t)
        {
            const uint32_t t4 = uint32_t(t) * 0x01010101u;
            if constexpr (V == 16)
                d[int64_t(t) * nq] =
                    make_uint4((eq[0] & bytes_le(tw[0], t4)) >> 7, (eq[1] & bytes_le(tw[1], t4)) >> 7,
                               (eq[2] & bytes_le(tw[2], t4)) >> 7, (eq[3] & bytes_le(tw[3], t4)) >> 7);
            else
                d[int64_t(t) * nq] = (eq[0] & bytes_le(tw[0], t4)) >> 7;
        }
    }
}

// Maps above 16384 pixels (per-pixel winner and first-step bytes in global
// memory): a grid of CTAs per sample (blockIdx.y), each thread one 16-byte
// chunk of a step's (channel, pixel) slab for every step; pooled spikes a
// 4-cell word at a time, each cell's first firing step for the word's channel
// taken over its window (T: never) and compared with every step.  Needs
// C x OH x OW a multiple of 16, OH x OW and the pooled width multiples of 4.
__global__ void __launch_bounds__(256) search_write_large_kernel(const uint8_t *__restrict__ codes, int64_t npix,
                                                                 const int *negw, const int *flag,
                                                                 uint8_t *__restrict__ spikes,
                                                                 uint8_t *__restrict__ pooled, int T, int C, int ohw,
                                                                 int ow, int pky, int pkx, int poh, int pow_)
{
    const bool lean = !*negw && !*flag;
    const int64_t smp = blockIdx.y;
    const uint8_t *wb = codes + smp * ohw, *tb = codes + npix + smp * ohw;
    const int64_t step = int64_t(gridDim.x) * blockDim.x;
    {
        const int64_t slab = int64_t(C) * ohw, nq = slab / 16;
        uint4 *dst = reinterpret_cast<uint4 *>(spikes + smp * T * slab);
        for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < nq; q += step)
        {
            uint32_t eq[4], tw[4];
#pragma unroll
            for (int r = 0; r < 4; ++r)
            {
                const int64_t f = 16 * q + 4 * r;
                const int c = int(f / ohw), px = int(f - int64_t(c) * ohw);
                eq[r] = lean ? bytes_eq(*reinterpret_cast<const uint32_t *>(wb + px), uint32_t(c) * 0x01010101u) : 0u;
                tw[r] = *reinterpret_cast<const uint32_t *>(tb + px);
            }
            for (int t = 0; t < T; ++t)
            {
                const uint32_t t4 = uint32_t(t) * 0x01010101u;
                dst[int64_t(t) * nq + q] =
                    make_uint4((eq[0] & bytes_le(tw[0], t4)) >> 7, (eq[1] & bytes_le(tw[1], t4)) >> 7,
                               (eq[2] & bytes_le(tw[2], t4)) >> 7, (eq[3] & bytes_le(tw[3], t4)) >> 7);
            }
        }
    }
    if (pooled == nullptr) return;
    const int phw = poh * pow_;
    const int64_t slab = int64_t(C) * phw, nw = slab / 4;
    uint32_t *dst = reinterpret_cast<uint32_t *>(pooled + smp * T * slab);
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < nw; q += step)
    {
        const int64_t f = 4 * q;
        const int c = int(f / phw), cell = int(f - int64_t(c) * phw), py = cell / pow_, px = cell - py * pow_;
        uint32_t first = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            int m = T;
            for (int dy = 0; dy < pky; ++dy)
                for (int dx = 0; dx < pkx; ++dx)
                {
                    const int i = (py * pky + dy) * ow + (px + j) * pkx + dx;
                    if (int(wb[i]) == c) m = min(m, int(tb[i]));
                }
            first |= uint32_t(m) << (8 * j);
        }
        for (int t = 0; t < T; ++t)
            dst[int64_t(t) * nw + q] = lean ? bytes_le(first, uint32_t(t) * 0x01010101u) >> 7 : 0u;
    }
}

__global__ void __launch_bounds__(256) search_write_kernel(const int4 *__restrict__ records,
                                                           const uint8_t *__restrict__ gcodes, int64_t npix,
                                                           const int *negw, const int *flag,
                                                           uint8_t *__restrict__ spikes, uint8_t *__restrict__ pooled,
                                                           int64_t b, int T, int C, int ohw, int ow, int pky,
                                                           int pkx, int poh, int pow_, int ptab)
{
    // [ohw16] winner bytes, [ohw16] first-step bytes, then [C][phw16] pooled first steps
    extern __shared__ __align__(16) uint8_t wsm_[];
    const bool lean = !*negw && !*flag;
    const int ohw16 = (ohw + 15) & ~15, phw = poh * pow_, phw16 = (phw + 15) & ~15;
    // (maps above 16384 pixels keep their bytes in global memory: the table
    // then starts at byte 32, as the launch sizes it)
    uint8_t *sw = wsm_, *st = wsm_ + ohw16, *first = wsm_ + (gcodes ? 32 : 2 * ohw16);
    for (int64_t smp = blockIdx.x; smp < b; smp += gridDim.x)
    {
        const uint8_t *wsrc = gcodes ? gcodes + smp * ohw : sw;
        const uint8_t *tsrc = gcodes ? gcodes + npix + smp * ohw : st;
        if (lean && !gcodes)
            for (int p = threadIdx.x; p < ohw; p += blockDim.x)
            {
                const int4 r = records[smp * ohw + p];
                sw[p] = uint8_t(r.x), st[p] = uint8_t(min(r.y, T));
            }
        if (lean && ptab)
            for (int i = threadIdx.x; i < C * phw16; i += blockDim.x) first[i] = uint8_t(T);
        __syncthreads();
        if (lean && ptab)
        {
            // earliest t0 per (channel, cell): bytes updated through their word
            for (int p = threadIdx.x; p < ohw; p += blockDim.x)
            {
                const int y = p / ow, x = p - y * ow, py = y / pky, px = x / pkx;
                const int t0 = int(tsrc[p]);
                if (py < poh && px < pow_ && t0 < T)
                {
                    const int idx = int(wsrc[p]) * phw16 + py * pow_ + px;
                    unsigned *word = reinterpret_cast<unsigned *>(first + (idx & ~3));
                    const int sh = 8 * (idx & 3);
                    unsigned old = *word;
                    while (int((old >> sh) & 0xFF) > t0)
                    {
                        const unsigned nw = (old & ~(0xFFu << sh)) | (unsigned(t0) << sh);
                        const unsigned seen = atomicCAS(word, old, nw);
                        if (seen == old) break;
                        old = seen;
                    }
                }
            }
            __syncthreads();
        }
        for (int pass = 0; pass < (pooled ? 2 : 1); ++pass)
        {
            const int hw = pass == 0 ? ohw : phw;
            const int64_t n = int64_t(T) * C * hw;
            uint8_t *dst = (pass == 0 ? spikes : pooled) + smp * n;
            const bool table = pass == 0 || ptab || !lean;
            const uintptr_t a = reinterpret_cast<uintptr_t>(dst);
            if (table && (int64_t(C) * hw) % 16 == 0 && hw % 4 == 0 && (a & 15) == 0 &&
                (gcodes == nullptr || ohw % 4 == 0))
                write_slab_words<16>(dst, T, C, hw, lean, pass == 0, wsrc, pass == 0 ? tsrc : first, phw16);
            else if (table && (int64_t(C) * hw) % 4 == 0 && hw % 4 == 0 && (a & 3) == 0 &&
                     (gcodes == nullptr || ohw % 4 == 0))
                write_slab_words<4>(dst, T, C, hw, lean, pass == 0, wsrc, pass == 0 ? tsrc : first, phw16);
            else
                for (int64_t f = threadIdx.x; f < n; f += blockDim.x)
                {
                    uint8_t v = 0;
                    if (lean)
                    {
                        const int plane = int(f / hw), px = int(f - int64_t(plane) * hw);
                        const int t = plane / C, c = plane - t * C;
                        if (pass == 0)
                            v = (int(wsrc[px]) == c && int(tsrc[px]) <= t) ? 1 : 0;
                        else if (ptab)
                            v = int(first[c * phw16 + px]) <= t ? 1 : 0;
                        else
                        {
                            const int py = px / pow_, pxx = px - py * pow_;
                            for (int dy = 0; dy < pky; ++dy)
                                for (int dx = 0; dx < pkx; ++dx)
                                {
                                    const int q = (py * pky + dy) * ow + pxx * pkx + dx;
                                    v |= (int(wsrc[q]) == c && int(tsrc[q]) <= t) ? 1 : 0;
                                }
                        }
                    }
                    dst[f] = v;
                }
        }
        __syncthreads();
    }
}

inline size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Schedule overrides of the tensor-core kernels (0 = automatic), set by an
// autotuner through spk_set_conv_schedule: pipeline stages, accumulators,
// resident CTAs per SM.
struct Schedule
{
    int stages = 0, nacc = 0, ctas = 0;
};
Schedule g_schedule;

struct Plan
{
    int nsplit, n_tile, n_tiles, kblocks, cpad, stages, nacc;
    int parts = 1;  // search plans: channel parts of n_tile run one after another per tile
    bool nhwc;
    uint32_t tmem_cols;
    size_t wimg_bytes, xt_bytes, smem;
};

// single_tile: all output channels in one CTA (required by the fused epilogue).
Plan make_plan(int64_t n, int64_t cin, int64_t h, int64_t w, int64_t cout, int64_t kh, int64_t kw, int precision,
               bool single_tile, int64_t t_fused = 0, bool times = false, int nsplit = 0, bool cl = false)
{
    Plan pl{};
    pl.nsplit = nsplit > 0 ? nsplit : (precision == SPK_CONV_BF16X3 ? 3 : 2);
    const int64_t npad = ceil_div(cout, 16) * 16;
    const int64_t cap = single_tile ? npad : (pl.nsplit == 3 ? 128 : 256);
    pl.n_tiles = int(ceil_div(npad, cap));
    pl.n_tile = int(ceil_div(ceil_div(npad, pl.n_tiles), 16) * 16);
    if (nsplit > 0)
    {
        // search: the channels in parts whose accumulators fit the tensor memory
        while (int64_t(pl.nsplit) * ceil_div(ceil_div(npad, pl.parts), 16) * 16 > 512) ++pl.parts;
        pl.n_tile = int(ceil_div(ceil_div(npad, pl.parts), 16) * 16);
    }
    // channels-last from 8 input channels, and always where the fused layer
    // can take the search path (cl; its kernels gather 8-channel groups)
    pl.nhwc = cin >= 8 || cl || nsplit > 0;
    pl.cpad = int(ceil_div(cin, 8) * 8);
    const int64_t kreal = pl.nhwc ? kh * kw * pl.cpad : kh * kw * cin;
    // search plans (nsplit given): 8-bit operands, 128 elements per K block
    // in the same 128-byte rows
    pl.kblocks = int(ceil_div(kreal, nsplit > 0 ? 2 * BK : BK));
    // two accumulators (the epilogue of one tile overlaps the MMAs of the
    // next) when they fit in the 512 tensor-memory columns
    const uint32_t acc_cols = uint32_t(pl.nsplit * pl.n_tile);
    pl.nacc = 2 * acc_cols <= 512 ? 2 : 1;
    if (g_schedule.nacc == 1) pl.nacc = 1;
    uint32_t cols = 32;
    while (cols < pl.nacc * acc_cols) cols <<= 1;
    pl.tmem_cols = cols;
    pl.wimg_bytes = size_t(pl.n_tiles) * pl.parts * pl.kblocks * pl.nsplit * pl.n_tile * BK * 2;
    // staged copy of the spikes: channels-last [N, H, W, Cpad] (plain), or
    // the first-spike map [B, H, W, Cpad or Cin] plus a flag word (fused)
    if (t_fused > 0)
        pl.xt_bytes = align256(size_t(n / t_fused) * h * w * (pl.nhwc ? pl.cpad : cin)) + 256;
    else
        pl.xt_bytes = pl.nhwc ? size_t(n) * h * w * pl.cpad : 0;
    // (kTimes: the table is followed by the per-warp first-step candidates,
    // two buffers of 4 warps x n_tile ints)
    // (search: 16 group entries per K block, the channels' scales and bounds
    // and two buffers of tile entries)
    const size_t tab = nsplit > 0   ? size_t(pl.kblocks) * 256 + size_t(pl.parts) * pl.n_tile * 8 + 64 + 2 * BM * 8
                       : t_fused > 0 ? (size_t(pl.kblocks) * BK + 8) * 16 + (times ? size_t(pl.n_tile) * 32 : 0)
                       : !pl.nhwc   ? size_t(pl.kblocks) * BK * 16
                                    : size_t(pl.kblocks) * 8 * 16;
    const size_t stage = size_t(BM * BK * 2) + size_t(pl.nsplit) * pl.n_tile * BK * 2;
    // the search kernel aims at two CTAs per SM where its tensor memory allows
    const bool two = nsplit > 0 && cols <= 256;
    const size_t budget = (two ? 110 * 1024 : 225 * 1024) - tab;
    pl.stages = int(std::min<size_t>(g_schedule.stages > 0 ? size_t(g_schedule.stages) : 4, budget / stage));
    size_t smem = size_t(pl.stages) * stage + tab;
    // At most 512 / tmem_cols CTAs may share an SM's tensor memory: size the
    // shared memory so that no more fit.
    const int per_sm = int(512 / cols);
    const size_t floor_smem = (228 * 1024) / size_t(per_sm + 1) + 1024;
    pl.smem = std::max(smem, floor_smem) + 1024;
    return pl;
}

// Split the weights and stage the spikes into the workspace; fill the
// fields of P shared by both epilogues.
//
// Fused staging: the first-spike map [B, H, W, Cp] u8 (Cp = Cpad or Cin) of
// the input [B, T, Cin, H, W]: the first step with a non-zero value, T when
// none, 0xFF in pad channels.  A value other than 0/1, or a zero after a
// one, sets *flag: the producers then gather from the spikes themselves.
__global__ void fst_stage_kernel(const uint8_t *__restrict__ in, uint8_t *__restrict__ fst, int *__restrict__ flag,
                                 int64_t b, int t, int c, int64_t hw, int cp)
{
    const int64_t total = b * cp * hw, st = int64_t(c) * hw;
    bool bad = false;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t px = i % hw, r = i / hw, smp = r / cp;
        const int ch = int(r - smp * cp);
        int first = 0xFF;
        if (ch < c)
        {
            const uint8_t *p = in + (smp * t * c + ch) * hw + px;
            first = t;
            for (int q0 = 0; q0 < t; q0 += 8)
            {
                uint32_t v[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) v[u] = (q0 + u < t) ? p[int64_t(q0 + u) * st] : 0u;
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (q0 + u < t)
                    {
                        bad |= v[u] > 1 || (v[u] == 0 && first < t);
                        if (v[u] != 0 && first == t) first = q0 + u;
                    }
            }
        }
        fst[(smp * hw + px) * cp + ch] = uint8_t(first);
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

// The same map from 32-bit words (H*W a multiple of 4, input 4-byte
// aligned): a CTA takes one sample and a range of npx pixels of every
// channel.  For one step those are C runs of npx bytes, the whole contiguous
// [C, H*W] block when the range is the image, so consecutive threads read
// consecutive words (four pixels of one channel).  The [pixel][channel] tile
// (rows padded to Cp + 1 bytes, which spreads a warp's stores over the
// banks) goes out as contiguous rows.
__global__ void __launch_bounds__(256) fst_stage_words_kernel(const uint8_t *__restrict__ in, uint8_t *__restrict__ fst,
                                                              int *__restrict__ flag, int t, int c, int hw, int cp,
                                                              int ppc)
{
    extern __shared__ uint8_t tile[];  // [ppc][cp + 1]
    const int rs = cp + 1;
    const int64_t smp = blockIdx.y;
    const int px0 = blockIdx.x * ppc;
    const int npx = min(ppc, hw - px0);
    const int gw = npx / 4;  // words per channel run
    const int64_t st = int64_t(c) * hw / 4;
    const uint32_t *base = reinterpret_cast<const uint32_t *>(in + smp * t * c * int64_t(hw) + px0);
    bool bad = false;
    for (int it = threadIdx.x; it < c * gw; it += blockDim.x)
    {
        const int ch = it / gw, p = 4 * (it - ch * gw);
        const uint32_t *src = base + (int64_t(ch) * hw + p) / 4;
        // On cumulative 0/1 input the first spike is the number of zero
        // steps: T minus the byte-wise sum of the words (no carries, as each
        // byte sum is at most T < 256).  Any other byte value, or a one
        // followed by a zero, is flagged.
        // All (up to 16) steps' loads are in flight together.
        uint32_t sum = 0, prev = 0, odd = 0;
        for (int q0 = 0; q0 < t; q0 += 16)
        {
            uint32_t v[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) v[u] = (q0 + u < t) ? src[int64_t(q0 + u) * st] : 0u;
#pragma unroll
            for (int u = 0; u < 16; ++u)
                if (q0 + u < t)  // the same for every thread
                {
                    sum += v[u];
                    odd |= (v[u] & 0xFEFEFEFEu) | (prev & ~v[u]);
                    prev = v[u];
                }
        }
        bad |= odd != 0;
        const uint32_t first = uint32_t(t) * 0x01010101u - sum;
#pragma unroll
        for (int l = 0; l < 4; ++l) tile[(p + l) * rs + ch] = uint8_t(first >> (8 * l));
    }
    for (int it = threadIdx.x; it < npx * (cp - c); it += blockDim.x)
    {
        const int px = it / (cp - c);
        tile[px * rs + c + (it - px * (cp - c))] = 0xFF;
    }
    __syncthreads();
    uint8_t *dst = fst + (smp * hw + px0) * int64_t(cp);
    if (cp % 4 == 0)
        for (int i = threadIdx.x; i < npx * cp / 4; i += blockDim.x)
        {
            const int px = (4 * i) / cp, ch = 4 * i - px * cp;
            const uint8_t *r = tile + px * rs + ch;
            reinterpret_cast<uint32_t *>(dst)[i] =
                uint32_t(r[0]) | uint32_t(r[1]) << 8 | uint32_t(r[2]) << 16 | uint32_t(r[3]) << 24;
        }
    else
        for (int i = threadIdx.x; i < npx * cp; i += blockDim.x) dst[i] = tile[(i / cp) * rs + i % cp];
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

// The same for a whole image per CTA whose step slab (C * H * W bytes) is a
// multiple of 8: the slab is read as flat 8-byte words (a warp reads 256
// contiguous bytes of every step, twice the run of the word version, which
// keeps DRAM pages open longer), each byte placed by its (channel, pixel).
__global__ void __launch_bounds__(256) fst_stage_slab_kernel(const uint8_t *__restrict__ in, uint8_t *__restrict__ fst,
                                                             int *__restrict__ flag, int t, int c, int hw, int cp)
{
    extern __shared__ uint8_t tile[];  // [hw][cp + 1]
    const int rs = cp + 1;
    const int64_t smp = blockIdx.y;
    const int64_t words = int64_t(c) * hw / 8;  // per step
    const uint2 *base = reinterpret_cast<const uint2 *>(in + smp * t * c * int64_t(hw));
    bool bad = false;
    for (int it = threadIdx.x; it < words; it += blockDim.x)
    {
        const uint2 *src = base + it;
        uint32_t s0 = 0, s1 = 0, p0 = 0, p1 = 0, odd = 0;
        for (int q0 = 0; q0 < t; q0 += 16)
        {
            uint2 v[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) v[u] = (q0 + u < t) ? src[int64_t(q0 + u) * words] : make_uint2(0u, 0u);
#pragma unroll
            for (int u = 0; u < 16; ++u)
                if (q0 + u < t)  // the same for every thread
                {
                    s0 += v[u].x, s1 += v[u].y;
                    odd |= (v[u].x & 0xFEFEFEFEu) | (p0 & ~v[u].x) | (v[u].y & 0xFEFEFEFEu) | (p1 & ~v[u].y);
                    p0 = v[u].x, p1 = v[u].y;
                }
        }
        bad |= odd != 0;
        const uint32_t f0 = uint32_t(t) * 0x01010101u - s0, f1 = uint32_t(t) * 0x01010101u - s1;
        int pos = 8 * it, ch = pos / hw, px = pos - ch * hw;
#pragma unroll
        for (int l = 0; l < 8; ++l)
        {
            tile[px * rs + ch] = uint8_t((l < 4 ? f0 : f1) >> (8 * (l & 3)));
            if (++px == hw) px = 0, ++ch;
        }
    }
    for (int it = threadIdx.x; it < hw * (cp - c); it += blockDim.x)
    {
        const int px = it / (cp - c);
        tile[px * rs + c + (it - px * (cp - c))] = 0xFF;
    }
    __syncthreads();
    uint8_t *dst = fst + smp * hw * int64_t(cp);
    if (cp % 4 == 0)
        for (int i = threadIdx.x; i < hw * cp / 4; i += blockDim.x)
        {
            const int px = (4 * i) / cp, ch = 4 * i - px * cp;
            const uint8_t *r = tile + px * rs + ch;
            reinterpret_cast<uint32_t *>(dst)[i] =
                uint32_t(r[0]) | uint32_t(r[1]) << 8 | uint32_t(r[2]) << 16 | uint32_t(r[3]) << 24;
        }
    else
        for (int i = threadIdx.x; i < hw * cp; i += blockDim.x) dst[i] = tile[(i / cp) * rs + i % cp];
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

// First-spike map [B, H, W, Cp] from F32 times [B, C, H, W] (values >= T or
// not finite: never = T; pad channels 0xFF).
__global__ void times_fst_kernel(const float *__restrict__ tin, uint8_t *__restrict__ fst, int64_t b, int c, int64_t hw,
                                 int cp, int T)
{
    const int64_t total = b * hw * cp;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x)
    {
        const int ch = int(i % cp);
        const int64_t r = i / cp, px = r % hw, smp = r / hw;
        uint8_t v = 0xFF;
        if (ch < c)
        {
            const float t = tin[(smp * c + ch) * hw + px];
            v = uint8_t((t >= 0.f && t < float(T)) ? int(t) : T);
        }
        fst[i] = v;
    }
}

// t_fused > 0: stage for the fused (pixel, time) rows of t_fused steps.
TcParams prepare(const Plan &pl, const void *in, const float *kernel, int64_t n, int64_t cin, int64_t h, int64_t w,
                 int64_t cout, int64_t kh, int64_t kw, int64_t sy, int64_t sx, Pad4 p, int64_t oh, int64_t ow,
                 uint8_t *ws, cudaStream_t s, int64_t t_fused = 0, int64_t nnets = 1, const float *times = nullptr)
{
    SPK_REQUIRE(pl.kblocks <= kMaxKBlocks, "Cin*KH*KW is too large for the tensor-core path");
    SPK_REQUIRE(pl.stages >= 2 && pl.smem <= 227 * 1024, "tile does not fit in shared memory");
    SPK_REQUIRE((reinterpret_cast<uintptr_t>(ws) & 255) == 0, "workspace must be 256-byte aligned");
    uint8_t *wimg = ws;
    const int64_t wthreads = int64_t(pl.n_tiles) * pl.kblocks * pl.n_tile * 8;
    SPK_REQUIRE(nnets >= 1 && nnets <= 65535, "invalid number of networks");
    int *negw = nullptr;
    if (t_fused > 0)
    {
        // the flag word sits after the first-spike map's flag
        const int64_t cp = pl.nhwc ? pl.cpad : cin;
        negw = reinterpret_cast<int *>(ws + size_t(nnets) * align256(pl.wimg_bytes) +
                                       align256(size_t(n / t_fused) * h * w * cp) + 128);
        SPK_CUDA(cudaMemsetAsync(negw, 0, sizeof(int), s));
    }
    const dim3 sgrid(grid_for(wthreads, 256), unsigned(nnets));
    split_weights_kernel<<<sgrid, 256, 0, s>>>(kernel, reinterpret_cast<uint4 *>(wimg), int(cout), int(cin),
                                               int(kh * kw), pl.nhwc ? 1 : 0, pl.cpad, pl.kblocks, pl.n_tile,
                                               pl.n_tiles, pl.nsplit, int64_t(align256(pl.wimg_bytes) / 16), negw);
    SPK_LAUNCHED();
    const uint8_t *a_src = static_cast<const uint8_t *>(in);
    TcParams P{};
    P.negw = negw;
    P.wimg_stride = int64_t(align256(pl.wimg_bytes));
    uint8_t *xt = wimg + size_t(nnets) * align256(pl.wimg_bytes);
    if (t_fused > 0)
    {
        const int64_t b = n / t_fused, cp = pl.nhwc ? pl.cpad : cin;
        int *flag = reinterpret_cast<int *>(xt + align256(size_t(b) * h * w * cp));
        SPK_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s));
        if (times)
        {
            times_fst_kernel<<<grid_for(b * h * w * cp, 256), 256, 0, s>>>(times, xt, b, int(cin), h * w, int(cp),
                                                                          int(t_fused));
            SPK_LAUNCHED();
            P.raw = nullptr;
            P.flag = flag;
            P.img_stride = h * w * cp;
            a_src = xt;
        }
        else
        {
            // whole images when their tile fits in 48 KB, else the longest runs
            // of whole words that do
            const int64_t ppc = std::min<int64_t>(h * w, (48 * 1024 / (cp + 1)) & ~int64_t(3));
            const size_t tile = size_t(ppc) * (cp + 1);
            if (ppc == h * w && (cin * h * w) % 8 == 0 && reinterpret_cast<uintptr_t>(a_src) % 8 == 0 &&
                b <= 65535)
                fst_stage_slab_kernel<<<dim3(1u, unsigned(b)), 256, tile, s>>>(a_src, xt, flag, int(t_fused), int(cin),
                                                                              int(h * w), int(cp));
            else if ((h * w) % 4 == 0 && reinterpret_cast<uintptr_t>(a_src) % 4 == 0 && ppc >= 4 &&
                     h * w < (int64_t(1) << 31) && b <= 65535)
                fst_stage_words_kernel<<<dim3(unsigned(ceil_div(h * w, ppc)), unsigned(b)), 256, tile, s>>>(
                    a_src, xt, flag, int(t_fused), int(cin), int(h * w), int(cp), int(ppc));
            else
                fst_stage_kernel<<<grid_for(b * cp * h * w, 256), 256, 0, s>>>(a_src, xt, flag, b, int(t_fused), int(cin),
                                                                               h * w, int(cp));
            SPK_LAUNCHED();
            P.raw = a_src;
            P.flag = flag;
            a_src = xt;
            P.img_stride = h * w * cp;  // per sample
        }
    }
    else if (pl.nhwc)
    {
        const int64_t work = n * h * w * (pl.cpad / 8);
        to_channels_last_kernel<<<grid_for(work, 256), 256, 0, s>>>(a_src, reinterpret_cast<uint2 *>(xt), n,
                                                                    int(cin), h * w, pl.cpad);
        SPK_LAUNCHED();
        a_src = xt;
        P.ps = pl.cpad, P.rs = w * pl.cpad, P.cs = 1;
        P.img_stride = h * w * pl.cpad;
    }
    else
    {
        P.ps = 1, P.rs = w, P.cs = h * w;
        P.img_stride = cin * h * w;
    }
    P.in = a_src;
    P.wimg = wimg;
    P.ohw = oh * ow;
    {
        const DivMagic a = div_magic(uint32_t(oh * ow)), c = div_magic(uint32_t(ow));
        P.ohw_m = a.m, P.ohw_sh = a.sh, P.ow_m = c.m, P.ow_sh = c.sh;
    }
    P.cin = int(cin), P.h = int(h), P.w = int(w), P.cout = int(cout), P.kh = int(kh), P.kw = int(kw);
    P.oh = int(oh), P.ow = int(ow), P.sy = int(sy), P.sx = int(sx), P.top = int(p.top), P.left = int(p.left);
    P.kblocks = pl.kblocks, P.n_tile = pl.n_tile, P.n_tiles = pl.n_tiles, P.nsplit = pl.nsplit;
    P.cpad = pl.cpad, P.nhwc = pl.nhwc ? 1 : 0;
    P.tmem_cols = pl.tmem_cols;
    P.stages = pl.stages, P.nacc = pl.nacc;
    P.idesc = idesc_bf16_f32(BM, pl.n_tile);
    return P;
}

template <int MODE>
void launch(const TcParams &P, const Plan &pl, cudaStream_t s)
{
    const bool two = MODE == kSearch && pl.tmem_cols <= 256;
    auto kern = two ? search_ws_kernel : conv_ws_kernel<MODE>;
    const int threads = two ? kSearchThreads : kWsThreads;
    SPK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(pl.smem)));
    SPK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    int per_sm = 1;
    SPK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, pl.smem));
    // the two-CTA search kernel is sized for two per SM (its registers, shared
    // memory and tensor memory were chosen for it); the runtime's estimate
    // can fall short of what the hardware places
    if (two) per_sm = std::max(per_sm, 2);
    per_sm = std::max(1, std::min<int>(per_sm, int(512 / pl.tmem_cols)));
    if (g_schedule.ctas > 0) per_sm = std::min(per_sm, g_schedule.ctas);
    const int64_t grid = std::min<int64_t>(P.tiles, int64_t(sm_count()) * per_sm);
    kern<<<unsigned(grid), threads, pl.smem, s>>>(P);
    SPK_LAUNCHED();
}

struct FusedLayout
{
    Plan pl, pl4;  // dense fused kernel; search kernels (3 or 4 split terms)
    int tp_log2, pp;
    int64_t npix, oh, ow;
    size_t rec_off, min_off, max_off;
    // search path (search_ok): fixed-split weights, channel bounds + launch
    // info, counters, per-pixel state, two bisection lists, the list of
    // winners to re-read at T - 1, two lists of rows to recompute
    bool search_ok;
    size_t w4_off, echan_off, wm_off, cnt_off, state_off, la_off, lb_off, fin_off, fa_off, fb_off, va_off, vb_off;
    size_t lt_off, bc_off;  // the rows' next entries by row index; the compaction's per-block counts
    size_t tlo_off;         // per pixel, the first step the bound allows a spike at
    size_t total;
};

FusedLayout fused_layout(int64_t b, int64_t t, int64_t cin, int64_t h, int64_t w, int64_t cout, int64_t kh, int64_t kw,
                         int64_t sy, int64_t sx, Pad4 p, int precision, int64_t nnets = 1)
{
    FusedLayout L{};
    L.oh = (h + p.top + p.bottom - kh) / sy + 1;
    L.ow = (w + p.left + p.right - kw) / sx + 1;
    L.pl = make_plan(b * t, cin, h, w, cout, kh, kw, precision, true, t, false, 0, nnets == 1);
    // three-term accumulators of more than 170 channels exceed the 512
    // tensor-memory columns: the dense kernel then keeps two terms (its
    // near-threshold rows are re-decided in FP64 at either split)
    if (precision == SPK_CONV_BF16X3 && L.pl.nsplit * L.pl.n_tile > 512)
        L.pl = make_plan(b * t, cin, h, w, cout, kh, kw, SPK_CONV_BF16X2, true, t, false, 0, nnets == 1);
    int tp = 1, lg = 0;
    while (tp < t) tp <<= 1, ++lg;
    L.tp_log2 = lg;
    L.pp = BM / tp;
    L.npix = b * L.oh * L.ow;
    size_t off = size_t(nnets) * align256(L.pl.wimg_bytes) + align256(L.pl.xt_bytes);
    L.rec_off = off;
    off += align256(size_t(L.npix) * 16);
    L.min_off = off;
    off += align256(size_t(b) * 4);
    L.max_off = off;
    off += align256(size_t(b) * 4);
    L.pl4 = make_plan(b * t, cin, h, w, cout, kh, kw, precision, true, t, false, kSearchTerms);
    L.search_ok = nnets == 1 && t <= 127 && L.pl4.n_tiles == 1 && L.pl4.parts <= 8 &&
                  L.pl4.nsplit * L.pl4.n_tile <= 512 &&
                  L.pl4.stages >= 2 && L.pl4.smem <= 227 * 1024 && L.pl4.kblocks <= kMaxKBlocks &&
                  L.pl.xt_bytes < (size_t(1) << 31) && h < 30000 && w < 30000;
    if (L.search_ok)
    {
        const size_t np = size_t(L.npix);
        L.w4_off = off, off += align256(L.pl4.wimg_bytes);
        L.echan_off = off, off += align256(size_t(L.pl4.parts) * L.pl4.n_tile * 8 + 8);
        L.wm_off = off, off += align256(size_t(cin * kh * kw) * 4);
        // 64 counters, then two buffers of per-block entry counts of the list
        // compaction (zeroed together)
        L.cnt_off = off, off += 256 + 2 * align256((np / kCompactItems + 2) * 4);
        L.bc_off = L.cnt_off + 256;
        L.state_off = off, off += align256(np * 16);
        L.la_off = off, off += align256(np * 8);
        L.lb_off = off, off += align256(np * 8);
        L.fin_off = off, off += align256(np * 8);
        L.fa_off = off, off += align256(np * 16);
        L.fb_off = off, off += align256(np * 16);
        L.va_off = off, off += align256(np * 16);
        L.vb_off = off, off += align256(np * 16);
        L.lt_off = off, off += align256(np * 8);
        L.tlo_off = off, off += align256(np);
    }
    L.total = off;
    return L;
}
}  // namespace

size_t conv_tc_workspace(int64_t n, int64_t cin, int64_t h, int64_t w, int64_t cout, int64_t kh, int64_t kw,
                         int precision)
{
    Plan pl = make_plan(n, cin, h, w, cout, kh, kw, precision, false);
    return align256(pl.wimg_bytes) + align256(pl.xt_bytes);
}

void conv_tc(const void *in, spk_dtype itype, const float *kernel, float *out, int64_t n, int64_t cin, int64_t h,
             int64_t w, int64_t cout, int64_t kh, int64_t kw, int64_t sy, int64_t sx, Pad4 p, int64_t oh, int64_t ow,
             int precision, void *ws, size_t ws_bytes, cudaStream_t s)
{
    if (itype != SPK_U8) throw Error(SPK_ERR_UNSUPPORTED, "the tensor-core path takes U8 spikes");
    Plan pl = make_plan(n, cin, h, w, cout, kh, kw, precision, false);
    SPK_REQUIRE(ws != nullptr && ws_bytes >= align256(pl.wimg_bytes) + align256(pl.xt_bytes), "workspace is too small");
    TcParams P = prepare(pl, in, kernel, n, cin, h, w, cout, kh, kw, sy, sx, p, oh, ow, static_cast<uint8_t *>(ws), s);
    P.out = out;
    P.M = n * oh * ow;
    P.tiles = ceil_div(P.M, BM) * pl.n_tiles;
    launch<kPotentials>(P, pl, s);
}
}  // namespace spk

using namespace spk;

extern "C" {

spk_status spk_set_conv_schedule(int stages, int nacc, int ctas_per_sm)
{
    return guarded([&] {
        SPK_REQUIRE(stages == 0 || (stages >= 2 && stages <= kMaxStages), "stages must be 0 or 2..6");
        SPK_REQUIRE(nacc == 0 || nacc == 1 || nacc == 2, "accumulators must be 0, 1 or 2");
        SPK_REQUIRE(ctas_per_sm >= 0 && ctas_per_sm <= 4, "CTAs per SM must be 0..4");
        g_schedule = Schedule{stages, nacc, ctas_per_sm};
    });
}

unsigned long long spk_recheck_count(int reset)
{
    unsigned long long v = 0;
    if (cudaMemcpyFromSymbol(&v, spk::g_rechecks, sizeof(v)) != cudaSuccess) return ~0ull;
    if (reset)
    {
        unsigned long long z = 0;
        if (cudaMemcpyToSymbol(spk::g_rechecks, &z, sizeof(z)) != cudaSuccess) return ~0ull;
    }
    return v;
}

unsigned long long spk_recompute_count(int reset)
{
    unsigned long long v = 0;
    if (cudaMemcpyFromSymbol(&v, spk::g_recomputes, sizeof(v)) != cudaSuccess) return ~0ull;
    if (reset)
    {
        unsigned long long z = 0;
        if (cudaMemcpyToSymbol(spk::g_recomputes, &z, sizeof(z)) != cudaSuccess) return ~0ull;
    }
    return v;
}

int spk_device_status(int reset)
{
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, spk::g_tc_status, sizeof(int)) != cudaSuccess) return -1;
    if (reset)
    {
        int z = 0;
        if (cudaMemcpyToSymbol(spk::g_tc_status, &z, sizeof(int)) != cudaSuccess) return -1;
    }
    return v;
}

size_t spk_conv_fire_wta_workspace(int64_t b, int64_t t, int64_t cin, int64_t h, int64_t w, int64_t cout, int64_t kh,
                                   int64_t kw, int64_t sy, int64_t sx, const int64_t *pad4, int precision)
{
    try
    {
        const FusedLayout L = fused_layout(b, t, cin, h, w, cout, kh, kw, sy, sx, pad_of(pad4), precision);
        // 0: this layer does not fit one CTA's tensor memory (no fused path)
        if (L.pl.n_tiles != 1 || L.pl.nsplit * L.pl.n_tile > 512) return 0;
        return L.total;
    }
    catch (...)
    {
        return 0;
    }
}

namespace
{
// Networks of a multi-network call: sample ranges on the host (checked),
// sample -> network and per-network thresholds on the device.
struct Nets
{
    int64_t n = 1;
    const int64_t *offsets = nullptr;
    const int32_t *sample_net = nullptr;
    const float *threshold = nullptr;
};

// Launch sequence of the search path (see search_epilogue): the fixed-grid
// split, round 0, ceil(log2 T) bisection rounds, the winners' values at
// T - 1 (with WTA), each round followed by the exact recompute of the rows
// it left open, then the spike writer.  The lists' lengths stay on the
// device (each launch reads them).  Off the search path (device flags) every
// one of these kernels leaves at once, except the writer, which zero-fills
// the spikes for the dense kernel.
void search_layer(const TcParams &P0, const FusedLayout &L, const float *kernel, int64_t count, int64_t pool_ky,
                  int64_t pool_kx, int64_t poh, int64_t pow_, uint8_t *spikes, uint8_t *pooled, uint8_t *base,
                  cudaStream_t s)
{
    const int64_t b = L.npix / (L.oh * L.ow);
    TcParams P = P0;
    const Plan &pl = L.pl4;
    P.wimg = base + L.w4_off;
    P.nsplit = pl.nsplit, P.n_tile = pl.n_tile, P.n_tiles = 1, P.kblocks = pl.kblocks;
    P.tmem_cols = pl.tmem_cols, P.stages = pl.stages, P.nacc = pl.nacc;
    const int nch = pl.parts * pl.n_tile;
    float *echan = reinterpret_cast<float *>(base + L.echan_off);
    float *cscale = echan + nch;
    unsigned *sinfo = reinterpret_cast<unsigned *>(cscale + nch);
    P.nparts = pl.parts;
    P.cscale = cscale;
    int *cnt = reinterpret_cast<int *>(base + L.cnt_off);
    P.echan = echan, P.sinfo = sinfo;
    P.state = reinterpret_cast<int4 *>(base + L.state_off);
    int2 *la = reinterpret_cast<int2 *>(base + L.la_off), *lb = reinterpret_cast<int2 *>(base + L.lb_off);
    int4 *fa = reinterpret_cast<int4 *>(base + L.fa_off), *fb = reinterpret_cast<int4 *>(base + L.fb_off);
    int4 *va = reinterpret_cast<int4 *>(base + L.va_off), *vb = reinterpret_cast<int4 *>(base + L.vb_off);
    P.final_list = reinterpret_cast<int2 *>(base + L.fin_off);
    P.final_count = cnt + 16;
    P.wta = count > 0 ? 1 : 0;
    const int taps = P.kh * P.kw;
    P.kreal = P.nhwc ? taps * P.cpad : taps * P.cin;
    P.tiles = ceil_div(L.npix, BM);
    // the bound pre-filter of round 0, for layers with few inputs per output
    const int cp = P.nhwc ? P.cpad : P.cin;
    const int kr = P.cin * taps;
    // with T <= 32 the pre-filter also bounds each pixel's first step (a bin
    // per step and thread, and the map's bytes, in shared memory)
    const bool want_tlo = P.T <= 32;
    const int64_t bound_base = ((int64_t(P.h) * P.w * 4 + 15) & ~int64_t(15)) + ((int64_t(taps) * P.cpad * 4 + 15) & ~int64_t(15));
    const int64_t bound_tlo = bound_base + ((int64_t(P.T) * 256 * 4 + 15) & ~int64_t(15)) + int64_t(P.h) * P.w * P.cpad;
    const bool use_tlo = want_tlo && bound_tlo <= 48 * 1024;
    const int64_t bound_smem = use_tlo ? bound_tlo : bound_base;
    const bool prefilter = P.nhwc && P.cpad <= 32 && bound_smem <= 48 * 1024;
    unsigned *wmax = reinterpret_cast<unsigned *>(base + L.wm_off);
    uint8_t *tlo = base + L.tlo_off;
    const size_t bcn = align256((size_t(L.npix) / kCompactItems + 2) * 4) / 4;  // ints per count buffer
    SPK_CUDA(cudaMemsetAsync(cnt, 0, 256 + 2 * bcn * 4, s));
    SPK_CUDA(cudaMemsetAsync(sinfo, 0, 8, s));
    if (prefilter) SPK_CUDA(cudaMemsetAsync(wmax, 0, size_t(kr) * 4, s));
    fixed_split_kernel<kSearchTerms><<<unsigned(nch), 256, 0, s>>>(
        kernel, reinterpret_cast<uint4 *>(base + L.w4_off), P.cout, P.cin, taps, P.cpad, pl.kblocks, pl.n_tile, echan,
        cscale, sinfo, P.negw, prefilter ? wmax : nullptr);
    SPK_LAUNCHED();
    if (count > 0)
    {
        search_init_kernel<<<grid_for(b, 256), 256, 0, s>>>(P.mins, P.maxs, b, P.negw, P.flag);
        SPK_LAUNCHED();
    }
    // Rows write their next entry at their own index of lt (step -1: settled);
    // a stable compaction makes the next round's list, in pixel order.
    // The writers of each list also count its valid entries per compaction
    // block, into the buffer of the compaction that will read them (two
    // buffers in turn; each compaction zeroes the other one).
    int2 *lt = reinterpret_cast<int2 *>(base + L.lt_off);
    int *bcs[2] = {reinterpret_cast<int *>(base + L.bc_off), reinterpret_cast<int *>(base + L.bc_off) + bcn};
    const unsigned cblocks = unsigned((L.npix + kCompactItems - 1) / kCompactItems);
    SPK_REQUIRE(cblocks <= 1024u * 64u, "too many output pixels for the list compaction");
    const int self_prefix = cblocks <= unsigned(kSelfPrefixBlocks) ? 1 : 0;
    int ncompact = 0;
    auto compact = [&](const int *n_dev, int2 *out, int *count_out) {
        int *bc = bcs[ncompact & 1], *bnext = bcs[(ncompact + 1) & 1];
        if (!self_prefix)
        {
            list_count_kernel<<<cblocks, 256, 0, s>>>(lt, n_dev, L.npix, bc, P.negw, P.flag);
            SPK_LAUNCHED();
            list_scan_kernel<<<1, 1024, 0, s>>>(bc, int(cblocks), count_out, P.negw, P.flag);
            SPK_LAUNCHED();
        }
        list_scatter_kernel<<<cblocks, 256, 0, s>>>(lt, n_dev, L.npix, bc, self_prefix, count_out, bnext,
                                                    int(cblocks), out, P.negw, P.flag);
        SPK_LAUNCHED();
        ++ncompact;
    };
    P.list_bc = bcs[0];
    if (prefilter)
    {
        search_bound_kernel<<<unsigned(std::min<int64_t>(b, 0x7FFFFFFF)), 256, size_t(bound_smem), s>>>(
            P, wmax, cp, lt, use_tlo ? tlo : nullptr);
        SPK_LAUNCHED();
        compact(nullptr, lb, cnt);
    }
    P.tlo = prefilter && use_tlo ? tlo : nullptr;
    const unsigned fix_grid = unsigned(sm_count() * 4);
    int nsr = 0;
    while ((1 << nsr) < P.T) ++nsr;
    const int rounds = 1 + nsr + (count > 0 ? 1 : 0);
    for (int r = 0; r < rounds; ++r)
    {
        const bool final = count > 0 && r == rounds - 1;
        P.round = r == 0 ? 0 : (final ? 2 : 1);
        P.r0_list = (r == 0 && prefilter) ? 1 : 0;
        P.list_in = final ? P.final_list : (r & 1 ? la : lb);
        P.count_in = final ? P.final_count : cnt + r;
        P.list_out = lt;
        P.list_bc = bcs[ncompact & 1];
        P.tile_ctr = cnt + 48 + r;  // tiles claimed in turn by the CTAs that are running
        P.fix_list = r & 1 ? fb : fa;
        P.fix_count = cnt + 17 + r;
        P.val_list = r & 1 ? vb : va;
        P.val_count = cnt + 40 + r;
        launch<kSearch>(P, pl, s);
        search_fix_kernel<<<fix_grid, 128, 0, s>>>(P, kernel, cp);
        SPK_LAUNCHED();
        // the next bisection round's list (round 0 without a list: all pixels)
        if (r < nsr) compact(r == 0 && !prefilter ? nullptr : P.count_in, r & 1 ? lb : la, cnt + r + 1);
    }
    const int ohw = int(L.oh * L.ow);
    uint8_t *gcodes = nullptr;
    const size_t ohw16 = size_t((ohw + 15) & ~15);
    size_t wsm = 2 * ohw16;
    if (ohw > 16384)
    {
        // the bisection state is no longer needed: its bytes hold the codes
        gcodes = reinterpret_cast<uint8_t *>(P.state);
        wsm = 2 * 16;
        search_codes_kernel<<<grid_for(L.npix, 256), 256, 0, s>>>(P.records, gcodes, L.npix, P.T, P.negw, P.flag);
        SPK_LAUNCHED();
    }
    if (gcodes && (int64_t(P.cout) * ohw) % 16 == 0 && ohw % 4 == 0 && reinterpret_cast<uintptr_t>(spikes) % 16 == 0 &&
        (pool_ky == 0 || (pow_ % 4 == 0 && reinterpret_cast<uintptr_t>(pooled) % 4 == 0)) && b <= 65535)
    {
        const int64_t nq = int64_t(P.cout) * ohw / 16;
        const unsigned xb = unsigned(std::max<int64_t>(1, std::min<int64_t>(ceil_div(nq, 256 * 8),
                                                                            ceil_div(int64_t(sm_count()) * 8, b))));
        search_write_large_kernel<<<dim3(xb, unsigned(b)), 256, 0, s>>>(
            gcodes, L.npix, P.negw, P.flag, spikes, pool_ky > 0 ? pooled : nullptr, P.T, P.cout, ohw, int(L.ow),
            int(pool_ky), int(pool_kx), int(poh), int(pow_));
        SPK_LAUNCHED();
        return;
    }
    // byte table of first firing steps per (channel, pooled cell) when it fits
    const size_t tab_bytes = size_t(P.cout) * size_t(((poh * pow_) + 15) & ~15);
    const int ptab = pool_ky > 0 && wsm + tab_bytes <= 160 * 1024 ? 1 : 0;
    if (ptab) wsm += tab_bytes;
    SPK_CUDA(cudaFuncSetAttribute(search_write_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(wsm)));
    search_write_kernel<<<unsigned(std::min<int64_t>(b, int64_t(sm_count()) * 16)), 256, wsm, s>>>(
        P.records, gcodes, L.npix, P.negw, P.flag, spikes, pool_ky > 0 ? pooled : nullptr, b, P.T, P.cout, ohw,
        int(L.ow), int(pool_ky), int(pool_kx), int(poh), int(pow_), ptab);
    SPK_LAUNCHED();
}

void fused_layer(const void *in, spk_dtype itype, const float *kernel, int64_t b, int64_t t, int64_t cin, int64_t h,
                 int64_t w, int64_t cout, int64_t kh, int64_t kw, int64_t sy, int64_t sx, const int64_t *pad4,
                 double threshold, double value, double inhibit_threshold, double fire_threshold, int64_t ry,
                 int64_t rx, int64_t count, double wta_threshold, uint8_t *spikes, int32_t *winners, int32_t *counts,
                 int64_t pool_ky, int64_t pool_kx, uint8_t *pooled, int precision, void *ws, size_t ws_bytes,
                 spk_stream stream, const Nets &nets)
{
    Pad4 p = pad_of(pad4);
    SPK_REQUIRE(itype == SPK_U8, "the fused layer takes U8 spikes");
    SPK_REQUIRE(precision == SPK_CONV_BF16X2 || precision == SPK_CONV_BF16X3, "the fused layer runs on tcgen05");
    SPK_REQUIRE(b >= 0 && t >= 1 && t <= 32 && cin >= 1 && cout >= 2 && kh >= 1 && kw >= 1 && sy >= 1 && sx >= 1,
                "the fused layer needs 1 <= T <= 32 and at least 2 output channels");
    SPK_REQUIRE(fire_threshold >= 0 && wta_threshold >= 0, "the fused layer needs fire/WTA thresholds >= 0");
    // count == 0: no winner selection (forward passes); winners and
    // counts may then be null
    SPK_REQUIRE(count >= 0 && ry >= 0 && rx >= 0, "invalid WTA radius or count");
    SPK_REQUIRE(spikes != nullptr && (count == 0 || (winners != nullptr && counts != nullptr)), "null output");
    FusedLayout L = fused_layout(b, t, cin, h, w, cout, kh, kw, sy, sx, p, precision, nets.n);
    SPK_REQUIRE(L.oh > 0 && L.ow > 0, "input and kernel shapes are not compatible");
    SPK_REQUIRE(L.pl.n_tiles == 1 && L.pl.nsplit * L.pl.n_tile <= 512, "too many output channels for one CTA");
    SPK_REQUIRE(count == 0 || L.oh * L.ow <= 16384, "the fused WTA keeps at most 16384 pixels per sample");
    SPK_REQUIRE(L.npix < (int64_t(1) << 31), "at most 2^31 - 1 output pixels per call");
    SPK_REQUIRE(ws != nullptr && ws_bytes >= L.total, "workspace is too small");
    if (nets.n > 1 || nets.offsets)
    {
        SPK_REQUIRE(nets.offsets != nullptr && nets.sample_net != nullptr && nets.threshold != nullptr,
                    "null network tables");
        SPK_REQUIRE(nets.offsets[0] == 0 && nets.offsets[nets.n] == b, "network offsets must span the batch");
        for (int64_t q = 0; q < nets.n; ++q)
        {
            SPK_REQUIRE(nets.offsets[q] <= nets.offsets[q + 1], "network offsets must not decrease");
            // a tile is pp consecutive output pixels: none may hold two networks
            SPK_REQUIRE((nets.offsets[q] * L.oh * L.ow) % L.pp == 0,
                        "each network's first output pixel must start a tile (pad the networks' batches)");
        }
    }
    if (b == 0) return;
    cudaStream_t s = stream_of(stream);
    uint8_t *base = static_cast<uint8_t *>(ws);
    TcParams P = prepare(L.pl, in, kernel, b * t, cin, h, w, cout, kh, kw, sy, sx, p, L.oh, L.ow, base, s, t, nets.n);
    if (nets.offsets) P.snet = nets.sample_net, P.net_thr = nets.threshold;
    P.T = int(t), P.tp_log2 = L.tp_log2, P.pp = L.pp, P.npix = L.npix;
    int lp = 0;
    while ((1 << lp) < L.pp) ++lp;
    P.lp_log2 = lp;
    P.thr = float(threshold), P.thv = float(value), P.inh_thr = float(inhibit_threshold);
    P.fire_thr = float(fire_threshold), P.wta_thr = float(wta_threshold);
    P.spikes = spikes;
    int64_t poh = 0, pow_ = 0;
    if (pool_ky > 0)
    {
        SPK_REQUIRE(pool_kx > 0 && pooled != nullptr, "pooling needs a window and an output");
        poh = (L.oh - pool_ky) / pool_ky + 1, pow_ = (L.ow - pool_kx) / pool_kx + 1;
        SPK_REQUIRE(L.oh >= pool_ky && L.ow >= pool_kx, "the pooling window is larger than the output");
        P.pooled = pooled, P.pky = int(pool_ky), P.pkx = int(pool_kx), P.poh = int(poh), P.pow_ = int(pow_);
    }
    // The search path (lean layers, kSearch): chosen here by the thresholds
    // and by the fit of the layer; the kernels themselves check the weights'
    // signs and the input's form and leave the work to the dense kernel
    // otherwise.
    const float fthr = float(threshold), fthv = float(value), finh = float(inhibit_threshold);
    const float ffire = float(fire_threshold), fwta = float(wta_threshold);
    const bool search = L.search_ok && !nets.offsets && fthv <= finh && fthv <= ffire && fthv <= fwta &&
                        finh <= fthr && ffire <= fthr && fwta <= fthr;
    if (count > 0 || search)
    {
        P.records = reinterpret_cast<int4 *>(base + L.rec_off);
        P.mins = reinterpret_cast<unsigned *>(base + L.min_off);
        P.maxs = reinterpret_cast<unsigned *>(base + L.max_off);
    }
    P.M = L.npix * (int64_t(1) << L.tp_log2);
    P.tiles = ceil_div(L.npix, L.pp);
    if (search)
    {
        search_layer(P, L, kernel, count, pool_ky, pool_kx, poh, pow_, spikes, pooled, base, s);
        P.skip_when_lean = 1;
        if (count == 0) P.records = nullptr;
    }
    else
    {
        if (count > 0)
        {
            SPK_CUDA(cudaMemsetAsync(P.mins, 0xFF, size_t(b) * 4, s));
            SPK_CUDA(cudaMemsetAsync(P.maxs, 0x00, size_t(b) * 4, s));
        }
        SPK_CUDA(cudaMemsetAsync(spikes, 0, size_t(b) * t * cout * L.oh * L.ow, s));
        if (pool_ky > 0) SPK_CUDA(cudaMemsetAsync(pooled, 0, size_t(b) * t * cout * poh * pow_, s));
    }
    launch<kFused>(P, L.pl, s);
    if (count == 0) return;
    const int hw = int(L.oh * L.ow);
    const unsigned wgrid = unsigned(ceil_div(b, 4));
    if (hw <= 256)
        wta_records_warp_kernel<8><<<wgrid, 128, 0, s>>>(P.records, P.mins, P.maxs, b, hw, int(L.ow), int(t), int(ry),
                                                          int(rx), int(count), winners, counts);
    else if (hw <= 800)
        wta_records_warp_kernel<25><<<wgrid, 128, 0, s>>>(P.records, P.mins, P.maxs, b, hw, int(L.ow), int(t),
                                                           int(ry), int(rx), int(count), winners, counts);
    else if (hw <= 1024)
        wta_records_warp_kernel<32><<<wgrid, 128, 0, s>>>(P.records, P.mins, P.maxs, b, hw, int(L.ow), int(t),
                                                           int(ry), int(rx), int(count), winners, counts);
    else
        wta_records_kernel<<<unsigned(b), 256, size_t(hw) * 8, s>>>(P.records, P.mins, P.maxs, hw, int(L.ow), int(t),
                                                                    int(ry), int(rx), int(count), winners, counts);
    SPK_LAUNCHED();
}
}  // namespace

spk_status spk_conv_fire_wta(const void *in, spk_dtype itype, const float *kernel, int64_t b, int64_t t, int64_t cin,
                             int64_t h, int64_t w, int64_t cout, int64_t kh, int64_t kw, int64_t sy, int64_t sx,
                             const int64_t *pad4, double threshold, double value, double inhibit_threshold,
                             double fire_threshold, int64_t ry, int64_t rx, int64_t count, double wta_threshold,
                             uint8_t *spikes, int32_t *winners, int32_t *counts, int64_t pool_ky, int64_t pool_kx,
                             uint8_t *pooled, int precision, void *ws, size_t ws_bytes, spk_stream stream)
{
    return guarded([&] {
        fused_layer(in, itype, kernel, b, t, cin, h, w, cout, kh, kw, sy, sx, pad4, threshold, value,
                    inhibit_threshold, fire_threshold, ry, rx, count, wta_threshold, spikes, winners, counts, pool_ky,
                    pool_kx, pooled, precision, ws, ws_bytes, stream, Nets{});
    });
}

size_t spk_fst_conv_times_workspace(int64_t b, int64_t cin, int64_t h, int64_t w, int64_t cout, int64_t kh,
                                    int64_t kw, int64_t time, int precision)
{
    try
    {
        const Plan pl = make_plan(b * time, cin, h, w, cout, kh, kw, precision, true, time, true);
        if (pl.n_tiles != 1 || pl.nsplit * pl.n_tile > 512) return 0;
        return align256(pl.wimg_bytes) + align256(pl.xt_bytes);
    }
    catch (...)
    {
        return 0;
    }
}

spk_status spk_fst_conv_times(const float *t_in, int64_t b, int64_t cin, int64_t h, int64_t w, const float *kernel,
                              int64_t cout, int64_t kh, int64_t kw, int64_t sy, int64_t sx, const int64_t *pad4,
                              int64_t time, double threshold, float *t_out, int precision, void *ws, size_t ws_bytes,
                              spk_stream stream)
{
    return guarded([&] {
        const Pad4 p = pad_of(pad4);
        SPK_REQUIRE(precision == SPK_CONV_BF16X2 || precision == SPK_CONV_BF16X3, "the layer runs on tcgen05");
        SPK_REQUIRE(b >= 0 && time >= 1 && time <= 126 && cin >= 1 && cout >= 1 && kh >= 1 && kw >= 1 && sy >= 1 &&
                        sx >= 1,
                    "needs 1 <= T <= 126");
        SPK_REQUIRE(t_in != nullptr && kernel != nullptr && t_out != nullptr, "null pointer");
        const int64_t oh = (h + p.top + p.bottom - kh) / sy + 1, ow = (w + p.left + p.right - kw) / sx + 1;
        SPK_REQUIRE(oh > 0 && ow > 0 && h + p.top + p.bottom >= kh && w + p.left + p.right >= kw,
                    "input and kernel shapes are not compatible");
        Plan pl = make_plan(b * time, cin, h, w, cout, kh, kw, precision, true, time, true);
        SPK_REQUIRE(pl.n_tiles == 1 && pl.nsplit * pl.n_tile <= 512, "too many output channels for one CTA");
        SPK_REQUIRE(ws != nullptr && ws_bytes >= align256(pl.wimg_bytes) + align256(pl.xt_bytes),
                    "workspace is too small");
        const int64_t npix = b * oh * ow;
        SPK_REQUIRE(npix < (int64_t(1) << 31), "at most 2^31 - 1 output pixels per call");
        if (b == 0) return;
        cudaStream_t s = stream_of(stream);
        TcParams P = prepare(pl, nullptr, kernel, b * time, cin, h, w, cout, kh, kw, sy, sx, p, oh, ow,
                             static_cast<uint8_t *>(ws), s, time, 1, t_in);
        int tp = 1, lg = 0;
        while (tp < time) tp <<= 1, ++lg;
        P.T = int(time), P.tp_log2 = lg, P.pp = BM / tp, P.npix = npix;
        P.thr = float(threshold);
        P.tout = t_out;
        P.M = npix * tp;
        P.tiles = ceil_div(npix, P.pp);
        launch<kTimes>(P, pl, s);
    });
}

size_t spk_conv_fire_wta_nets_workspace(int64_t nnets, int64_t b, int64_t t, int64_t cin, int64_t h, int64_t w,
                                        int64_t cout, int64_t kh, int64_t kw, int64_t sy, int64_t sx,
                                        const int64_t *pad4, int precision)
{
    try
    {
        if (nnets < 1) return 0;
        const FusedLayout L = fused_layout(b, t, cin, h, w, cout, kh, kw, sy, sx, pad_of(pad4), precision, nnets);
        if (L.pl.n_tiles != 1 || L.pl.nsplit * L.pl.n_tile > 512) return 0;
        return L.total;
    }
    catch (...)
    {
        return 0;
    }
}

spk_status spk_conv_fire_wta_nets(const void *in, spk_dtype itype, const float *kernels, int64_t nnets,
                                  const int64_t *net_offsets_host, const int32_t *sample_net,
                                  const float *net_threshold, int64_t b, int64_t t, int64_t cin, int64_t h, int64_t w,
                                  int64_t cout, int64_t kh, int64_t kw, int64_t sy, int64_t sx, const int64_t *pad4,
                                  double value, double inhibit_threshold, double fire_threshold, int64_t ry,
                                  int64_t rx, int64_t count, double wta_threshold, uint8_t *spikes, int32_t *winners,
                                  int32_t *counts, int64_t pool_ky, int64_t pool_kx, uint8_t *pooled, int precision,
                                  void *ws, size_t ws_bytes, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(nnets >= 1, "at least one network");
        Nets nets;
        nets.n = nnets, nets.offsets = net_offsets_host, nets.sample_net = sample_net, nets.threshold = net_threshold;
        fused_layer(in, itype, kernels, b, t, cin, h, w, cout, kh, kw, sy, sx, pad4, 0.0, value, inhibit_threshold,
                    fire_threshold, ry, rx, count, wta_threshold, spikes, winners, counts, pool_ky, pool_kx, pooled,
                    precision, ws, ws_bytes, stream, nets);
    });
}

}  // extern "C"
