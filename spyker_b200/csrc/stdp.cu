// STDP for conv and fc layers as a per-feature-map ordered scan.
//
// src/spyker/cpu/stdp.cpp:42-169.  The reference applies, sample after sample
// and winner after winner, a soft-bound update to the winner's kernel slice:
//   old = w (F64); m = stabilize ? (old - lower) * (upper - old) : 1;
//   w = clamp(old + (pre <= post ? positive : negative) * m, lower, upper),
// stored back to F32, where pre is the first-spike time of each input in the
// winner's receptive field (T when silent or in the zero pad) and post the
// first-spike time of the winner.  Within a sample winners have distinct
// feature maps, so the only serial dependency is the order of updates to the
// same map.  Kernel A computes (pre, post) for every winner in parallel;
// kernel B gives every (feature map, chunk of weights) a CTA that keeps its
// weights in registers and walks the winner list in the reference order.
#include "common.cuh"

namespace spk
{
inline size_t align256(size_t v) { return (v + 255) & ~size_t(255); }
size_t convstdp_prepost_bytes(int64_t b, int64_t count, int64_t cin, int64_t kh, int64_t kw);

namespace
{
constexpr int kMaxConfigs = 16;
constexpr int kScanThreads = 256;
constexpr int kWinnerTile = 1024;  // winner records compacted per pass (4 per thread)

struct Configs
{
    double pos[kMaxConfigs], neg[kMaxConfigs], lo[kMaxConfigs], hi[kMaxConfigs];
    int stab[kMaxConfigs];
    int n;
};

// First step with a non-zero value (t when none).  Loads go in groups of 8
// independent reads, so a thread waits for memory twice per 16 steps instead
// of once per step.
template <typename T>
__device__ __forceinline__ uint16_t first_spike(const T *p, int t, int64_t stride)
{
    for (int q0 = 0; q0 < t; q0 += 8)
    {
        T v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = (q0 + u < t) ? p[int64_t(q0 + u) * stride] : T(0);
        int f = -1;
#pragma unroll
        for (int u = 7; u >= 0; --u)
            if (v[u] != T(0)) f = u;
        if (f >= 0) return uint16_t(q0 + f);
    }
    return uint16_t(t);
}

// Kernel A (conv): one CTA per (sample, winner slot).
template <typename T>
__global__ void conv_prepost_kernel(const T *__restrict__ in, const T *__restrict__ out, int t, int cin, int h, int w,
                                    int cout, int oh, int ow, int kh, int kw, int sy, int sx, int top, int left,
                                    const int32_t *__restrict__ winners, const int32_t *__restrict__ counts, int count,
                                    uint16_t *__restrict__ pre, uint16_t *__restrict__ post)
{
    const int s = blockIdx.x / count, j = blockIdx.x % count;
    if (j >= counts[s]) return;
    const int32_t *e = winners + (int64_t(s) * count + j) * 5;
    const int wz = e[2], wy = e[3], wx = e[4];
    const int k = cin * kh * kw;
    uint16_t *p = pre + (int64_t(s) * count + j) * k;
    const int64_t istride = int64_t(cin) * h * w;
    for (int i = threadIdx.x; i < k; i += blockDim.x)
    {
        int c = i / (kh * kw), r = i % (kh * kw), ky = r / kw, kx = r % kw;
        int yy = wy * sy + ky - top, xx = wx * sx + kx - left;
        uint16_t v = uint16_t(t);
        if (yy >= 0 && yy < h && xx >= 0 && xx < w)
            v = first_spike(in + int64_t(s) * t * istride + (int64_t(c) * h + yy) * w + xx, t, istride);
        p[i] = v;
    }
    if (threadIdx.x == 0)
    {
        const int64_t ostride = int64_t(cout) * oh * ow;
        bool ok = wz >= 0 && wz < cout && wy >= 0 && wy < oh && wx >= 0 && wx < ow;
        post[int64_t(s) * count + j] =
            ok ? first_spike(out + int64_t(s) * t * ostride + (int64_t(wz) * oh + wy) * ow + wx, t, ostride) : 0;
    }
}

// First-spike map of the whole input, [B, Cin, H, W] u16 (T when silent):
// one coalesced pass over the spikes instead of T strided loads per
// receptive-field element and winner.
template <typename T>
__global__ void first_spike_map_kernel(const T *__restrict__ in, uint16_t *__restrict__ fst, int64_t b, int t,
                                       int64_t x)
{
    const int64_t total = b * x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t s = k / x, j = k - s * x;
        fst[k] = first_spike(in + s * t * x + j, t, x);
    }
}

// U8 spikes with X a multiple of 4: four neighbouring positions per thread
// from 32-bit loads.
__global__ void first_spike_map_u8x4_kernel(const uint32_t *__restrict__ in, uint2 *__restrict__ fst, int64_t b, int t,
                                            int64_t x4)
{
    const int64_t total = b * x4;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t s = k / x4, j = k - s * x4;
        const uint32_t *p = in + s * t * x4 + j;
        uint32_t f[4] = {uint32_t(t), uint32_t(t), uint32_t(t), uint32_t(t)};
        uint32_t seen = 0;  // byte lanes that have spiked
        for (int q0 = 0; q0 < t && seen != 0x0f; q0 += 8)
        {
            uint32_t v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) v[u] = (q0 + u < t) ? p[int64_t(q0 + u) * x4] : 0u;
#pragma unroll
            for (int u = 0; u < 8; ++u)
#pragma unroll
                for (int l = 0; l < 4; ++l)
                    if (!(seen & (1u << l)) && ((v[u] >> (8 * l)) & 0xffu))
                        f[l] = uint32_t(q0 + u), seen |= 1u << l;
        }
        fst[k] = make_uint2(f[0] | (f[1] << 16), f[2] | (f[3] << 16));
    }
}

// The same for T < 256 with every step's load in flight (16 at a time):
// on cumulative 0/1 spikes the first spike of a byte lane is T minus the
// lane's byte sum (no carries for T < 256); a word with any other value, or a
// one followed by a zero, is redone with the lane-by-lane scan.
__global__ void first_spike_map_u8x4_sum_kernel(const uint32_t *__restrict__ in, uint2 *__restrict__ fst, int64_t b,
                                                int t, int64_t x4)
{
    const int64_t total = b * x4;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t s = k / x4, j = k - s * x4;
        const uint32_t *p = in + s * t * x4 + j;
        uint32_t sum = 0, prev = 0, odd = 0;
        for (int q0 = 0; q0 < t; q0 += 16)
        {
            uint32_t v[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) v[u] = (q0 + u < t) ? __ldg(p + int64_t(q0 + u) * x4) : 0u;
#pragma unroll
            for (int u = 0; u < 16; ++u)
                if (q0 + u < t)  // the same for every thread
                {
                    sum += v[u];
                    odd |= (v[u] & 0xFEFEFEFEu) | (prev & ~v[u]);
                    prev = v[u];
                }
        }
        uint32_t f[4];
        if (odd == 0)
        {
#pragma unroll
            for (int l = 0; l < 4; ++l) f[l] = uint32_t(t) - ((sum >> (8 * l)) & 0xffu);
        }
        else
        {
            f[0] = f[1] = f[2] = f[3] = uint32_t(t);
            uint32_t seen = 0;
            for (int q = 0; q < t && seen != 0x0f; ++q)
            {
                const uint32_t v = p[int64_t(q) * x4];
#pragma unroll
                for (int l = 0; l < 4; ++l)
                    if (!(seen & (1u << l)) && ((v >> (8 * l)) & 0xffu)) f[l] = uint32_t(q), seen |= 1u << l;
            }
        }
        fst[k] = make_uint2(f[0] | (f[1] << 16), f[2] | (f[3] << 16));
    }
}

// The same on 8-byte words (8 positions per thread): a warp reads 256
// contiguous bytes of every step, twice the run of the 4-byte version, for
// rows of a multiple of 8 bytes.
__global__ void first_spike_map_u8x8_sum_kernel(const uint2 *__restrict__ in, uint4 *__restrict__ fst, int64_t b,
                                                int t, int64_t x8)
{
    const int64_t total = b * x8;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t s = k / x8, j = k - s * x8;
        const uint2 *p = in + s * t * x8 + j;
        uint32_t sum0 = 0, sum1 = 0, prev0 = 0, prev1 = 0, odd = 0;
        for (int q0 = 0; q0 < t; q0 += 16)
        {
            uint2 v[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) v[u] = (q0 + u < t) ? __ldg(p + int64_t(q0 + u) * x8) : make_uint2(0u, 0u);
#pragma unroll
            for (int u = 0; u < 16; ++u)
                if (q0 + u < t)  // the same for every thread
                {
                    sum0 += v[u].x, sum1 += v[u].y;
                    odd |= (v[u].x & 0xFEFEFEFEu) | (prev0 & ~v[u].x) | (v[u].y & 0xFEFEFEFEu) | (prev1 & ~v[u].y);
                    prev0 = v[u].x, prev1 = v[u].y;
                }
        }
        uint32_t f[8];
        if (odd == 0)
        {
#pragma unroll
            for (int l = 0; l < 4; ++l)
                f[l] = uint32_t(t) - ((sum0 >> (8 * l)) & 0xffu), f[4 + l] = uint32_t(t) - ((sum1 >> (8 * l)) & 0xffu);
        }
        else
        {
#pragma unroll
            for (int l = 0; l < 8; ++l) f[l] = uint32_t(t);
            uint32_t seen = 0;
            for (int q = 0; q < t && seen != 0xff; ++q)
            {
                const uint2 v = p[int64_t(q) * x8];
#pragma unroll
                for (int l = 0; l < 8; ++l)
                {
                    const uint32_t byte = ((l < 4 ? v.x : v.y) >> (8 * (l & 3))) & 0xffu;
                    if (!(seen & (1u << l)) && byte) f[l] = uint32_t(q), seen |= 1u << l;
                }
            }
        }
        fst[k] = make_uint4(f[0] | (f[1] << 16), f[2] | (f[3] << 16), f[4] | (f[5] << 16), f[6] | (f[7] << 16));
    }
}

// Kernel A (conv) on the first-spike map: one CTA per (sample, winner slot).
template <typename T>
__global__ void conv_prepost_map_kernel(const uint16_t *__restrict__ fst, const T *__restrict__ out, int t, int cin,
                                        int h, int w, int cout, int oh, int ow, int kh, int kw, int sy, int sx, int top,
                                        int left, const int32_t *__restrict__ winners,
                                        const int32_t *__restrict__ counts, int count, uint16_t *__restrict__ pre,
                                        uint16_t *__restrict__ post)
{
    const int s = blockIdx.x / count, j = blockIdx.x % count;
    if (j >= counts[s]) return;
    const int32_t *e = winners + (int64_t(s) * count + j) * 5;
    const int wz = e[2], wy = e[3], wx = e[4];
    const int k = cin * kh * kw;
    uint16_t *p = pre + (int64_t(s) * count + j) * k;
    const uint16_t *f = fst + int64_t(s) * cin * h * w;
    // (c, ky, kx) of element i by multiplying with rounded reciprocals: for
    // i < 2^16 the products' error (< 2^-7) stays below the 0.5 / divisor
    // margin that the +0.5 keeps from the next integer, so the quotients are
    // exact without integer divisions
    const int taps = kh * kw;
    const float inv_taps = 1.0f / float(taps), inv_kw = 1.0f / float(kw);
    for (int i = threadIdx.x; i < k; i += blockDim.x)
    {
        int c, r, ky;
        if (k < 65536)
        {
            c = __float2int_rz(__fmul_rn(float(i) + 0.5f, inv_taps));
            r = i - c * taps;
            ky = __float2int_rz(__fmul_rn(float(r) + 0.5f, inv_kw));
        }
        else
            c = i / taps, r = i - c * taps, ky = r / kw;
        const int kx = r - ky * kw;
        const int yy = wy * sy + ky - top, xx = wx * sx + kx - left;
        p[i] = (yy >= 0 && yy < h && xx >= 0 && xx < w) ? f[(int64_t(c) * h + yy) * w + xx] : uint16_t(t);
    }
    if (threadIdx.x == 0)
    {
        const int64_t ostride = int64_t(cout) * oh * ow;
        const bool ok = wz >= 0 && wz < cout && wy >= 0 && wy < oh && wx >= 0 && wx < ow;
        post[int64_t(s) * count + j] =
            ok ? first_spike(out + int64_t(s) * t * ostride + (int64_t(wz) * oh + wy) * ow + wx, t, ostride) : 0;
    }
}

// Kernel A (fc): pre per (sample, input), post per (sample, winner slot).
template <typename T>
__global__ void fc_prepost_kernel(const T *__restrict__ in, const T *__restrict__ out, int64_t b, int t, int ni, int no,
                                  const int32_t *__restrict__ winners, const int32_t *__restrict__ counts, int count,
                                  uint16_t *__restrict__ pre, uint16_t *__restrict__ post)
{
    const int64_t total = b * ni;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        int64_t s = k / ni, i = k % ni;
        pre[k] = first_spike(in + s * t * ni + i, t, ni);
    }
    const int64_t nw = b * count;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < nw; k += int64_t(gridDim.x) * blockDim.x)
    {
        int64_t s = k / count, j = k % count;
        if (j >= counts[s]) continue;
        int wx = winners[k * 5 + 4];
        post[k] = (wx >= 0 && wx < no) ? first_spike(out + s * t * no + wx, t, no) : 0;
    }
}

// Kernel B: CTA (map, chunk of 256 weights); every thread owns one weight
// and applies the map's winners to it in (sample, slot) order.  Per tile of
// 1024 winner records the CTA compacts the ones of its map (order kept) into
// shared memory; then each thread walks them with the (pre, post) loads of
// the next 8 winners in flight while it updates its weight, so the critical
// path is the weight's own chain of dependent updates.  The map index of a
// winner is field `field` of its record (z for conv, x for fc).
// pre address: pre + s * ps + j * pw + element; post index s * count + j.
// F32_RULE: the event-list STDP of src/spyker/sparse/stdp.cpp:95-97, which
// rounds the soft-bound factor and the updated weight to F32 before the clamp.
// v rounded to the nearest F32 (ties to even), returned as a double: a
// conversion there and back (exact for every value, infinities and
// denormals included).  On B200 this is the shorter dependency: a chain of
// updates measures about 95 cycles per update with it against 149 with the
// rounding done by 64-bit integer operations on the double's bits.
__device__ __forceinline__ double round_f32(double v) { return double(__double2float_rn(v)); }

// One update of a weight kept as a double holding an F32 value.
template <bool F32_RULE>
__device__ __forceinline__ double stdp_update(double old, double d, double lo, double hi, bool stab)
{
    if (F32_RULE)
    {
        const double m = round_f32(stab ? (old - lo) * (hi - old) : 1.0);
        double v = round_f32(fma(d, m, old));
        v = (hi < v) ? hi : v;
        v = (lo < v) ? v : lo;
        return round_f32(v);
    }
    const double m = stab ? (old - lo) * (hi - old) : 1.0;
    double v = fma(d, m, old);
    v = (hi < v) ? hi : v;  // std::min(v, upper)
    v = (lo < v) ? v : lo;  // std::max(lower, .)
    return round_f32(v);
}

constexpr int kAhead = 8;  // winners whose loads are in flight

// The weight's chain over the n compacted winners of this tile; with one
// STDP config (the common case) its constants stay in registers.
template <bool F32_RULE, bool ONE>
__device__ __forceinline__ double stdp_chain(double w, int n, int64_t e, bool act, const int64_t *s_off,
                                             const uint16_t *s_post, const uint8_t *s_cfg,
                                             const uint16_t *__restrict__ pre, const double *s_pos,
                                             const double *s_neg, const double *s_lo, const double *s_hi,
                                             const int *s_stab)
{
    const double pos0 = s_pos[0], neg0 = s_neg[0], lo0 = s_lo[0], hi0 = s_hi[0];
    const bool stab0 = s_stab[0] != 0;
    uint16_t pv[kAhead];
#pragma unroll
    for (int u = 0; u < kAhead; ++u) pv[u] = (act && u < n) ? pre[s_off[u] + e] : 0;
    for (int i0 = 0; i0 < n; i0 += kAhead)
    {
        uint16_t cv[kAhead];
#pragma unroll
        for (int u = 0; u < kAhead; ++u)
        {
            cv[u] = pv[u];
            const int i = i0 + kAhead + u;
            pv[u] = (act && i < n) ? pre[s_off[i] + e] : 0;
        }
#pragma unroll
        for (int u = 0; u < kAhead; ++u)
        {
            const int i = i0 + u;
            if (i < n)
            {
                const bool direct = cv[u] <= s_post[i];
                if (ONE)
                    w = stdp_update<F32_RULE>(w, direct ? pos0 : neg0, lo0, hi0, stab0);
                else
                {
                    const int c = s_cfg[i];
                    w = stdp_update<F32_RULE>(w, direct ? s_pos[c] : s_neg[c], s_lo[c], s_hi[c], s_stab[c] != 0);
                }
            }
        }
    }
    return w;
}

// Several networks (NETS): blockIdx.z = network n with kernels
// [N, maps, k], its samples order[noff[n] .. noff[n+1]) (or the range itself
// when order is null) walked in that order, and its configs
// net_cfg[n][nconf][5] (positive, negative, stabilize, lower, upper).
struct NetScan
{
    const int64_t *noff;
    const int32_t *order;
    const double *net_cfg;
};

// At most 40 registers a thread (six CTAs' worth of an SM's registers): a
// CTA of this long-running scan then fits beside two CTAs of the fused
// layer's search kernel when the update overlaps that layer's rounds.
template <bool F32_RULE, bool NETS>
__global__ void __launch_bounds__(kScanThreads, 6)
    stdp_scan_kernel(float *__restrict__ kernel, int64_t k, int64_t b, int count, int field,
                     const int32_t *__restrict__ winners, const int32_t *__restrict__ counts,
                     const uint16_t *__restrict__ pre, int64_t ps, int64_t pw, const uint16_t *__restrict__ post,
                     Configs cfg, NetScan nets)
{
    // per compacted winner: offset of its pre row, its post time, its config
    __shared__ int64_t s_off[kWinnerTile];
    __shared__ uint16_t s_post[kWinnerTile];
    __shared__ uint8_t s_cfg[kWinnerTile];
    __shared__ int s_warp[kScanThreads / 32];
    __shared__ double s_pos[kMaxConfigs], s_neg[kMaxConfigs], s_lo[kMaxConfigs], s_hi[kMaxConfigs];
    __shared__ int s_stab[kMaxConfigs];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int64_t s_first = 0;  // the network's first slot in order / first sample
    if (NETS)
    {
        const int net = blockIdx.z;
        s_first = nets.noff[net];
        b = nets.noff[net + 1] - s_first;
        kernel += int64_t(net) * gridDim.x * k;
        if (tid < cfg.n)
        {
            const double *c = nets.net_cfg + (int64_t(net) * cfg.n + tid) * 5;
            s_pos[tid] = c[0], s_neg[tid] = c[1], s_stab[tid] = c[2] != 0.0, s_lo[tid] = c[3], s_hi[tid] = c[4];
        }
    }
    else if (tid < cfg.n)
        s_pos[tid] = cfg.pos[tid], s_neg[tid] = cfg.neg[tid], s_lo[tid] = cfg.lo[tid], s_hi[tid] = cfg.hi[tid],
        s_stab[tid] = cfg.stab[tid];
    __syncthreads();
    const int map = blockIdx.x;
    const int64_t e = int64_t(blockIdx.y) * kScanThreads + tid;
    const bool act = e < k;
    // warps whose weights are all past k only help with the compaction
    const bool warp_act = int64_t(blockIdx.y) * kScanThreads + warp * 32 < k;
    double w = act ? double(kernel[int64_t(map) * k + e]) : 0.0;
    const int64_t total = b * count;
    constexpr int per = kWinnerTile / kScanThreads;
    for (int64_t start = 0; start < total; start += kWinnerTile)
    {
        // records start + 4 tid .. + 3: ordered compaction of this map's ones
        unsigned m4 = 0;
        int32_t rr[per];
        uint8_t c4[per];
#pragma unroll
        for (int q = 0; q < per; ++q)
        {
            const int64_t r = start + int64_t(tid) * per + q;
            c4[q] = 0, rr[q] = int32_t(r);
            if (r < total)
            {
                int smp = int(r) / count;
                const int j = int(r) - smp * count;  // r < 2^31
                if (NETS) smp = nets.order ? nets.order[s_first + smp] : int(s_first) + smp;
                if (j < counts[smp])
                {
                    const int32_t *rec = winners + (int64_t(smp) * count + j) * 5;
                    const int32_t c = rec[0];
                    if (rec[field] == map && c >= 0 && c < cfg.n) m4 |= 1u << q, c4[q] = uint8_t(c);
                }
            }
        }
        int x = __popc(m4);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s_warp[warp] = x;
        __syncthreads();
        int before = x - __popc(m4), n = 0;
#pragma unroll
        for (int q = 0; q < kScanThreads / 32; ++q)
        {
            before += q < warp ? s_warp[q] : 0;
            n += s_warp[q];
        }
#pragma unroll
        for (int q = 0; q < per; ++q)
            if (m4 & (1u << q))
            {
                const int r = rr[q], j = r - (r / count) * count;
                int smp = r / count;
                if (NETS) smp = nets.order ? nets.order[s_first + smp] : int(s_first) + smp;
                s_off[before] = int64_t(smp) * ps + int64_t(j) * pw;
                s_post[before] = post[int64_t(smp) * count + j];
                s_cfg[before] = c4[q];
                ++before;
            }
        __syncthreads();
        if (warp_act)
        {
            if (cfg.n == 1)
                w = stdp_chain<F32_RULE, true>(w, n, e, act, s_off, s_post, s_cfg, pre, s_pos, s_neg, s_lo, s_hi,
                                               s_stab);
            else
                w = stdp_chain<F32_RULE, false>(w, n, e, act, s_off, s_post, s_cfg, pre, s_pos, s_neg, s_lo, s_hi,
                                                s_stab);
        }
        __syncthreads();  // the per-winner arrays are rewritten by the next tile
    }
    if (act) kernel[int64_t(map) * k + e] = float(w);  // exact: w holds an F32 value
}

Configs make_configs(const double *c, int64_t n)
{
    SPK_REQUIRE(n > 0, "at least one STDP config must be given");
    SPK_REQUIRE(n <= kMaxConfigs, "at most 16 STDP configs are supported");
    SPK_REQUIRE(c != nullptr, "null configs");
    Configs cfg{};
    for (int64_t i = 0; i < n; ++i)
    {
        cfg.pos[i] = c[i * 5 + 0], cfg.neg[i] = c[i * 5 + 1], cfg.stab[i] = c[i * 5 + 2] != 0;
        cfg.lo[i] = c[i * 5 + 3], cfg.hi[i] = c[i * 5 + 4];
    }
    cfg.n = int(n);
    return cfg;
}

}  // namespace

// Ordered per-map STDP scan over precomputed (pre, post) times; the entry
// point of the event-list STDP.
void launch_stdp_scan(float *kernel, int64_t k, int64_t nmaps, int64_t b, int64_t count, int field,
                      const int32_t *winners, const int32_t *counts, const uint16_t *pre, int64_t ps, int64_t pw,
                      const uint16_t *post, const double *configs, int64_t nconf, bool f32_rule, cudaStream_t s)
{
    Configs cfg = make_configs(configs, nconf);
    SPK_REQUIRE(b * count < (int64_t(1) << 31), "at most 2^31 - 1 winner records");
    dim3 grid(unsigned(nmaps), unsigned(ceil_div(k, kScanThreads)));
    if (f32_rule)
        stdp_scan_kernel<true, false><<<grid, kScanThreads, 0, s>>>(kernel, k, b, int(count), field, winners, counts,
                                                                   pre, ps, pw, post, cfg, NetScan{});
    else
        stdp_scan_kernel<false, false><<<grid, kScanThreads, 0, s>>>(kernel, k, b, int(count), field, winners, counts,
                                                                    pre, ps, pw, post, cfg, NetScan{});
    SPK_LAUNCHED();
}

// The scan of several networks in one launch (see NetScan).
void launch_stdp_scan_nets(float *kernels, int64_t nnets, int64_t k, int64_t nmaps, int64_t b, int64_t count,
                           int field, const int32_t *winners, const int32_t *counts, const uint16_t *pre, int64_t ps,
                           int64_t pw, const uint16_t *post, const int64_t *noff, const int32_t *order,
                           const double *net_cfg, int64_t nconf, bool f32_rule, cudaStream_t s)
{
    SPK_REQUIRE(nconf >= 1 && nconf <= kMaxConfigs, "1 to 16 STDP configs per network");
    SPK_REQUIRE(nnets >= 1 && nnets <= 65535 && noff != nullptr && net_cfg != nullptr, "invalid network tables");
    SPK_REQUIRE(b * count < (int64_t(1) << 31), "at most 2^31 - 1 winner records");
    Configs cfg{};
    cfg.n = int(nconf);
    const NetScan nets{noff, order, net_cfg};
    dim3 grid(unsigned(nmaps), unsigned(ceil_div(k, kScanThreads)), unsigned(nnets));
    if (f32_rule)
        stdp_scan_kernel<true, true><<<grid, kScanThreads, 0, s>>>(kernels, k, b, int(count), field, winners, counts,
                                                                  pre, ps, pw, post, cfg, nets);
    else
        stdp_scan_kernel<false, true><<<grid, kScanThreads, 0, s>>>(kernels, k, b, int(count), field, winners, counts,
                                                                   pre, ps, pw, post, cfg, nets);
    SPK_LAUNCHED();
}

// (pre, post) times of every conv winner: the first-spike map of the input
// (fst, [B, Cin, H, W] u16), then each winner's receptive field.
void conv_prepost(const void *in, spk_dtype itype, int64_t b, int64_t t, int64_t cin, int64_t h, int64_t w,
                  int64_t cout, int64_t kh, int64_t kw, const void *out, int64_t oh, int64_t ow,
                  const int32_t *winners, const int32_t *counts, int64_t count, int64_t sy, int64_t sx, Pad4 p,
                  uint16_t *fst, uint16_t *pre, uint16_t *post, cudaStream_t s)
{
    auto prep = [&](auto z) {
        using T = decltype(z);
        const int64_t x = cin * h * w;
        if (sizeof(T) == 1 && x % 8 == 0 && reinterpret_cast<uintptr_t>(in) % 8 == 0 &&
            reinterpret_cast<uintptr_t>(fst) % 16 == 0 && t < 256)
            first_spike_map_u8x8_sum_kernel<<<grid_for(b * x / 8, 256, 16), 256, 0, s>>>(
                (const uint2 *)in, reinterpret_cast<uint4 *>(fst), b, int(t), x / 8);
        else if (sizeof(T) == 1 && x % 4 == 0 && reinterpret_cast<uintptr_t>(in) % 4 == 0 && t < 256)
            first_spike_map_u8x4_sum_kernel<<<grid_for(b * x / 4, 256, 16), 256, 0, s>>>(
                (const uint32_t *)in, reinterpret_cast<uint2 *>(fst), b, int(t), x / 4);
        else if (sizeof(T) == 1 && x % 4 == 0 && reinterpret_cast<uintptr_t>(in) % 4 == 0)
            first_spike_map_u8x4_kernel<<<grid_for(b * x / 4, 256, 16), 256, 0, s>>>(
                (const uint32_t *)in, reinterpret_cast<uint2 *>(fst), b, int(t), x / 4);
        else
            first_spike_map_kernel<T><<<grid_for(b * x, 256, 16), 256, 0, s>>>((const T *)in, fst, b, int(t), x);
        SPK_LAUNCHED();
        conv_prepost_map_kernel<T><<<unsigned(b * count), 128, 0, s>>>(
            fst, (const T *)out, int(t), int(cin), int(h), int(w), int(cout), int(oh), int(ow), int(kh), int(kw),
            int(sy), int(sx), int(p.top), int(p.left), winners, counts, int(count), pre, post);
        SPK_LAUNCHED();
    };
    if (itype == SPK_U8)
        prep(uint8_t());
    else if (itype == SPK_F32)
        prep(float());
    else
        throw Error(SPK_ERR_UNSUPPORTED, "STDP spikes must be U8 or F32");
}

// Bytes of the (pre, post) first-spike scratch of conv STDP.
size_t convstdp_prepost_bytes(int64_t b, int64_t count, int64_t cin, int64_t kh, int64_t kw)
{
    return align256(size_t(b * count * cin * kh * kw) * 2) + align256(size_t(b * count) * 2);
}

// Conv STDP with the (pre, post) scratch at a given device address; used by
// the entry point that draws its scratch from a static device array.
void convstdp_into(const void *in, spk_dtype itype, int64_t b, int64_t t, int64_t cin, int64_t h, int64_t w,
                   float *kernel, int64_t cout, int64_t kh, int64_t kw, const void *out, int64_t oh, int64_t ow,
                   const double *configs, int64_t nconf, const int32_t *winners, const int32_t *counts, int64_t count,
                   int64_t sy, int64_t sx, const int64_t *pad4, void *scratch, cudaStream_t s)
{
    Pad4 p = pad_of(pad4);
    Configs cfg = make_configs(configs, nconf);
    SPK_REQUIRE(b >= 0 && t >= 1 && t < 65535 && cin >= 1 && cout >= 1 && kh >= 1 && kw >= 1, "invalid dims");
    SPK_REQUIRE(count >= 1 && b * count < (int64_t(1) << 31), "winner count must be positive (at most 2^31 - 1 records)");
    SPK_REQUIRE(oh == (h + p.top + p.bottom - kh) / sy + 1 && ow == (w + p.left + p.right - kw) / sx + 1,
                "tensor shapes are not compatible");
    if (b == 0) return;
    const int64_t k = cin * kh * kw;
    uint16_t *pre = reinterpret_cast<uint16_t *>(scratch);
    uint16_t *post = reinterpret_cast<uint16_t *>(static_cast<char *>(scratch) + align256(size_t(b * count * k) * 2));
    if (itype == SPK_U8)
        conv_prepost_kernel<uint8_t><<<unsigned(b * count), 128, 0, s>>>(
            (const uint8_t *)in, (const uint8_t *)out, int(t), int(cin), int(h), int(w), int(cout), int(oh), int(ow),
            int(kh), int(kw), int(sy), int(sx), int(p.top), int(p.left), winners, counts, int(count), pre, post);
    else if (itype == SPK_F32)
        conv_prepost_kernel<float><<<unsigned(b * count), 128, 0, s>>>(
            (const float *)in, (const float *)out, int(t), int(cin), int(h), int(w), int(cout), int(oh), int(ow),
            int(kh), int(kw), int(sy), int(sx), int(p.top), int(p.left), winners, counts, int(count), pre, post);
    else
        throw Error(SPK_ERR_UNSUPPORTED, "STDP spikes must be U8 or F32");
    SPK_LAUNCHED();
    dim3 grid(unsigned(cout), unsigned(ceil_div(k, kScanThreads)));
    stdp_scan_kernel<false, false><<<grid, kScanThreads, 0, s>>>(kernel, k, b, int(count), 2, winners, counts, pre,
                                                                count * k, k, post, cfg, NetScan{});
    SPK_LAUNCHED();
}
}  // namespace spk

using namespace spk;

extern "C" {

size_t spk_rank_convstdp_workspace(int64_t b, int64_t count, int64_t cin, int64_t h, int64_t w, int64_t kh,
                                   int64_t kw)
{
    return spk::convstdp_prepost_bytes(b, count, cin, kh, kw) + align256(size_t(b * cin * h * w) * 2);
}

spk_status spk_rank_convstdp(const void *in, spk_dtype itype, int64_t b, int64_t t, int64_t cin, int64_t h, int64_t w,
                             float *kernel, int64_t cout, int64_t kh, int64_t kw, const void *out, int64_t oh,
                             int64_t ow, const double *configs, int64_t nconf, const int32_t *winners,
                             const int32_t *counts, int64_t count, int64_t sy, int64_t sx, const int64_t *pad4,
                             void *ws, size_t ws_bytes, spk_stream stream)
{
    return guarded([&] {
        Pad4 p = pad_of(pad4);
        Configs cfg = make_configs(configs, nconf);
        SPK_REQUIRE(b >= 0 && t >= 1 && t < 65535 && cin >= 1 && cout >= 1 && kh >= 1 && kw >= 1, "invalid dims");
        SPK_REQUIRE(count >= 1 && b * count < (int64_t(1) << 31), "winner count must be positive (at most 2^31 - 1 records)");
        SPK_REQUIRE(oh == (h + p.top + p.bottom - kh) / sy + 1 && ow == (w + p.left + p.right - kw) / sx + 1,
                    "tensor shapes are not compatible");
        if (b == 0) return;
        const int64_t k = cin * kh * kw;
        const size_t need = spk_rank_convstdp_workspace(b, count, cin, h, w, kh, kw);
        SPK_REQUIRE(ws != nullptr && ws_bytes >= need, "workspace is too small");
        uint16_t *pre = reinterpret_cast<uint16_t *>(ws);
        uint16_t *post = reinterpret_cast<uint16_t *>(static_cast<char *>(ws) + align256(size_t(b * count * k) * 2));
        cudaStream_t s = stream_of(stream);
        uint16_t *fst = reinterpret_cast<uint16_t *>(static_cast<char *>(ws) +
                                                     convstdp_prepost_bytes(b, count, cin, kh, kw));
        conv_prepost(in, itype, b, t, cin, h, w, cout, kh, kw, out, oh, ow, winners, counts, count, sy, sx, p, fst,
                     pre, post, s);
        dim3 grid(unsigned(cout), unsigned(ceil_div(k, kScanThreads)));
        stdp_scan_kernel<false, false><<<grid, kScanThreads, 0, s>>>(kernel, k, b, int(count), 2, winners, counts, pre,
                                                                    count * k, k, post, cfg, NetScan{});
        SPK_LAUNCHED();
    });
}

size_t spk_rank_convstdp_prepost_workspace(int64_t b, int64_t cin, int64_t h, int64_t w)
{
    return align256(size_t(b * cin * h * w) * 2);
}

spk_status spk_rank_convstdp_prepost(const void *in, spk_dtype itype, int64_t b, int64_t t, int64_t cin, int64_t h,
                                     int64_t w, int64_t cout, int64_t kh, int64_t kw, const void *out, int64_t oh,
                                     int64_t ow, const int32_t *winners, const int32_t *counts, int64_t count,
                                     int64_t sy, int64_t sx, const int64_t *pad4_host, uint16_t *pre, uint16_t *post,
                                     void *ws, size_t ws_bytes, spk_stream stream)
{
    return guarded([&] {
        Pad4 p = pad_of(pad4_host);
        SPK_REQUIRE(b >= 0 && t >= 1 && t < 65535 && cin >= 1 && cout >= 1 && kh >= 1 && kw >= 1, "invalid dims");
        SPK_REQUIRE(count >= 1, "winner count must be positive");
        SPK_REQUIRE(oh == (h + p.top + p.bottom - kh) / sy + 1 && ow == (w + p.left + p.right - kw) / sx + 1,
                    "tensor shapes are not compatible");
        SPK_REQUIRE(pre != nullptr && post != nullptr, "null output");
        if (b == 0) return;
        SPK_REQUIRE(ws != nullptr && ws_bytes >= spk_rank_convstdp_prepost_workspace(b, cin, h, w),
                    "workspace is too small");
        conv_prepost(in, itype, b, t, cin, h, w, cout, kh, kw, out, oh, ow, winners, counts, count, sy, sx, p,
                     static_cast<uint16_t *>(ws), pre, post, stream_of(stream));
    });
}

spk_status spk_stdp_scan(float *kernel, int64_t nmaps, int64_t k, int64_t b, int64_t count, int64_t field,
                         const int32_t *winners, const int32_t *counts, const uint16_t *pre, int64_t pre_sample_stride,
                         int64_t pre_slot_stride, const uint16_t *post, const double *configs_host, int64_t nconf,
                         int f32_rule, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(nmaps >= 1 && k >= 1 && b >= 0 && count >= 1, "invalid dims");
        SPK_REQUIRE(field == 2 || field == 4, "the map field is 2 (z, conv) or 4 (x, fc)");
        SPK_REQUIRE(kernel && winners && counts && pre && post, "null pointer");
        if (b == 0) return;
        launch_stdp_scan(kernel, k, nmaps, b, count, int(field), winners, counts, pre, pre_sample_stride,
                         pre_slot_stride, post, configs_host, nconf, f32_rule != 0, stream_of(stream));
    });
}

spk_status spk_stdp_scan_nets(float *kernels, int64_t nnets, int64_t nmaps, int64_t k, int64_t b, int64_t count,
                              int64_t field, const int32_t *winners, const int32_t *counts, const uint16_t *pre,
                              int64_t pre_sample_stride, int64_t pre_slot_stride, const uint16_t *post,
                              const int64_t *net_offsets, const int32_t *order, const double *net_configs,
                              int64_t nconf, int f32_rule, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(nmaps >= 1 && nmaps <= 65535 && k >= 1 && b >= 0 && count >= 1, "invalid dims");
        SPK_REQUIRE(field == 2 || field == 4, "the map field is 2 (z, conv) or 4 (x, fc)");
        SPK_REQUIRE(kernels && winners && counts && pre && post && net_offsets && net_configs, "null pointer");
        if (b == 0) return;
        launch_stdp_scan_nets(kernels, nnets, k, nmaps, b, count, int(field), winners, counts, pre, pre_sample_stride,
                              pre_slot_stride, post, net_offsets, order, net_configs, nconf, f32_rule != 0,
                              stream_of(stream));
    });
}

size_t spk_rank_fcstdp_workspace(int64_t b, int64_t, int64_t ni)
{
    // pre [B, I] + post [B, 64] (count is bounded by 64 on this path)
    return align256(size_t(b * ni) * 2) + align256(size_t(b) * 64 * 2);
}

spk_status spk_rank_fcstdp(const void *in, spk_dtype itype, int64_t b, int64_t t, int64_t ni, float *kernel,
                           int64_t no, const void *out, const double *configs, int64_t nconf, const int32_t *winners,
                           const int32_t *counts, int64_t count, void *ws, size_t ws_bytes, spk_stream stream)
{
    return guarded([&] {
        Configs cfg = make_configs(configs, nconf);
        SPK_REQUIRE(b >= 0 && t >= 1 && t < 65535 && ni >= 1 && no >= 1, "invalid dims");
        SPK_REQUIRE(count >= 1 && count <= 64, "winner count must be in [1, 64]");
        if (b == 0) return;
        SPK_REQUIRE(ws != nullptr && ws_bytes >= spk_rank_fcstdp_workspace(b, t, ni), "workspace is too small");
        uint16_t *pre = reinterpret_cast<uint16_t *>(ws);
        uint16_t *post = reinterpret_cast<uint16_t *>(static_cast<char *>(ws) + align256(size_t(b * ni) * 2));
        cudaStream_t s = stream_of(stream);
        if (itype == SPK_U8)
            fc_prepost_kernel<uint8_t><<<grid_for(b * ni, 256), 256, 0, s>>>(
                (const uint8_t *)in, (const uint8_t *)out, b, int(t), int(ni), int(no), winners, counts, int(count), pre,
                post);
        else if (itype == SPK_F32)
            fc_prepost_kernel<float><<<grid_for(b * ni, 256), 256, 0, s>>>((const float *)in, (const float *)out, b,
                                                                          int(t), int(ni), int(no), winners, counts,
                                                                          int(count), pre, post);
        else
            throw Error(SPK_ERR_UNSUPPORTED, "STDP spikes must be U8 or F32");
        SPK_LAUNCHED();
        dim3 grid(unsigned(no), unsigned(ceil_div(ni, kScanThreads)));
        stdp_scan_kernel<false, false><<<grid, kScanThreads, 0, s>>>(kernel, ni, b, int(count), 4, winners, counts, pre,
                                                                    ni, 0, post, cfg, NetScan{});
        SPK_LAUNCHED();
    });
}

}  // extern "C"
