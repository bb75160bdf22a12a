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
constexpr int kScanPerThread = 4;  // weights per thread held in registers
constexpr int kScanChunk = kScanThreads * kScanPerThread;
constexpr int kWinnerTile = 1024;
constexpr int kPreBatch = 14;  // winners whose pre rows are staged at once (28 KB)

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
    for (int i = threadIdx.x; i < k; i += blockDim.x)
    {
        const int c = i / (kh * kw), r = i % (kh * kw), ky = r / kw, kx = r % kw;
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

// Kernel B: CTA (map, chunk) walks winners in (sample, slot) order.  The map
// index of a winner is field `field` of its record (z for conv, x for fc).
// pre address: pre + s * ps + j * pw + element.
// F32_RULE: the event-list STDP of src/spyker/sparse/stdp.cpp:95-97, which
// rounds the soft-bound factor and the updated weight to F32 before the clamp.
template <bool F32_RULE>
__global__ void __launch_bounds__(kScanThreads)
    stdp_scan_kernel(float *__restrict__ kernel, int64_t k, int64_t b, int count, int field,
                     const int32_t *__restrict__ winners, const int32_t *__restrict__ counts,
                     const uint16_t *__restrict__ pre, int64_t ps, int64_t pw, const uint16_t *__restrict__ post,
                     Configs cfg)
{
    __shared__ int32_t s_rec[kWinnerTile][3];  // (config, sample, slot) of matching winners
    __shared__ uint16_t s_pre[kPreBatch][kScanChunk];
    __shared__ uint16_t s_post[kPreBatch];
    __shared__ int s_n;
    const int map = blockIdx.x;
    const int64_t base = int64_t(blockIdx.y) * kScanChunk;
    float wv[kScanPerThread];
    int64_t idx[kScanPerThread];
#pragma unroll
    for (int q = 0; q < kScanPerThread; ++q)
    {
        idx[q] = base + threadIdx.x + int64_t(q) * kScanThreads;
        wv[q] = idx[q] < k ? kernel[int64_t(map) * k + idx[q]] : 0.f;
    }
    const int64_t total = b * count;
    for (int64_t start = 0; start < total; start += kWinnerTile)
    {
        if (threadIdx.x == 0) s_n = 0;
        __syncthreads();
        // Compact the matching winners of this tile, preserving order.
        const int64_t end = min(total, start + kWinnerTile);
        for (int64_t r0 = start; r0 < end; r0 += blockDim.x)
        {
            int64_t r = r0 + threadIdx.x;
            bool m = false;
            int32_t c = 0;
            if (r < end)
            {
                int64_t s = r / count, j = r % count;
                if (j < counts[s])
                {
                    const int32_t *e = winners + r * 5;
                    c = e[0];
                    m = (e[field] == map) && c >= 0 && c < cfg.n;
                }
            }
            unsigned bal = __ballot_sync(0xffffffffu, m);
            // Order-preserving slot: block-wide prefix over warps.
            __shared__ int s_warp[kScanThreads / 32];
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            if (lane == 0) s_warp[warp] = __popc(bal);
            __syncthreads();
            int before = 0;
            for (int q = 0; q < warp; ++q) before += s_warp[q];
            int total_here = 0;
            for (int q = 0; q < kScanThreads / 32; ++q) total_here += s_warp[q];
            if (m)
            {
                int slot = s_n + before + __popc(bal & ((1u << lane) - 1));
                s_rec[slot][0] = c, s_rec[slot][1] = int32_t(r / count), s_rec[slot][2] = int32_t(r % count);
            }
            __syncthreads();
            if (threadIdx.x == 0) s_n += total_here;
            __syncthreads();
        }
        const int n = s_n;
        // Matching winners in batches: their pre rows (this CTA's chunk) are
        // staged in shared memory with coalesced loads, then applied in order.
        for (int q0 = 0; q0 < n; q0 += kPreBatch)
        {
            const int nb = min(kPreBatch, n - q0);
            const int len = (k - base < int64_t(kScanChunk)) ? int(k - base) : kScanChunk;
            for (int i = threadIdx.x; i < nb * len; i += blockDim.x)
            {
                const int q = i / len, e = i % len;
                const int64_t s = s_rec[q0 + q][1], j = s_rec[q0 + q][2];
                s_pre[q][e] = pre[s * ps + j * pw + base + e];
                if (e == 0) s_post[q] = post[s * count + j];
            }
            __syncthreads();
            for (int q = 0; q < nb; ++q)
            {
                const int c = s_rec[q0 + q][0];
                const uint16_t po = s_post[q];
                const double pos = cfg.pos[c], neg = cfg.neg[c], lo = cfg.lo[c], hi = cfg.hi[c];
                const bool stab = cfg.stab[c] != 0;
#pragma unroll
                for (int u = 0; u < kScanPerThread; ++u)
                    if (idx[u] < k)
                    {
                        const double old = double(wv[u]);
                        const double d = s_pre[q][idx[u] - base] <= po ? pos : neg;
                        if (F32_RULE)
                        {
                            const float m = __double2float_rn(stab ? (old - lo) * (hi - old) : 1.0);
                            double v = double(__double2float_rn(fma(d, double(m), old)));
                            v = (hi < v) ? hi : v;
                            v = (lo < v) ? v : lo;
                            wv[u] = __double2float_rn(v);
                        }
                        else
                        {
                            const double m = stab ? (old - lo) * (hi - old) : 1.0;
                            double v = fma(d, m, old);
                            v = (hi < v) ? hi : v;  // std::min(v, upper)
                            v = (lo < v) ? v : lo;  // std::max(lower, .)
                            wv[u] = __double2float_rn(v);
                        }
                    }
            }
            __syncthreads();
        }
        __syncthreads();  // everyone has read s_n before it is reset
    }
#pragma unroll
    for (int q = 0; q < kScanPerThread; ++q)
        if (idx[q] < k) kernel[int64_t(map) * k + idx[q]] = wv[q];
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
    dim3 grid(unsigned(nmaps), unsigned(ceil_div(k, kScanChunk)));
    if (f32_rule)
        stdp_scan_kernel<true><<<grid, kScanThreads, 0, s>>>(kernel, k, b, int(count), field, winners, counts, pre, ps,
                                                            pw, post, cfg);
    else
        stdp_scan_kernel<false><<<grid, kScanThreads, 0, s>>>(kernel, k, b, int(count), field, winners, counts, pre,
                                                             ps, pw, post, cfg);
    SPK_LAUNCHED();
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
    SPK_REQUIRE(count >= 1, "winner count must be positive");
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
    dim3 grid(unsigned(cout), unsigned(ceil_div(k, kScanChunk)));
    stdp_scan_kernel<false><<<grid, kScanThreads, 0, s>>>(kernel, k, b, int(count), 2, winners, counts, pre, count * k, k,
                                                   post, cfg);
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
        SPK_REQUIRE(count >= 1, "winner count must be positive");
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
        auto prep = [&](auto z) {
            using T = decltype(z);
            const int64_t x = cin * h * w;
            if (sizeof(T) == 1 && x % 4 == 0 && reinterpret_cast<uintptr_t>(in) % 4 == 0)
                first_spike_map_u8x4_kernel<<<grid_for(b * x / 4, 256, 16), 256, 0, s>>>(
                    (const uint32_t *)in, reinterpret_cast<uint2 *>(fst), b, int(t), x / 4);
            else
                first_spike_map_kernel<T><<<grid_for(b * x, 256, 16), 256, 0, s>>>((const T *)in, fst, b, int(t), x);
            SPK_LAUNCHED();
            conv_prepost_map_kernel<T><<<unsigned(b * count), 128, 0, s>>>(
                fst, (const T *)out, int(t), int(cin), int(h), int(w), int(cout), int(oh), int(ow), int(kh), int(kw),
                int(sy), int(sx), int(p.top), int(p.left), winners, counts, int(count), pre, post);
        };
        if (itype == SPK_U8)
            prep(uint8_t());
        else if (itype == SPK_F32)
            prep(float());
        else
            throw Error(SPK_ERR_UNSUPPORTED, "STDP spikes must be U8 or F32");
        SPK_LAUNCHED();
        dim3 grid(unsigned(cout), unsigned(ceil_div(k, kScanChunk)));
        stdp_scan_kernel<false><<<grid, kScanThreads, 0, s>>>(kernel, k, b, int(count), 2, winners, counts, pre, count * k, k,
                                                       post, cfg);
        SPK_LAUNCHED();
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
        dim3 grid(unsigned(no), unsigned(ceil_div(ni, kScanChunk)));
        stdp_scan_kernel<false><<<grid, kScanThreads, 0, s>>>(kernel, ni, b, int(count), 4, winners, counts, pre, ni, 0, post,
                                                       cfg);
        SPK_LAUNCHED();
    });
}

}  // extern "C"
