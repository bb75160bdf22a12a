// Winner-take-all selection (convwta / fcwta), GPU resident: one CTA per
// sample computes the keys, then runs `count` rounds of block-wide argmax and
// suppression without any host round trip.
//
// src/spyker/cpu/wta.cpp:40-152.  For floating-point input, per sample:
//   min, max over all [T, X] values; diff = (max - min) * 2;
//   key(j) = (T - 1 - t0) + (x[t0, j] - min) / diff, t0 = first t with
//   x[t, j] > threshold, else -FLT_MAX (all in F32).
// For integer input: key(j) = T - t0 with t0 the first non-zero step, else 0.
// Each round takes the first index of the maximum key (std::max_element),
// stops on the sentinel, records the winner and suppresses the
// (2ry+1) x (2rx+1) box over all channels plus (convwta) the whole channel.
#include "common.cuh"

namespace spk
{
namespace
{
constexpr int kWtaThreads = 1024;
constexpr int64_t kWtaSmemKeys = 40 * 1024;  // keys kept in shared memory up to 160 KB

struct BestPair
{
    float v;
    int64_t i;
};

__device__ __forceinline__ BestPair better(BestPair a, BestPair b)
{
    if (b.v > a.v) return b;
    if (a.v > b.v) return a;
    return (b.i < a.i) ? b : a;
}

// Block-wide first-index argmax with std::max_element semantics.
__device__ int64_t block_argmax(const float *keys, int64_t n, BestPair *s_pairs)
{
    BestPair best{-INFINITY, INT64_MAX};
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x)
    {
        float v = keys[i];
        if (v != v) continue;  // NaN never replaces the running maximum
        if (best.i == INT64_MAX || best.v < v) best = {v, i};
    }
    for (int o = 16; o > 0; o >>= 1)
    {
        BestPair other{__shfl_xor_sync(0xffffffffu, best.v, o), __shfl_xor_sync(0xffffffffu, best.i, o)};
        best = better(best, other);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) s_pairs[warp] = best;
    __syncthreads();
    if (warp == 0)
    {
        int nw = blockDim.x >> 5;
        best = lane < nw ? s_pairs[lane] : BestPair{-INFINITY, INT64_MAX};
        for (int o = 16; o > 0; o >>= 1)
        {
            BestPair other{__shfl_xor_sync(0xffffffffu, best.v, o), __shfl_xor_sync(0xffffffffu, best.i, o)};
            best = better(best, other);
        }
        if (lane == 0) s_pairs[32] = best;
    }
    __syncthreads();
    int64_t idx = s_pairs[32].i;
    float k0 = keys[0];
    if (k0 != k0 || idx == INT64_MAX) idx = 0;
    __syncthreads();
    return idx;
}

template <typename T>
__device__ __forceinline__ void minmax_update(T v, T &mn, T &mx)
{
    mn = (v < mn) ? v : mn;  // std::min(mn, v)
    mx = (mx < v) ? v : mx;  // std::max(mx, v)
}

template <typename T, bool kFloat>
__global__ void __launch_bounds__(kWtaThreads)
    wta_kernel(const T *__restrict__ in, int t, int64_t x, int c, int h, int w, int ry, int rx, int count, bool whole,
               T thr, int32_t *__restrict__ winners, int32_t *__restrict__ counts, float *__restrict__ gkeys)
{
    extern __shared__ __align__(16) float smem_keys[];
    __shared__ BestPair s_pairs[33];
    __shared__ T s_mn[32], s_mx[32];
    const int64_t b = blockIdx.x;
    float *keys = gkeys ? gkeys + b * x : smem_keys;
    const T *sample = in + b * int64_t(t) * x;

    float low;
    if constexpr (kFloat)
    {
        T mn = sample[0], mx = sample[0];
        const int64_t tot = int64_t(t) * x;
        for (int64_t i = threadIdx.x; i < tot; i += blockDim.x) minmax_update(sample[i], mn, mx);
        for (int o = 16; o > 0; o >>= 1)
        {
            T a = __shfl_xor_sync(0xffffffffu, mn, o), bb = __shfl_xor_sync(0xffffffffu, mx, o);
            minmax_update(a, mn, mx);
            minmax_update(bb, mn, mx);
        }
        if ((threadIdx.x & 31) == 0) s_mn[threadIdx.x >> 5] = mn, s_mx[threadIdx.x >> 5] = mx;
        __syncthreads();
        mn = s_mn[0], mx = s_mx[0];
        for (int q = 1; q < int(blockDim.x >> 5); ++q) minmax_update(s_mn[q], mn, mx), minmax_update(s_mx[q], mn, mx);
        const float fmn = float(mn);
        const float diff = __fmul_rn(__fsub_rn(float(mx), fmn), 2.0f);
        for (int64_t j = threadIdx.x; j < x; j += blockDim.x)
        {
            float key = -FLT_MAX;
            for (int q = 0; q < t; ++q)
            {
                T v = sample[int64_t(q) * x + j];
                if (v > thr)
                {
                    key = __fadd_rn(float(t - q - 1), __fdiv_rn(__fsub_rn(float(v), fmn), diff));
                    break;
                }
            }
            keys[j] = key;
        }
        low = -FLT_MAX;
    }
    else
    {
        for (int64_t j = threadIdx.x; j < x; j += blockDim.x)
        {
            float key = 0.f;
            for (int q = 0; q < t; ++q)
                if (sample[int64_t(q) * x + j])
                {
                    key = float(t - q);
                    break;
                }
            keys[j] = key;
        }
        low = 0.f;
    }
    __syncthreads();

    const int64_t len = int64_t(h) * w;
    int found = 0;
    for (int r = 0; r < count; ++r)
    {
        int64_t idx = block_argmax(keys, x, s_pairs);
        float kv = keys[idx];
        bool stop = kFloat ? (fabsf(__fsub_rn(kv, -FLT_MAX)) < 1e-5f) : (fabsf(kv) < 1e-5f);
        if (stop) break;
        const int z = int(idx / len), y = int((idx % len) / w), xx = int((idx % len) % w);
        if (threadIdx.x == 0)
        {
            int32_t *e = winners + (b * count + r) * 5;
            e[0] = 0, e[1] = 0, e[2] = z, e[3] = y, e[4] = xx;
        }
        const int sj = max(0, y - ry), ej = min(h, y + ry + 1);
        const int sk = max(0, xx - rx), ek = min(w, xx + rx + 1);
        const int bw = ek - sk, bh = ej - sj;
        const int64_t box = int64_t(c) * bh * bw;
        for (int64_t i = threadIdx.x; i < box; i += blockDim.x)
        {
            int64_t ch = i / (int64_t(bh) * bw), rem = i % (int64_t(bh) * bw);
            keys[(ch * h + sj + rem / bw) * w + sk + rem % bw] = low;
        }
        if (whole)
            for (int64_t i = threadIdx.x; i < len; i += blockDim.x) keys[int64_t(z) * len + i] = low;
        __syncthreads();
        ++found;
    }
    if (threadIdx.x == 0) counts[b] = found;
}

template <typename T, bool kFloat>
void launch_wta(const void *in, int64_t b, int64_t t, int64_t c, int64_t h, int64_t w, int64_t ry, int64_t rx,
                int64_t count, bool whole, double thr, int32_t *winners, int32_t *counts, void *ws, size_t ws_bytes,
                cudaStream_t s)
{
    const int64_t x = c * h * w;
    float *gkeys = nullptr;
    size_t smem = 0;
    if (x <= kWtaSmemKeys)
        smem = size_t(x) * 4;
    else
    {
        SPK_REQUIRE(ws != nullptr && ws_bytes >= size_t(b) * size_t(x) * 4, "workspace is too small");
        gkeys = reinterpret_cast<float *>(ws);
    }
    auto k = wta_kernel<T, kFloat>;
    SPK_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    k<<<unsigned(b), kWtaThreads, smem, s>>>((const T *)in, int(t), x, int(c), int(h), int(w), int(ry), int(rx),
                                             int(count), whole, scalar_to<T>(thr), winners, counts, gkeys);
    SPK_LAUNCHED();
}

void wta_dispatch(const void *in, spk_dtype type, int64_t b, int64_t t, int64_t c, int64_t h, int64_t w, int64_t ry,
                  int64_t rx, int64_t count, bool whole, double thr, int32_t *winners, int32_t *counts, void *ws,
                  size_t ws_bytes, cudaStream_t s)
{
    SPK_REQUIRE(count > 0, "winners count can't be less than 1");
    SPK_REQUIRE(ry >= 0 && rx >= 0, "radius can't be less than 0");
    SPK_REQUIRE(b >= 0 && t >= 1 && c >= 1 && h >= 1 && w >= 1, "invalid dims");
    SPK_REQUIRE(winners != nullptr && counts != nullptr, "null winners buffer");
    if (b == 0) return;
    switch (type)
    {
    case SPK_F32: launch_wta<float, true>(in, b, t, c, h, w, ry, rx, count, whole, thr, winners, counts, ws, ws_bytes, s); break;
    case SPK_U8: launch_wta<uint8_t, false>(in, b, t, c, h, w, ry, rx, count, whole, thr, winners, counts, ws, ws_bytes, s); break;
    case SPK_I32: launch_wta<int32_t, false>(in, b, t, c, h, w, ry, rx, count, whole, thr, winners, counts, ws, ws_bytes, s); break;
    default: throw Error(SPK_ERR_UNSUPPORTED, "WTA supports U8/I32/F32/F64 input");
    }
}
}  // namespace
}  // namespace spk

using namespace spk;

extern "C" {

size_t spk_rank_convwta_workspace(int64_t b, int64_t, int64_t c, int64_t h, int64_t w)
{
    int64_t x = c * h * w;
    return x <= kWtaSmemKeys ? 0 : size_t(b) * size_t(x) * 4;
}

spk_status spk_rank_convwta(const void *in, spk_dtype type, int64_t b, int64_t t, int64_t c, int64_t h, int64_t w,
                            int64_t ry, int64_t rx, int64_t count, double threshold, int32_t *winners, int32_t *counts,
                            void *ws, size_t ws_bytes, spk_stream stream)
{
    return guarded([&] {
        wta_dispatch(in, type, b, t, c, h, w, ry, rx, count, true, threshold, winners, counts, ws, ws_bytes,
                     stream_of(stream));
    });
}

size_t spk_rank_fcwta_workspace(int64_t b, int64_t, int64_t n) { return n <= kWtaSmemKeys ? 0 : size_t(b) * size_t(n) * 4; }

spk_status spk_rank_fcwta(const void *in, spk_dtype type, int64_t b, int64_t t, int64_t n, int64_t radius,
                          int64_t count, double threshold, int32_t *winners, int32_t *counts, void *ws, size_t ws_bytes,
                          spk_stream stream)
{
    return guarded([&] {
        wta_dispatch(in, type, b, t, 1, 1, n, 0, radius, count, false, threshold, winners, counts, ws, ws_bytes,
                     stream_of(stream));
    });
}

}  // extern "C"
