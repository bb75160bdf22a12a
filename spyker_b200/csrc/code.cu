// Rank-order and latency coding of intensities into cumulative spikes.
//
// src/spyker/cpu/code.cpp:42-132.  Per image (row of X values):
//   sort=1: rank r of every value in descending order (ties in index order),
//           cnt = #values strictly above the row minimum,
//           scale = F32(T + 1e-5) / cnt, time = U16(r * scale);
//   sort=0: time = U16(end - scale * (x - min)), end = T + 1e-5,
//           scale = end / (max - min).
//   out[t, j] = (time_j <= t), cumulative u8 spikes [B, T, X].
//
// The reference sorts with an unstable std::sort, so elements with equal
// values straddling a time-bin boundary may be ordered differently there;
// this implementation uses the stable order (value desc, index asc).
//
// One CTA per image: the (value, index) keys are sorted by a bitonic network
// in shared memory (X <= 16384), the times are scattered to shared memory and
// the T output rows are written as 16-byte vectors.
#include "common.cuh"

namespace spk
{
namespace
{
constexpr int kCodeThreads = 1024;
constexpr int64_t kMaxSortX = 16384;

// Order-preserving map of a value to u32 (ascending), -0.0 folded into +0.0
// so that zeros of either sign are ties, as under the reference comparator.
__device__ __forceinline__ uint32_t order_key(float v)
{
    if (v == 0.0f) v = 0.0f;
    uint32_t u = __float_as_uint(v);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ uint32_t order_key(uint8_t v) { return uint32_t(v); }

template <typename O>
__device__ __forceinline__ void write_rows(O *__restrict__ out, const uint16_t *__restrict__ tm, int64_t x, int t)
{
    // out: [T, X] of this image.  Vector path when rows are 16-byte aligned.
    const bool vec = (sizeof(O) == 1) && (x % 16 == 0) && ((reinterpret_cast<uintptr_t>(out) & 15) == 0);
    if (vec)
    {
        const int64_t nv = x / 16;
        for (int64_t v = threadIdx.x; v < nv; v += blockDim.x)
        {
            uint16_t mine[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) mine[q] = tm[v * 16 + q];
            for (int s = 0; s < t; ++s)
            {
                uint32_t w[4];
#pragma unroll
                for (int q = 0; q < 4; ++q)
                {
                    uint32_t a = 0;
#pragma unroll
                    for (int e = 0; e < 4; ++e) a |= uint32_t(mine[q * 4 + e] <= uint16_t(s)) << (8 * e);
                    w[q] = a;
                }
                reinterpret_cast<uint4 *>(out + int64_t(s) * x)[v] = make_uint4(w[0], w[1], w[2], w[3]);
            }
        }
    }
    else
    {
        for (int64_t j = threadIdx.x; j < x; j += blockDim.x)
        {
            uint16_t m = tm[j];
            for (int s = 0; s < t; ++s) out[int64_t(s) * x + j] = O(m <= uint16_t(s));
        }
    }
}

// TIMES: write the u16 times [B, X] instead of the spike rows (event lists
// are built from them).
template <typename I, typename O, bool TIMES = false>
__global__ void __launch_bounds__(kCodeThreads) rank_sorted_kernel(const I *__restrict__ in, O *__restrict__ out,
                                                                    int64_t x, int t, int npow2)
{
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t *keys = reinterpret_cast<uint64_t *>(smem);
    uint16_t *tm = reinterpret_cast<uint16_t *>(keys + npow2);
    __shared__ uint32_t s_cnt;

    const I *row = in + int64_t(blockIdx.x) * x;
    for (int i = threadIdx.x; i < npow2; i += blockDim.x)
    {
        uint64_t k = ~uint64_t(0);
        if (i < x) k = (uint64_t(~order_key(row[i])) << 32) | uint32_t(i);
        keys[i] = k;
    }
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();

    // Bitonic sort ascending.
    for (int size = 2; size <= npow2; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1)
        {
            for (int i = threadIdx.x; i < npow2 / 2; i += blockDim.x)
            {
                int lo = 2 * i - (i & (stride - 1));
                int hi = lo + stride;
                bool up = (lo & size) == 0;
                uint64_t a = keys[lo], b = keys[hi];
                if ((a > b) == up) keys[lo] = b, keys[hi] = a;
            }
            __syncthreads();
        }

    // cnt = number of values strictly greater than the row minimum.
    const I vmin = row[uint32_t(keys[x - 1])];
    uint32_t local = 0;
    for (int64_t i = threadIdx.x; i < x; i += blockDim.x) local += (row[i] > vmin);
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&s_cnt, local);
    __syncthreads();

    const float scale = (float(t) + 1e-5f) / float(s_cnt);
    for (int64_t i = threadIdx.x; i < x; i += blockDim.x)
    {
        uint32_t j = uint32_t(keys[i]);
        tm[j] = f2u16(float(i) * scale);
    }
    __syncthreads();
    if constexpr (TIMES)
    {
        for (int64_t j = threadIdx.x; j < x; j += blockDim.x) out[int64_t(blockIdx.x) * x + j] = O(tm[j]);
    }
    else
        write_rows<O>(out + int64_t(blockIdx.x) * t * x, tm, x, t);
}

// Reduction type of the latency code: the value itself for floats, int for
// u8 (the reference subtracts promoted integers).
template <typename I>
struct Acc
{
    using T = I;
};
template <>
struct Acc<uint8_t>
{
    using T = int;
};

template <typename I, typename O, bool TIMES = false>
__global__ void __launch_bounds__(kCodeThreads) latency_kernel(const I *__restrict__ in, O *__restrict__ out, int64_t x,
                                                                int t)
{
    using A = typename Acc<I>::T;
    __shared__ A s_min[32], s_max[32];
    const I *row = in + int64_t(blockIdx.x) * x;
    A mn = A(row[0]), mx = A(row[0]);
    for (int64_t i = threadIdx.x; i < x; i += blockDim.x)
    {
        A v = A(row[i]);
        mn = (v < mn) ? v : mn;
        mx = (mx < v) ? v : mx;
    }
    for (int o = 16; o > 0; o >>= 1)
    {
        A a = __shfl_xor_sync(0xffffffffu, mn, o), b = __shfl_xor_sync(0xffffffffu, mx, o);
        mn = (a < mn) ? a : mn;
        mx = (mx < b) ? b : mx;
    }
    if ((threadIdx.x & 31) == 0) s_min[threadIdx.x >> 5] = mn, s_max[threadIdx.x >> 5] = mx;
    __syncthreads();
    mn = s_min[0], mx = s_max[0];
    for (int w = 1; w < int(blockDim.x >> 5); ++w)
    {
        mn = (s_min[w] < mn) ? s_min[w] : mn;
        mx = (mx < s_max[w]) ? s_max[w] : mx;
    }
    const float end = float(t) + 1e-5f;
    const float scale = __fdiv_rn(end, float(mx - mn));
    O *orow = out + int64_t(blockIdx.x) * t * x;
    for (int64_t j = threadIdx.x; j < x; j += blockDim.x)
    {
        // end - scale * d, fused as the reference's -O3 FMA build computes it.
        uint16_t m = f2u16(__fmaf_rn(-scale, float(A(row[j]) - mn), end));
        if constexpr (TIMES)
            out[int64_t(blockIdx.x) * x + j] = O(m);
        else
            for (int s = 0; s < t; ++s) orow[int64_t(s) * x + j] = O(m <= uint16_t(s));
    }
}
}  // namespace

// First-spike times [B, X] u16 of the rank-order (sort) or latency code.
void rank_times(const void *in, spk_dtype itype, uint16_t *times, int64_t b, int64_t t, int64_t x, int sort,
                cudaStream_t s)
{
    SPK_REQUIRE(itype == SPK_F32 || itype == SPK_U8, "coding supports F32/U8 input");
    if (b == 0) return;
    if (sort)
    {
        if (x > kMaxSortX)
            throw Error(SPK_ERR_UNSUPPORTED, "sorted rank coding supports at most 16384 values per image");
        int npow2 = 2;
        while (npow2 < x) npow2 <<= 1;
        const size_t smem = size_t(npow2) * 8 + size_t(x) * 2 + 16;
        auto go = [&](auto k, const auto *p) {
            SPK_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
            k<<<unsigned(b), kCodeThreads, smem, s>>>(p, times, x, int(t), npow2);
        };
        if (itype == SPK_F32)
            go(rank_sorted_kernel<float, uint16_t, true>, (const float *)in);
        else
            go(rank_sorted_kernel<uint8_t, uint16_t, true>, (const uint8_t *)in);
    }
    else if (itype == SPK_F32)
        latency_kernel<float, uint16_t, true><<<unsigned(b), kCodeThreads, 0, s>>>((const float *)in, times, x, int(t));
    else
        latency_kernel<uint8_t, uint16_t, true><<<unsigned(b), kCodeThreads, 0, s>>>((const uint8_t *)in, times, x,
                                                                                    int(t));
    SPK_LAUNCHED();
}
}  // namespace spk

using namespace spk;

extern "C" {

size_t spk_rank_code_workspace(int64_t, int64_t, int) { return 0; }

spk_status spk_rank_code(const void *in, spk_dtype itype, void *out, spk_dtype otype, int64_t b, int64_t t, int64_t x,
                         int sort, void *, size_t, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(t > 0, "input time can't be less than 1");
        SPK_REQUIRE(b >= 0 && x >= 1, "invalid dims");
        SPK_REQUIRE(t <= 65535, "time is limited to 65535 steps");
        if (b == 0) return;
        if (sort)
        {
            if (x > kMaxSortX)
                throw Error(SPK_ERR_UNSUPPORTED, "sorted rank coding supports at most 16384 values per image");
            int npow2 = 2;
            while (npow2 < x) npow2 <<= 1;
            size_t smem = size_t(npow2) * 8 + size_t(x) * 2 + 16;
            SPK_REQUIRE(otype == SPK_U8 || otype == SPK_F32, "output type must be U8 or F32");
            if (itype == SPK_F32 && otype == SPK_U8)
            {
                auto k = rank_sorted_kernel<float, uint8_t>;
                SPK_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
                k<<<unsigned(b), kCodeThreads, smem, stream_of(stream)>>>((const float *)in, (uint8_t *)out, x, int(t),
                                                                          npow2);
            }
            else if (itype == SPK_F32 && otype == SPK_F32)
            {
                auto k = rank_sorted_kernel<float, float>;
                SPK_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
                k<<<unsigned(b), kCodeThreads, smem, stream_of(stream)>>>((const float *)in, (float *)out, x, int(t),
                                                                          npow2);
            }
            else if (itype == SPK_U8 && otype == SPK_U8)
            {
                auto k = rank_sorted_kernel<uint8_t, uint8_t>;
                SPK_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
                k<<<unsigned(b), kCodeThreads, smem, stream_of(stream)>>>((const uint8_t *)in, (uint8_t *)out, x,
                                                                          int(t), npow2);
            }
            else
                throw Error(SPK_ERR_UNSUPPORTED, "sorted rank coding supports F32/U8 input");
            SPK_LAUNCHED();
        }
        else
        {
            SPK_REQUIRE(otype == SPK_U8 || otype == SPK_F32, "output type must be U8 or F32");
            if (itype == SPK_F32 && otype == SPK_U8)
                latency_kernel<float, uint8_t><<<unsigned(b), kCodeThreads, 0, stream_of(stream)>>>(
                    (const float *)in, (uint8_t *)out, x, int(t));
            else if (itype == SPK_F32 && otype == SPK_F32)
                latency_kernel<float, float><<<unsigned(b), kCodeThreads, 0, stream_of(stream)>>>(
                    (const float *)in, (float *)out, x, int(t));
            else if (itype == SPK_U8 && otype == SPK_U8)
                latency_kernel<uint8_t, uint8_t><<<unsigned(b), kCodeThreads, 0, stream_of(stream)>>>(
                    (const uint8_t *)in, (uint8_t *)out, x, int(t));
            else
                throw Error(SPK_ERR_UNSUPPORTED, "latency coding supports F32/U8 input");
            SPK_LAUNCHED();
        }
    });
}

}  // extern "C"
