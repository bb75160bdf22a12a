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

    if (npow2 == 2 * kCodeThreads && blockDim.x == kCodeThreads)
    {
        // Two keys per thread (elements 2 tid, 2 tid + 1) in registers: a
        // stage of stride 1 is a swap inside the thread, strides 2..32 a
        // shuffle with thread tid ^ (stride / 2) of the same warp, and only
        // strides >= 64 go through shared memory (15 of the 66 stages).
        const int e0 = 2 * threadIdx.x;
        uint64_t k0 = keys[e0], k1 = keys[e0 + 1];
        for (int size = 2; size <= npow2; size <<= 1)
        {
            if (size > 64)
            {
                __syncthreads();
                keys[e0] = k0, keys[e0 + 1] = k1;
                __syncthreads();
                for (int stride = size >> 1; stride >= 64; stride >>= 1)
                {
                    const int i = threadIdx.x;
                    const int lo = 2 * i - (i & (stride - 1)), hi = lo + stride;
                    const bool up = (lo & size) == 0;
                    const uint64_t a = keys[lo], c = keys[hi];
                    if ((a > c) == up) keys[lo] = c, keys[hi] = a;
                    __syncthreads();
                }
                k0 = keys[e0], k1 = keys[e0 + 1];
            }
            const bool up = (e0 & size) == 0;
            for (int stride = (size >> 1) < 32 ? (size >> 1) : 32; stride >= 2; stride >>= 1)
            {
                const int lane_x = stride >> 1;
                const uint64_t p0 = __shfl_xor_sync(0xffffffffu, k0, lane_x);
                const uint64_t p1 = __shfl_xor_sync(0xffffffffu, k1, lane_x);
                const bool lower = (e0 & stride) == 0;  // this thread's elements are the lower of their pairs
                const bool keep_min = lower == up;
                k0 = keep_min ? (k0 < p0 ? k0 : p0) : (k0 > p0 ? k0 : p0);
                k1 = keep_min ? (k1 < p1 ? k1 : p1) : (k1 > p1 ? k1 : p1);
            }
            if ((k0 > k1) == up)
            {
                const uint64_t tmp = k0;
                k0 = k1, k1 = tmp;
            }
        }
        __syncthreads();
        keys[e0] = k0, keys[e0 + 1] = k1;
    }
    else
    // Bitonic sort ascending.  Pair i of a stage is handled by thread i mod
    // blockDim; for strides <= 32 the pairs of a warp's 32 consecutive i
    // stay inside one 64-key segment, so two such stages in a row need only
    // the warp to synchronise.
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
            const int next = stride > 1 ? stride >> 1 : size;  // stride of the next stage
            if (stride >= 64 || next >= 64)
                __syncthreads();
            else
                __syncwarp();
        }
    __syncthreads();

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

// Rows of 257 .. 2048 values with 256 threads.  Only the values above the
// row minimum are sorted: they are compacted in index order into shared
// memory (a value equal to the minimum at index i has rank cnt + the number
// of minimum values before it, known from the same prefix count), then
// sorted by a bitonic network on N = 512, 1024 or 2048 keys (the next power
// of two, at least 512) whose keys stay in registers: thread i holds
// positions ITEMS i .. ITEMS i + ITEMS - 1 (ITEMS = N / 256), a stage of
// stride < ITEMS is a compare-exchange inside the thread, strides up to
// 32 ITEMS / 2 a shuffle with the thread owning the partner positions, and
// only larger strides go through shared memory.  With many values tied at
// the minimum (zero filter responses) the sort is a fraction of the row.
constexpr int kRegThreads = 256, kRegMax = 8 * kRegThreads;

template <int ITEMS>
__device__ __forceinline__ void bitonic_block(uint64_t *keys)
{
    constexpr int N = kRegThreads * ITEMS;
    const int tid = threadIdx.x, e0 = ITEMS * tid;
    uint64_t k[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) k[j] = keys[e0 + j];
    for (int size = 2; size <= N; size <<= 1)
    {
        int stride = size >> 1;
        if (stride >= 32 * ITEMS)
        {
            __syncthreads();
#pragma unroll
            for (int j = 0; j < ITEMS; ++j) keys[e0 + j] = k[j];
            __syncthreads();
            for (; stride >= 32 * ITEMS; stride >>= 1)
            {
                for (int q = tid; q < N / 2; q += kRegThreads)
                {
                    const int lo = 2 * q - (q & (stride - 1)), hi = lo + stride;
                    const bool up = (lo & size) == 0;
                    const uint64_t a = keys[lo], c = keys[hi];
                    if ((a > c) == up) keys[lo] = c, keys[hi] = a;
                }
                __syncthreads();
            }
#pragma unroll
            for (int j = 0; j < ITEMS; ++j) k[j] = keys[e0 + j];
        }
        for (; stride >= ITEMS; stride >>= 1)
        {
            const int lx = stride / ITEMS;
            const bool keep_min = ((e0 & stride) == 0) == ((e0 & size) == 0);
#pragma unroll
            for (int j = 0; j < ITEMS; ++j)
            {
                const uint64_t pk = __shfl_xor_sync(0xffffffffu, k[j], lx);
                k[j] = keep_min ? (k[j] < pk ? k[j] : pk) : (k[j] > pk ? k[j] : pk);
            }
        }
        // strides below ITEMS: compile-time strides keep k[] in registers
#pragma unroll
        for (int st = ITEMS / 2; st >= 1; st >>= 1)
        {
            if (st > stride) continue;
#pragma unroll
            for (int j = 0; j < ITEMS; ++j)
                if ((j & st) == 0)
                {
                    const bool up = ((e0 + j) & size) == 0;
                    const uint64_t a = k[j], c = k[j + st];
                    if ((a > c) == up) k[j] = c, k[j + st] = a;
                }
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) keys[e0 + j] = k[j];
    __syncthreads();
}

template <typename I, typename O, bool TIMES>
__global__ void __launch_bounds__(kRegThreads) rank_compact_kernel(const I *__restrict__ in, O *__restrict__ out,
                                                                   int64_t x, int t)
{
    constexpr int IT = kRegMax / kRegThreads;  // values per thread on load
    __shared__ uint64_t keys[kRegMax];
    __shared__ __align__(16) uint16_t tm[kRegMax];
    __shared__ uint32_t s_warp[kRegThreads / 32], s_min, s_off[kRegThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, e0 = IT * tid;
    const I *row = in + int64_t(blockIdx.x) * x;
    uint32_t kv[IT];
    uint32_t mn = 0xFFFFFFFFu;
#pragma unroll
    for (int j = 0; j < IT; ++j)
    {
        kv[j] = e0 + j < x ? order_key(row[e0 + j]) : 0xFFFFFFFFu;
        mn = min(mn, kv[j]);
    }
    mn = __reduce_min_sync(0xffffffffu, mn);
    if (lane == 0) s_warp[warp] = mn;
    __syncthreads();
    if (tid == 0)
    {
        uint32_t m = s_warp[0];
        for (int w = 1; w < kRegThreads / 32; ++w) m = min(m, s_warp[w]);
        s_min = m;
    }
    __syncthreads();
    const uint32_t minkey = s_min;
    // keep: the values above the minimum, compacted in index order
    uint32_t mine = 0;
#pragma unroll
    for (int j = 0; j < IT; ++j) mine += (e0 + j < x && kv[j] != minkey) ? 1u : 0u;
    uint32_t incl = mine;
    for (int o = 1; o < 32; o <<= 1)
    {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (tid == 0)
    {
        uint32_t run = 0;
        for (int w = 0; w < kRegThreads / 32; ++w) s_off[w] = run, run += s_warp[w];
        s_min = run;  // cnt
    }
    __syncthreads();
    const int cnt = int(s_min);
    const float scale = (float(t) + 1e-5f) / float(cnt);
    int kp = int(s_off[warp] + incl - mine);  // keep values before this thread's first
#pragma unroll
    for (int j = 0; j < IT; ++j)
    {
        const int i = e0 + j;
        if (i < x)
        {
            if (kv[j] != minkey)
                keys[kp++] = (uint64_t(~kv[j]) << 32) | uint32_t(i);
            else
                tm[i] = f2u16(float(cnt + i - kp) * scale);  // rank among the ties at the minimum
        }
    }
    int n = 512;
    while (n < cnt) n <<= 1;
    for (int i = cnt + tid; i < n; i += kRegThreads) keys[i] = ~uint64_t(0);
    __syncthreads();
    if (n == 512)
        bitonic_block<2>(keys);
    else if (n == 1024)
        bitonic_block<4>(keys);
    else
        bitonic_block<8>(keys);
    for (int i = tid; i < cnt; i += kRegThreads) tm[uint32_t(keys[i])] = f2u16(float(i) * scale);
    __syncthreads();
    if constexpr (TIMES)
    {
        for (int64_t j = tid; j < x; j += kRegThreads) out[int64_t(blockIdx.x) * x + j] = O(tm[j]);
    }
    else
    {
        O *o = out + int64_t(blockIdx.x) * t * x;
        if (sizeof(O) == 1 && x % 16 == 0 && (reinterpret_cast<uintptr_t>(o) & 15) == 0)
        {
            // (row, 16-position vector) pairs over the block
            const int nv = int(x / 16);
            for (int q = tid; q < t * nv; q += kRegThreads)
            {
                const int srow = q / nv, v = q - srow * nv;
                const uint4 ta = *reinterpret_cast<const uint4 *>(tm + 16 * v);
                const uint4 tb = *reinterpret_cast<const uint4 *>(tm + 16 * v + 8);
                const uint32_t hw[8] = {ta.x, ta.y, ta.z, ta.w, tb.x, tb.y, tb.z, tb.w};
                uint32_t w[4];
#pragma unroll
                for (int r = 0; r < 4; ++r)
                {
                    const uint32_t a = hw[2 * r], b = hw[2 * r + 1];
                    w[r] = uint32_t((a & 0xFFFFu) <= uint32_t(srow)) | (uint32_t((a >> 16) <= uint32_t(srow)) << 8) |
                           (uint32_t((b & 0xFFFFu) <= uint32_t(srow)) << 16) |
                           (uint32_t((b >> 16) <= uint32_t(srow)) << 24);
                }
                reinterpret_cast<uint4 *>(o + int64_t(srow) * x)[v] = make_uint4(w[0], w[1], w[2], w[3]);
            }
        }
        else
            for (int64_t j = tid; j < x; j += kRegThreads)
            {
                const uint16_t m = tm[j];
                for (int srow = 0; srow < t; ++srow) o[int64_t(srow) * x + j] = O(m <= uint16_t(srow));
            }
    }
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
// ---- images larger than one CTA's shared memory (X > 16384) ---------------
// The same (value desc, index asc) order from a device-wide sort per image:
// CTAs sort 8192-key chunks in shared memory, then merge-path rounds double
// the sorted runs until each image is one run; times and rows follow.
constexpr int kChunk = 8192, kMergeItems = 8;

inline int64_t padded_x(int64_t x) { return ceil_div(x, kChunk) * kChunk; }

template <typename I>
__global__ void __launch_bounds__(kCodeThreads) chunk_sort_kernel(const I *__restrict__ in, uint64_t *__restrict__ keys,
                                                                   int64_t x, int64_t xp)
{
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t *sk = reinterpret_cast<uint64_t *>(smem);
    const int64_t img = blockIdx.y, base = int64_t(blockIdx.x) * kChunk;
    const I *row = in + img * x;
    for (int i = threadIdx.x; i < kChunk; i += blockDim.x)
    {
        const int64_t j = base + i;
        sk[i] = (j < x) ? ((uint64_t(~order_key(row[j])) << 32) | uint32_t(j)) : ~uint64_t(0);
    }
    __syncthreads();
    for (int size = 2; size <= kChunk; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1)
        {
            for (int i = threadIdx.x; i < kChunk / 2; i += blockDim.x)
            {
                const int lo = 2 * i - (i & (stride - 1)), hi = lo + stride;
                const bool up = (lo & size) == 0;
                const uint64_t a = sk[lo], b = sk[hi];
                if ((a > b) == up) sk[lo] = b, sk[hi] = a;
            }
            __syncthreads();
        }
    uint64_t *out = keys + img * xp + base;
    for (int i = threadIdx.x; i < kChunk; i += blockDim.x) out[i] = sk[i];
}

// One merge round: runs of length L pairwise into runs of 2L; each thread
// finds its diagonal on the merge path and writes kMergeItems outputs.
__global__ void merge_round_kernel(const uint64_t *__restrict__ src, uint64_t *__restrict__ dst, int64_t b, int64_t xp,
                                   int64_t L)
{
    const int64_t total = b * xp / kMergeItems;
    for (int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < total; g += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t o = g * kMergeItems, img = o / xp, p = o - img * xp;
        const int64_t start = (p / (2 * L)) * (2 * L);
        const int64_t la = min(L, xp - start), lb = min(L, xp - start - la);
        const uint64_t *A = src + img * xp + start, *B = A + la;
        const int64_t d = p - start;
        int64_t lo = d > lb ? d - lb : 0, hi = d < la ? d : la;
        while (lo < hi)
        {
            const int64_t mid = (lo + hi) >> 1;
            if (A[mid] <= B[d - mid - 1])
                lo = mid + 1;
            else
                hi = mid;
        }
        int64_t i = lo, j = d - lo;
        uint64_t *out = dst + img * xp + p;
#pragma unroll
        for (int k = 0; k < kMergeItems; ++k)
        {
            const bool take_a = j >= lb || (i < la && A[i] <= B[j]);
            out[k] = take_a ? A[i++] : B[j++];
        }
    }
}

// Per image: cnt = values strictly above the minimum (the position of the
// first key carrying the minimum's value), then time of every sorted position.
__global__ void sorted_times_kernel(const uint64_t *__restrict__ keys, uint16_t *__restrict__ tm, int64_t b, int64_t x,
                                    int64_t xp, int t)
{
    const int64_t img = blockIdx.y;
    const uint64_t *S = keys + img * xp;
    const uint32_t vmin = uint32_t(S[x - 1] >> 32);
    int64_t lo = 0, hi = x - 1;
    while (lo < hi)
    {
        const int64_t mid = (lo + hi) >> 1;
        if (uint32_t(S[mid] >> 32) < vmin)
            lo = mid + 1;
        else
            hi = mid;
    }
    const float scale = (float(t) + 1e-5f) / float(lo);
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < x; i += int64_t(gridDim.x) * blockDim.x)
        tm[img * x + uint32_t(S[i])] = f2u16(float(i) * scale);
}

// out[img, s, j] = (tm[img, j] <= s), 16 positions per thread.
template <typename O>
__global__ void rows_from_times_kernel(const uint16_t *__restrict__ tm, O *__restrict__ out, int64_t b, int t,
                                       int64_t x)
{
    const int64_t groups = ceil_div(x, 16), total = b * groups;
    const bool vec = sizeof(O) == 1 && x % 16 == 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0;
    for (int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < total; g += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t img = g / groups, j0 = (g - img * groups) * 16;
        uint16_t m[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) m[q] = (j0 + q < x) ? tm[img * x + j0 + q] : uint16_t(0xffff);
        O *orow = out + img * t * x + j0;
        for (int s = 0; s < t; ++s)
        {
            if (vec)
            {
                uint32_t w[4];
#pragma unroll
                for (int q = 0; q < 4; ++q)
                {
                    uint32_t a = 0;
#pragma unroll
                    for (int e = 0; e < 4; ++e) a |= uint32_t(m[q * 4 + e] <= uint16_t(s)) << (8 * e);
                    w[q] = a;
                }
                *reinterpret_cast<uint4 *>(orow + int64_t(s) * x) = make_uint4(w[0], w[1], w[2], w[3]);
            }
            else
            {
#pragma unroll
                for (int q = 0; q < 16; ++q)
                    if (j0 + q < x) orow[int64_t(s) * x + q] = O(m[q] <= uint16_t(s));
            }
        }
    }
}

size_t large_sort_ws(int64_t b, int64_t x)
{
    const int64_t xp = padded_x(x);
    return 2 * ((size_t(b * xp) * 8 + 255) / 256) * 256 + ((size_t(b * x) * 2 + 255) / 256) * 256;
}

// Sorted times of images with X > 16384 into `tm` (inside or outside ws).
template <typename I>
void large_sorted_times(const I *in, uint16_t *tm, int64_t b, int64_t t, int64_t x, void *ws, cudaStream_t s)
{
    const int64_t xp = padded_x(x);
    SPK_REQUIRE(x < (int64_t(1) << 32), "at most 2^32 - 1 values per image");
    SPK_REQUIRE(b <= 65535, "at most 65535 images per call on the large-image path");
    uint64_t *k0 = static_cast<uint64_t *>(ws);
    uint64_t *k1 = reinterpret_cast<uint64_t *>(static_cast<char *>(ws) + ((size_t(b * xp) * 8 + 255) / 256) * 256);
    const size_t smem = size_t(kChunk) * 8;
    SPK_CUDA(cudaFuncSetAttribute(chunk_sort_kernel<I>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    chunk_sort_kernel<I><<<dim3(unsigned(xp / kChunk), unsigned(b)), kCodeThreads, smem, s>>>(in, k0, x, xp);
    SPK_LAUNCHED();
    for (int64_t L = kChunk; L < xp; L *= 2)
    {
        merge_round_kernel<<<grid_for(b * xp / kMergeItems, 256), 256, 0, s>>>(k0, k1, b, xp, L);
        SPK_LAUNCHED();
        std::swap(k0, k1);
    }
    sorted_times_kernel<<<dim3(unsigned(std::min<int64_t>(ceil_div(x, 256), 1024)), unsigned(b)), 256, 0, s>>>(
        k0, tm, b, x, xp, int(t));
    SPK_LAUNCHED();
}

// Workspace tail of the large path that holds the times.
uint16_t *large_times_slot(void *ws, int64_t b, int64_t x)
{
    const int64_t xp = padded_x(x);
    return reinterpret_cast<uint16_t *>(static_cast<char *>(ws) + 2 * ((size_t(b * xp) * 8 + 255) / 256) * 256);
}
}  // namespace

// Bytes of scratch the sorted code needs (0 when X <= 16384).
size_t rank_times_ws(int64_t b, int64_t x, int sort) { return (sort && x > kMaxSortX) ? large_sort_ws(b, x) : 0; }

// The compacting kernel for rows of 257 .. 2048 values (false: not taken).
template <typename I, typename O, bool TIMES>
bool rank_reg(const I *in, O *out, int64_t b, int64_t t, int64_t x, cudaStream_t s)
{
    if (x <= 256 || x > kRegMax || b > 0x7FFFFFFF) return false;
    rank_compact_kernel<I, O, TIMES><<<unsigned(b), kRegThreads, 0, s>>>(in, out, x, int(t));
    SPK_LAUNCHED();
    return true;
}

// First-spike times [B, X] u16 of the rank-order (sort) or latency code.
void rank_times(const void *in, spk_dtype itype, uint16_t *times, int64_t b, int64_t t, int64_t x, int sort, void *ws,
                cudaStream_t s)
{
    SPK_REQUIRE(itype == SPK_F32 || itype == SPK_U8, "coding supports F32/U8 input");
    if (b == 0) return;
    if (sort && x > kMaxSortX)
    {
        SPK_REQUIRE(ws != nullptr, "workspace is too small");
        if (itype == SPK_F32)
            large_sorted_times((const float *)in, times, b, t, x, ws, s);
        else
            large_sorted_times((const uint8_t *)in, times, b, t, x, ws, s);
        return;
    }
    if (sort)
    {
        int npow2 = 2;
        while (npow2 < x) npow2 <<= 1;
        const size_t smem = size_t(npow2) * 8 + size_t(x) * 2 + 16;
        auto go = [&](auto k, const auto *p) {
            SPK_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
            k<<<unsigned(b), kCodeThreads, smem, s>>>(p, times, x, int(t), npow2);
        };
        if (itype == SPK_F32)
        {
            if (!rank_reg<float, uint16_t, true>((const float *)in, times, b, t, x, s))
                go(rank_sorted_kernel<float, uint16_t, true>, (const float *)in);
        }
        else if (!rank_reg<uint8_t, uint16_t, true>((const uint8_t *)in, times, b, t, x, s))
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

size_t spk_rank_code_workspace(int64_t b, int64_t x, int sort) { return rank_times_ws(b, x, sort); }

spk_status spk_rank_code(const void *in, spk_dtype itype, void *out, spk_dtype otype, int64_t b, int64_t t, int64_t x,
                         int sort, void *ws, size_t ws_bytes, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(t > 0, "input time can't be less than 1");
        SPK_REQUIRE(b >= 0 && x >= 1, "invalid dims");
        SPK_REQUIRE(t <= 65535, "time is limited to 65535 steps");
        if (b == 0) return;
        if (sort && x > kMaxSortX)
        {
            SPK_REQUIRE(itype == SPK_F32 || itype == SPK_U8, "sorted rank coding supports F32/U8 input");
            SPK_REQUIRE(otype == SPK_U8 || otype == SPK_F32, "output type must be U8 or F32");
            SPK_REQUIRE(ws != nullptr && ws_bytes >= large_sort_ws(b, x), "workspace is too small");
            cudaStream_t s = stream_of(stream);
            uint16_t *tm = large_times_slot(ws, b, x);
            rank_times(in, itype, tm, b, t, x, sort, ws, s);
            if (otype == SPK_U8)
                rows_from_times_kernel<uint8_t><<<grid_for(b * ceil_div(x, 16), 256), 256, 0, s>>>(tm, (uint8_t *)out,
                                                                                                  b, int(t), x);
            else
                rows_from_times_kernel<float><<<grid_for(b * ceil_div(x, 16), 256), 256, 0, s>>>(tm, (float *)out, b,
                                                                                                int(t), x);
            SPK_LAUNCHED();
            return;
        }
        if (sort)
        {
            int npow2 = 2;
            while (npow2 < x) npow2 <<= 1;
            size_t smem = size_t(npow2) * 8 + size_t(x) * 2 + 16;
            SPK_REQUIRE(otype == SPK_U8 || otype == SPK_F32, "output type must be U8 or F32");
            cudaStream_t cs = stream_of(stream);
            if (itype == SPK_F32 && otype == SPK_U8 && rank_reg<float, uint8_t, false>((const float *)in, (uint8_t *)out,
                                                                                       b, t, x, cs))
                return;
            if (itype == SPK_F32 && otype == SPK_F32 && rank_reg<float, float, false>((const float *)in, (float *)out,
                                                                                      b, t, x, cs))
                return;
            if (itype == SPK_U8 && otype == SPK_U8 && rank_reg<uint8_t, uint8_t, false>((const uint8_t *)in,
                                                                                        (uint8_t *)out, b, t, x, cs))
                return;
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
