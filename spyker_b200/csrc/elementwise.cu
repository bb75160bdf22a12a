// Bandwidth-bound elementwise ops of the hot path: threshold, infinite, fire,
// gather, scatter, pad.  Each is a grid-stride loop over 16-byte vectors
// (128-bit loads/stores) with a scalar tail; grids are sized from the SM count.
#include "common.cuh"

namespace spk
{
namespace
{
template <typename T>
struct alignas(16) Vec16
{
    static constexpr int N = 16 / sizeof(T);
    T v[N];
};

template <typename T>
__device__ __forceinline__ bool aligned16(const void *p)
{
    return (reinterpret_cast<uintptr_t>(p) & 15) == 0;
}

// src/spyker/cpu/fire.cpp:41-51 — in place, `x <= threshold -> value`.
template <typename T>
__global__ void threshold_kernel(T *__restrict__ data, int64_t n, T thr, T value)
{
    constexpr int V = Vec16<T>::N;
    const int64_t nv = n / V;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    Vec16<T> *vd = reinterpret_cast<Vec16<T> *>(data);
    for (int64_t k = i; k < nv; k += stride)
    {
        Vec16<T> v = vd[k];
#pragma unroll
        for (int j = 0; j < V; ++j) v.v[j] = (v.v[j] <= thr) ? value : v.v[j];
        vd[k] = v;
    }
    for (int64_t k = nv * V + i; k < n; k += stride)
        if (data[k] <= thr) data[k] = value;
}

template <typename T>
__global__ void threshold_scalar_kernel(T *__restrict__ data, int64_t n, T thr, T value)
{
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += int64_t(gridDim.x) * blockDim.x)
        if (data[k] <= thr) data[k] = value;
}

// src/spyker/cpu/fire.cpp:59-65 — steps 0..T-2 of every sample set to value.
template <typename T>
__global__ void infinite_kernel(T *__restrict__ data, int64_t b, int64_t t, int64_t x, T value)
{
    const int64_t per = (t - 1) * x;
    const int64_t total = b * per;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        int64_t s = k / per, r = k % per;
        data[s * t * x + r] = value;
    }
}

// src/spyker/cpu/fire.cpp:67-82 — out = in > threshold.  The F32 -> U8 case
// reads four float4 vectors and writes one 16-byte vector per step.
template <typename I, typename O>
__global__ void fire_kernel(const I *__restrict__ in, O *__restrict__ out, int64_t n, I thr)
{
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const int64_t i0 = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    constexpr int V = 16;
    const int64_t nv = n / V;
    for (int64_t k = i0; k < nv; k += stride)
    {
        I src[V];
        const Vec16<I> *vi = reinterpret_cast<const Vec16<I> *>(in + k * V);
#pragma unroll
        for (int q = 0; q < V / Vec16<I>::N; ++q)
        {
            Vec16<I> v = vi[q];
#pragma unroll
            for (int j = 0; j < Vec16<I>::N; ++j) src[q * Vec16<I>::N + j] = v.v[j];
        }
        Vec16<O> *vo = reinterpret_cast<Vec16<O> *>(out + k * V);
#pragma unroll
        for (int q = 0; q < V / Vec16<O>::N; ++q)
        {
            Vec16<O> v;
#pragma unroll
            for (int j = 0; j < Vec16<O>::N; ++j) v.v[j] = O(src[q * Vec16<O>::N + j] > thr);
            vo[q] = v;
        }
    }
    for (int64_t k = nv * V + i0; k < n; k += stride) out[k] = O(in[k] > thr);
}

template <typename I, typename O>
__global__ void fire_scalar_kernel(const I *__restrict__ in, O *__restrict__ out, int64_t n, I thr)
{
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += int64_t(gridDim.x) * blockDim.x)
        out[k] = O(in[k] > thr);
}

// src/spyker/cpu/time.cpp:40-58 — first t with in > threshold, T if never.
template <typename I, typename O>
__global__ void gather_kernel(const I *__restrict__ in, O *__restrict__ out, int64_t b, int64_t t, int64_t x, I thr)
{
    const int64_t total = b * x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        int64_t s = k / x, j = k % x;
        const I *p = in + s * t * x + j;
        int64_t first = t;
        for (int64_t q = 0; q < t; ++q)
            if (p[q * x] > thr)
            {
                first = q;
                break;
            }
        out[k] = O(first);
    }
}

// src/spyker/cpu/time.cpp:60-78 — out[t] = (U32(t) >= in).
template <typename I, typename O>
__global__ void scatter_kernel(const I *__restrict__ in, O *__restrict__ out, int64_t b, int64_t t, int64_t x)
{
    const int64_t total = b * t * x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        int64_t j = k % x, r = k / x, q = r % t, s = r / t;
        out[k] = O(uint32_t(q) >= in[s * x + j]);
    }
}

// src/spyker/cpu/pool.cpp:41-51 — pad (top, left, bottom, right) with value.
template <typename T>
__global__ void pad_kernel(const T *__restrict__ in, T *__restrict__ out, int64_t n, int64_t h, int64_t w, int64_t oh,
                           int64_t ow, int64_t top, int64_t left, T value)
{
    const int64_t total = n * oh * ow;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        int64_t xo = k % ow, r = k / ow, yo = r % oh, p = r / oh;
        int64_t yi = yo - top, xi = xo - left;
        out[k] = (yi >= 0 && yi < h && xi >= 0 && xi < w) ? in[(p * h + yi) * w + xi] : value;
    }
}
}  // namespace
}  // namespace spk

using namespace spk;

extern "C" {

spk_status spk_threshold(void *data, spk_dtype type, int64_t n, double threshold, double value, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(n >= 0, "negative size");
        if (n == 0) return;
        SPK_REQUIRE(data != nullptr, "null data");
        dispatch(type, [&](auto z) {
            using T = decltype(z);
            if ((reinterpret_cast<uintptr_t>(data) % 16) == 0)
                threshold_kernel<T><<<grid_for(ceil_div(n, Vec16<T>::N), 256), 256, 0, stream_of(stream)>>>(
                    (T *)data, n, scalar_to<T>(threshold), scalar_to<T>(value));
            else
                threshold_scalar_kernel<T><<<grid_for(n, 256), 256, 0, stream_of(stream)>>>(
                    (T *)data, n, scalar_to<T>(threshold), scalar_to<T>(value));
            SPK_LAUNCHED();
        });
    });
}

spk_status spk_rank_infinite(void *data, spk_dtype type, int64_t b, int64_t t, int64_t x, double value,
                             spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(b >= 0 && t >= 1 && x >= 0, "invalid dims");
        if (b * (t - 1) * x == 0) return;
        dispatch(type, [&](auto z) {
            using T = decltype(z);
            infinite_kernel<T><<<grid_for(b * (t - 1) * x, 256), 256, 0, stream_of(stream)>>>((T *)data, b, t, x,
                                                                                            scalar_to<T>(value));
            SPK_LAUNCHED();
        });
    });
}

spk_status spk_rank_fire(const void *in, spk_dtype itype, void *out, spk_dtype otype, int64_t n, double threshold,
                         spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(n >= 0, "negative size");
        if (n == 0) return;
        dispatch(itype, [&](auto a) {
            dispatch(otype, [&](auto b) {
                using I = decltype(a);
                using O = decltype(b);
                bool al = (reinterpret_cast<uintptr_t>(in) % 16) == 0 && (reinterpret_cast<uintptr_t>(out) % 16) == 0;
                if (al)
                    fire_kernel<I, O><<<grid_for(ceil_div(n, 16), 256), 256, 0, stream_of(stream)>>>(
                        (const I *)in, (O *)out, n, scalar_to<I>(threshold));
                else
                    fire_scalar_kernel<I, O><<<grid_for(n, 256), 256, 0, stream_of(stream)>>>(
                        (const I *)in, (O *)out, n, scalar_to<I>(threshold));
                SPK_LAUNCHED();
            });
        });
    });
}

spk_status spk_rank_gather(const void *in, spk_dtype itype, void *out, spk_dtype otype, int64_t b, int64_t t,
                           int64_t x, double threshold, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(b >= 0 && t >= 1 && x >= 0, "invalid dims");
        if (b * x == 0) return;
        dispatch(itype, [&](auto a) {
            dispatch(otype, [&](auto c) {
                using I = decltype(a);
                using O = decltype(c);
                gather_kernel<I, O><<<grid_for(b * x, 256), 256, 0, stream_of(stream)>>>(
                    (const I *)in, (O *)out, b, t, x, scalar_to<I>(threshold));
                SPK_LAUNCHED();
            });
        });
    });
}

spk_status spk_rank_scatter(const void *in, spk_dtype itype, void *out, spk_dtype otype, int64_t b, int64_t t,
                            int64_t x, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(b >= 0 && t >= 1 && x >= 0, "invalid dims");
        if (b * t * x == 0) return;
        dispatch(itype, [&](auto a) {
            dispatch(otype, [&](auto c) {
                using I = decltype(a);
                using O = decltype(c);
                scatter_kernel<I, O><<<grid_for(b * t * x, 256), 256, 0, stream_of(stream)>>>((const I *)in, (O *)out,
                                                                                             b, t, x);
                SPK_LAUNCHED();
            });
        });
    });
}

spk_status spk_pad(const void *in, void *out, spk_dtype type, int64_t n, int64_t h, int64_t w, const int64_t *pad4,
                   double value, spk_stream stream)
{
    return guarded([&] {
        Pad4 p = pad_of(pad4);
        SPK_REQUIRE(n >= 0 && h >= 0 && w >= 0, "invalid dims");
        int64_t oh = h + p.top + p.bottom, ow = w + p.left + p.right;
        if (n * oh * ow == 0) return;
        dispatch(type, [&](auto z) {
            using T = decltype(z);
            pad_kernel<T><<<grid_for(n * oh * ow, 256), 256, 0, stream_of(stream)>>>(
                (const T *)in, (T *)out, n, h, w, oh, ow, p.top, p.left, scalar_to<T>(value));
            SPK_LAUNCHED();
        });
    });
}

}  // extern "C"
