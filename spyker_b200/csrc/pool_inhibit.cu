// Max pooling of spike / potential planes and per-pixel lateral inhibition.
#include "common.cuh"

namespace spk
{
namespace
{
// shuffle-able carrier of each element type
template <typename T>
struct Wide
{
    using type = T;
};
template <>
struct Wide<uint8_t>
{
    using type = int;
};
// src/spyker/cpu/pool.cpp:53-86: zero pad, then max over the window
// (initial value Limits<T>::min()); on cumulative spikes this is the earliest
// spike in the window.  One thread per output element.
// Index type I: 32-bit when the output has fewer than 2^31 elements (integer
// division by a runtime value is several times cheaper than in 64 bits).
template <typename T, typename I>
__global__ void pool_kernel(const T *__restrict__ in, T *__restrict__ out, I n, I h, I w, I oh, I ow, int ky, int kx,
                            int sy, int sx, int top, int left)
{
    const I total = n * oh * ow;
    for (I k = I(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += I(gridDim.x) * blockDim.x)
    {
        const I r = k / ow, xo = k - r * ow, p = r / oh, yo = r - p * oh;
        const T *plane = in + int64_t(p) * h * w;
        T m = Lowest<T>::v();
        for (int a = 0; a < ky; ++a)
        {
            const int yy = int(yo) * sy + a - top;
            for (int b = 0; b < kx; ++b)
            {
                const int xx = int(xo) * sx + b - left;
                T v = (yy >= 0 && yy < int(h) && xx >= 0 && xx < int(w)) ? plane[yy * int64_t(w) + xx] : T(0);
                m = (m < v) ? v : m;  // std::max(m, v)
            }
        }
        out[k] = m;
    }
}

// Large windows (e.g. global pooling): one warp per output element, the
// lanes striding over the window and a shuffle max at the end (max is order
// independent, so this equals the reference's sequential scan).
template <typename T, typename I>
__global__ void pool_warp_kernel(const T *__restrict__ in, T *__restrict__ out, I n, I h, I w, I oh, I ow, int ky,
                                 int kx, int sy, int sx, int top, int left)
{
    const int lane = threadIdx.x & 31;
    const I total = n * oh * ow;
    const I warps = (I(gridDim.x) * blockDim.x) >> 5;
    for (I k = (I(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; k < total; k += warps)
    {
        const I r = k / ow, xo = k - r * ow, p = r / oh, yo = r - p * oh;
        const T *plane = in + int64_t(p) * h * w;
        T m = Lowest<T>::v();
        int a = lane / kx, b = lane % kx;  // window position of this lane, advanced by 32 per step
        const int da = 32 / kx, db = 32 % kx;
        for (int i = lane; i < ky * kx; i += 32)
        {
            const int yy = int(yo) * sy + a - top, xx = int(xo) * sx + b - left;
            const T v = (yy >= 0 && yy < int(h) && xx >= 0 && xx < int(w)) ? plane[yy * int64_t(w) + xx] : T(0);
            m = (m < v) ? v : m;
            a += da, b += db;
            if (b >= kx) b -= kx, ++a;
        }
        for (int o = 16; o > 0; o >>= 1)
        {
            const T v = T(__shfl_xor_sync(0xffffffffu, (typename Wide<T>::type)(m), o));
            m = (m < v) ? v : m;
        }
        if (lane == 0) out[k] = m;
    }
}

// src/spyker/cpu/inhibit.cpp:41-121 over [B, T, C, X], one thread per (b, x):
// per step the first channel with the largest value (strict >), the number
// of steps whose maximum exceeds the threshold, the winning channel taken at
// step T - max(count, 1); every other channel is multiplied by zero at all
// steps (the reference's `id *= (index == channel)`).
template <typename T>
__global__ void inhibit_kernel(T *__restrict__ data, int64_t b, int t, int c, int64_t x, T thr)
{
    const int64_t total = b * x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        int64_t s = k / x, j = k % x;
        T *base = data + s * int64_t(t) * c * x + j;
        int sum = 0;
        for (int q = 0; q < t; ++q)
        {
            const T *row = base + int64_t(q) * c * x;
            T m = row[0];
            for (int z = 1; z < c; ++z)
            {
                T v = row[int64_t(z) * x];
                m = (v > m) ? v : m;
            }
            sum += (m > thr);
        }
        int ts = t - (sum > 1 ? sum : 1);
        const T *row = base + int64_t(ts) * c * x;
        T m = row[0];
        int win = 0;
        for (int z = 1; z < c; ++z)
        {
            T v = row[int64_t(z) * x];
            if (v > m) m = v, win = z;
        }
        for (int q = 0; q < t; ++q)
        {
            T *r = base + int64_t(q) * c * x;
            for (int z = 0; z < c; ++z)
                if (z != win) r[int64_t(z) * x] = r[int64_t(z) * x] * T(0);
        }
    }
}
}  // namespace
}  // namespace spk

using namespace spk;

extern "C" {

spk_status spk_rank_pool(const void *in, void *out, spk_dtype type, int64_t n, int64_t h, int64_t w, int64_t oh,
                         int64_t ow, int64_t ky, int64_t kx, int64_t sy, int64_t sx, const int64_t *pad4,
                         spk_stream stream)
{
    return guarded([&] {
        Pad4 p = pad_of(pad4);
        SPK_REQUIRE(ky >= 1 && kx >= 1 && sy >= 1 && sx >= 1, "kernel and stride must be at least 1");
        SPK_REQUIRE(oh == (h + p.top + p.bottom - ky) / sy + 1 && ow == (w + p.left + p.right - kx) / sx + 1,
                    "output shape is not compatible");
        SPK_REQUIRE(oh > 0 && ow > 0, "input and kernel shapes are not compatible");
        if (n == 0) return;
        dispatch(type, [&](auto z) {
            using T = decltype(z);
            const bool small = n * oh * ow * 32 < (int64_t(1) << 31) && n * h * w < (int64_t(1) << 31);
            auto go = [&](auto idx) {
                using I = decltype(idx);
                if (ky * kx >= 64)
                    pool_warp_kernel<T, I><<<grid_for(n * oh * ow * 32, 256, 16), 256, 0, stream_of(stream)>>>(
                        (const T *)in, (T *)out, I(n), I(h), I(w), I(oh), I(ow), int(ky), int(kx), int(sy), int(sx),
                        int(p.top), int(p.left));
                else
                    pool_kernel<T, I><<<grid_for(n * oh * ow, 256, 16), 256, 0, stream_of(stream)>>>(
                        (const T *)in, (T *)out, I(n), I(h), I(w), I(oh), I(ow), int(ky), int(kx), int(sy), int(sx),
                        int(p.top), int(p.left));
            };
            if (small)
                go(uint32_t());
            else
                go(int64_t());
            SPK_LAUNCHED();
        });
    });
}

spk_status spk_rank_inhibit(void *data, spk_dtype type, int64_t b, int64_t t, int64_t c, int64_t x, double threshold,
                            spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(b >= 0 && t >= 1 && c >= 1 && x >= 0, "invalid dims");
        SPK_REQUIRE(c <= 65535 && t <= 65535, "channel and time counts are limited to 65535");
        if (b * x == 0) return;
        dispatch(type, [&](auto z) {
            using T = decltype(z);
            inhibit_kernel<T><<<grid_for(b * x, 128), 128, 0, stream_of(stream)>>>((T *)data, b, int(t), int(c), x,
                                                                                  scalar_to<T>(threshold));
            SPK_LAUNCHED();
        });
    });
}

}  // extern "C"
