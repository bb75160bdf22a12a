// Max pooling of spike / potential planes and per-pixel lateral inhibition.
#include "common.cuh"

namespace spk
{
namespace
{
// src/spyker/cpu/pool.cpp:53-86: zero pad, then max over the window
// (initial value Limits<T>::min()); on cumulative spikes this is the earliest
// spike in the window.  One thread per output element.
template <typename T>
__global__ void pool_kernel(const T *__restrict__ in, T *__restrict__ out, int64_t n, int64_t h, int64_t w, int64_t oh,
                            int64_t ow, int ky, int kx, int sy, int sx, int top, int left)
{
    const int64_t total = n * oh * ow;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        int64_t xo = k % ow, r = k / ow, yo = r % oh, p = r / oh;
        const T *plane = in + p * h * w;
        T m = Lowest<T>::v();
        for (int a = 0; a < ky; ++a)
        {
            int64_t yy = yo * sy + a - top;
            for (int b = 0; b < kx; ++b)
            {
                int64_t xx = xo * sx + b - left;
                T v = (yy >= 0 && yy < h && xx >= 0 && xx < w) ? plane[yy * w + xx] : T(0);
                m = (m < v) ? v : m;  // std::max(m, v)
            }
        }
        out[k] = m;
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
            pool_kernel<T><<<grid_for(n * oh * ow, 256), 256, 0, stream_of(stream)>>>(
                (const T *)in, (T *)out, n, h, w, oh, ow, int(ky), int(kx), int(sy), int(sx), int(p.top), int(p.left));
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
