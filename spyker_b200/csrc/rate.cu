// Rate (Poisson) coding and its fire / gather / pool:
//   rate code   src/spyker/cpu/code.cpp:134-243 (interval table cpu/init.cpp:120-149)
//   rate fire   src/spyker/cpu/fire.cpp:84-113
//   rate gather src/spyker/cpu/time.cpp:87-92
//   rate pool   src/spyker/cpu/pool.cpp:88-137
// Spike counts are cumulative: output step t holds each neuron's number of
// spikes up to t.
#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include "common.cuh"

namespace spk
{
void rank_times(const void *in, spk_dtype itype, uint16_t *times, int64_t b, int64_t t, int64_t x, int sort, void *ws,
                cudaStream_t s);
size_t rank_times_ws(int64_t b, int64_t x, int sort);
uint64_t draw_seed();

namespace
{
constexpr int kBins = 1024;

// Inter-spike interval table, restated from cpu/init.cpp:120-149: row i (a
// position whose rank / latency time is i) holds kBins intervals; lambda =
// i + 1, r = ceil(scale sqrt(lambda)) (scale 5 for row 0, else 4); every j
// in [max(1, lambda - r), lambda + r] appears nearbyint(ztp(j, lambda) kBins)
// times (ztp = zero-truncated Poisson, F32 as the reference), the remaining
// slots hold lambda.  The reference then applies std::random_shuffle, whose
// order is implementation-defined; here each row is shuffled by Fisher-Yates
// with std::mt19937 seeded by the row, so the multiset of each row is the
// reference's and only the order differs.
void interval_table(int64_t time, uint16_t *out)
{
    auto ztp = [](uint16_t k, float a) {
        float p = 1 / (std::exp(a) - 1);
        for (int64_t i = 1; i <= k; ++i) p *= a / i;
        return p;
    };
    for (int64_t i = 0; i < time; ++i)
    {
        const float scale = i < 1 ? 5 : 4;
        const uint16_t lambda = uint16_t(i + 1), range = uint16_t(std::ceil(scale * std::sqrt(lambda)));
        const uint16_t start = uint16_t(std::max(1, lambda - range)), end = uint16_t(lambda + range);
        uint16_t *row = out + i * kBins;
        int64_t index = 0;
        for (uint16_t j = start; j <= end; ++j)
        {
            int64_t count = int64_t(std::nearbyint(ztp(j, lambda) * kBins));
            if (index + count > kBins) count = kBins - index;
            std::fill(row + index, row + index + count, j);
            index += count;
            if (j == 65535) break;
        }
        std::fill(row + index, row + kBins, lambda);
        std::mt19937 rng(static_cast<std::mt19937::result_type>(i + 1));
        for (int k = kBins - 1; k > 0; --k)
        {
            const int r = int(rng() % uint32_t(k + 1));
            std::swap(row[k], row[r]);
        }
    }
}

// Counter-based random index in [0, kBins): the n-th draw of position
// (sample, x) of a call seeded `seed` (SplitMix64 finaliser of a Weyl
// sequence; the reference draws from one std::mt19937 per sample).
__device__ __forceinline__ uint32_t draw_index(uint64_t seed, uint64_t pos, uint32_t n)
{
    uint64_t z = seed + pos * 0x9E3779B97F4A7C15ull + uint64_t(n) * 0xD1B54A32D192ED03ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return uint32_t(z) & (kBins - 1);
}

// Poisson process per position (cpu/code.cpp:177-191): the first spike
// after one interval drawn from the row of the position's time, each spike
// adds one and draws the next interval.  A time >= T (a position that never
// fires in the rank code) has no row in the table: it never spikes.
template <typename O>
__global__ void rate_code_kernel(const uint16_t *__restrict__ times, const uint16_t *__restrict__ table,
                                 O *__restrict__ out, int64_t b, int t, int64_t x, uint64_t seed)
{
    const int64_t total = b * x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t s = k / x, j = k - s * x;
        const int row = times[k];
        O *o = out + s * t * x + j;
        if (row >= t)
        {
            for (int i = 0; i < t; ++i) o[int64_t(i) * x] = O(0);
            continue;
        }
        const uint16_t *tr = table + int64_t(row) * kBins;
        uint32_t n = 0, value = 0;
        uint32_t next = tr[draw_index(seed, uint64_t(k), n++)];
        for (int i = 0; i < t; ++i)
        {
            if (next == uint32_t(i)) ++value, next += tr[draw_index(seed, uint64_t(k), n++)];
            o[int64_t(i) * x] = O(value);
        }
    }
}

// cpu/fire.cpp:84-113: a neuron spikes (count + 1) when its input exceeds
// the value at its last spike by more than the threshold; outputs are the
// running counts.
template <typename I, typename O>
__global__ void rate_fire_kernel(const I *__restrict__ in, O *__restrict__ out, int64_t b, int t, int64_t x, I thr)
{
    const int64_t total = b * x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t s = k / x, j = k - s * x;
        const I *p = in + s * t * x + j;
        O *o = out + s * t * x + j;
        I value = I(0);
        O spikes = O(0);
        for (int i = 0; i < t; ++i)
        {
            const I v = p[int64_t(i) * x];
            if (value + thr < v) spikes = O(spikes + O(1)), value = v;
            o[int64_t(i) * x] = spikes;
        }
    }
}

// cpu/time.cpp:87-92: the last step's counts.
template <typename I, typename O>
__global__ void rate_gather_kernel(const I *__restrict__ in, O *__restrict__ out, int64_t b, int t, int64_t x)
{
    const int64_t total = b * x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t s = k / x, j = k - s * x;
        out[k] = O(in[(s * t + t - 1) * x + j]);
    }
}

// cpu/pool.cpp:88-137: per output cell the window position with the highest
// rate (first in row-major window order on ties: strict >), then every step
// copies that position's value.
template <typename T, typename R>
__global__ void rate_pool_kernel(const T *__restrict__ in, const R *__restrict__ rates, T *__restrict__ out, int64_t b,
                                 int t, int64_t c, int h, int w, int oh, int ow, int ky, int kx, int sy, int sx)
{
    const int64_t total = b * c * oh * ow;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        const int ox = int(k % ow), oy = int((k / ow) % oh);
        const int64_t plane = k / (int64_t(oh) * ow), s = plane / c, ch = plane - s * c;
        const R *r = rates + plane * h * w;
        R best = Lowest<R>::v();
        int bi = 0;
        for (int a = 0; a < ky; ++a)
            for (int bb = 0; bb < kx; ++bb)
            {
                const int idx = (oy * sy + a) * w + ox * sx + bb;
                if (best < r[idx]) best = r[idx], bi = idx;
            }
        for (int i = 0; i < t; ++i)
            out[((s * t + i) * c + ch) * int64_t(oh) * ow + int64_t(oy) * ow + ox] =
                in[((s * t + i) * c + ch) * int64_t(h) * w + bi];
    }
}
}  // namespace
}  // namespace spk

using namespace spk;

extern "C" {

void spk_rate_interval_table(int64_t time, uint16_t *out_host) { interval_table(time, out_host); }

size_t spk_rate_code_workspace(int64_t b, int64_t t, int64_t x, int sort)
{
    auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
    return al(size_t(t) * kBins * 2) + al(size_t(b * x) * 2) + al(rank_times_ws(b, x, sort));
}

spk_status spk_rate_code(const void *in, spk_dtype itype, void *out, spk_dtype otype, int64_t b, int64_t t, int64_t x,
                         int sort, void *ws, size_t ws_bytes, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(t > 0 && t <= 65535, "time steps must be 1..65535");
        SPK_REQUIRE(b >= 0 && x >= 1, "invalid dims");
        SPK_REQUIRE(ws != nullptr && ws_bytes >= spk_rate_code_workspace(b, t, x, sort), "workspace is too small");
        if (b == 0) return;
        cudaStream_t s = stream_of(stream);
        auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
        uint8_t *base = static_cast<uint8_t *>(ws);
        uint16_t *table = reinterpret_cast<uint16_t *>(base);
        uint16_t *times = reinterpret_cast<uint16_t *>(base + al(size_t(t) * kBins * 2));
        void *sort_ws = base + al(size_t(t) * kBins * 2) + al(size_t(b * x) * 2);
        std::vector<uint16_t> host(size_t(t) * kBins);
        interval_table(t, host.data());
        SPK_CUDA(cudaMemcpyAsync(table, host.data(), host.size() * 2, cudaMemcpyHostToDevice, s));
        SPK_CUDA(cudaStreamSynchronize(s));  // the host table is released on return
        rank_times(in, itype, times, b, t, x, sort, sort_ws, s);
        const uint64_t seed = draw_seed();
        dispatch(otype, [&](auto z) {
            using O = decltype(z);
            rate_code_kernel<O><<<grid_for(b * x, 256), 256, 0, s>>>(times, table, static_cast<O *>(out), b, int(t), x,
                                                                      seed);
        });
        SPK_LAUNCHED();
    });
}

spk_status spk_rate_fire(const void *in, spk_dtype itype, void *out, spk_dtype otype, int64_t b, int64_t t, int64_t x,
                         double threshold, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(b >= 0 && t >= 1 && x >= 1, "invalid dims");
        if (b == 0) return;
        cudaStream_t s = stream_of(stream);
        dispatch(itype, [&](auto zi) {
            using I = decltype(zi);
            dispatch(otype, [&](auto zo) {
                using O = decltype(zo);
                rate_fire_kernel<I, O><<<grid_for(b * x, 256), 256, 0, s>>>(
                    static_cast<const I *>(in), static_cast<O *>(out), b, int(t), x, scalar_to<I>(threshold));
            });
        });
        SPK_LAUNCHED();
    });
}

spk_status spk_rate_gather(const void *in, spk_dtype itype, void *out, spk_dtype otype, int64_t b, int64_t t,
                           int64_t x, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(b >= 0 && t >= 1 && x >= 1, "invalid dims");
        if (b == 0) return;
        cudaStream_t s = stream_of(stream);
        dispatch(itype, [&](auto zi) {
            using I = decltype(zi);
            dispatch(otype, [&](auto zo) {
                using O = decltype(zo);
                rate_gather_kernel<I, O><<<grid_for(b * x, 256), 256, 0, s>>>(static_cast<const I *>(in),
                                                                               static_cast<O *>(out), b, int(t), x);
            });
        });
        SPK_LAUNCHED();
    });
}

spk_status spk_rate_pool(const void *in, const void *rates, spk_dtype type, spk_dtype rtype, void *out, int64_t b,
                         int64_t t, int64_t c, int64_t h, int64_t w, int64_t oh, int64_t ow, const int64_t *kernel2,
                         const int64_t *stride2, const int64_t *pad4, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(kernel2 != nullptr && stride2 != nullptr, "null kernel or stride");
        const Pad4 p = pad_of(pad4);
        SPK_REQUIRE(p.top == 0 && p.left == 0 && p.bottom == 0 && p.right == 0,
                    "padding is not supported in rate pooling");
        SPK_REQUIRE(b >= 0 && t >= 1 && c >= 1 && h >= 1 && w >= 1 && kernel2[0] >= 1 && kernel2[1] >= 1 &&
                        stride2[0] >= 1 && stride2[1] >= 1,
                    "invalid dims");
        SPK_REQUIRE(oh == (h - kernel2[0]) / stride2[0] + 1 && ow == (w - kernel2[1]) / stride2[1] + 1 && h >= kernel2[0] &&
                        w >= kernel2[1],
                    "output shape does not match");
        if (b == 0) return;
        cudaStream_t s = stream_of(stream);
        dispatch(type, [&](auto zt) {
            using T = decltype(zt);
            dispatch(rtype, [&](auto zr) {
                using R = decltype(zr);
                rate_pool_kernel<T, R><<<grid_for(b * c * oh * ow, 256), 256, 0, s>>>(
                    static_cast<const T *>(in), static_cast<const R *>(rates), static_cast<T *>(out), b, int(t), c,
                    int(h), int(w), int(oh), int(ow), int(kernel2[0]), int(kernel2[1]), int(stride2[0]),
                    int(stride2[1]));
            });
        });
        SPK_LAUNCHED();
    });
}

}  // extern "C"
