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

constexpr int64_t kPoolTileBytes = 16 * 1024;  // planes staged per CTA (at least one)
constexpr int64_t kPoolPlaneMax = 96 * 1024;   // larger planes take the direct kernels

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

// Byte-wise max of four u8 lanes; spikes (0/1 bytes) take the OR.
__device__ __forceinline__ uint32_t bmax4(uint32_t a, uint32_t b)
{
    const uint32_t o = a | b;
    return (o & 0xFEFEFEFEu) ? __vmaxu4(a, b) : o;
}

// Whole planes staged in shared memory: a CTA takes `per_tile` consecutive
// planes (one contiguous byte range, copied with 16-byte loads) and computes
// their outputs from shared memory, so global traffic is one coalesced read
// of the input and one of the output.  Max is order independent except for
// NaN, and the thread kind takes the taps in the reference's row-major order.
// KIND 0: thread per output; 1: warp per output (windows of 64 taps and
// more); 2: u8, windows 2 wide with stride 2 and no padding: four outputs
// per thread from 32-bit words; 3: u8, the window is the whole plane: a
// thread reduces a plane's words.
template <typename T, int KIND>
__global__ void __launch_bounds__(256) pool_plane_kernel(const T *__restrict__ in, T *__restrict__ out, int64_t n,
                                                         int h, int w, int oh, int ow, int ky, int kx, int sy, int sx,
                                                         int top, int left, int per_tile)
{
    constexpr bool WARP = KIND == 1;
    extern __shared__ __align__(16) unsigned char pool_smem[];
    const int hw = h * w, ohw = oh * ow;
    const int64_t tiles = (n + per_tile - 1) / per_tile;
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x)
    {
        const int64_t p0 = tile * per_tile;
        const int np = int(min(int64_t(per_tile), n - p0));
        __syncthreads();  // the previous tile's outputs are done
        const int shift = stage_bytes(pool_smem, reinterpret_cast<const unsigned char *>(in + p0 * hw),
                                      int64_t(np) * hw * int64_t(sizeof(T)));
        __syncthreads();
        const T *sp = reinterpret_cast<const T *>(pool_smem + shift);
        T *op = out + p0 * ohw;
        const int cnt = np * ohw;
        if constexpr (KIND == 2)
        {
            const unsigned char *sb = pool_smem + shift;
            const int G = (ow + 3) >> 2;
            for (int it = threadIdx.x; it < np * oh * G; it += blockDim.x)
            {
                const int g = it % G, r = it / G, yo = r % oh, pl = r / oh;
                const unsigned char *row = sb + pl * hw + yo * ky * w + 8 * g;
                uint32_t a0 = *reinterpret_cast<const uint32_t *>(row), a1 = *reinterpret_cast<const uint32_t *>(row + 4);
                for (int a = 1; a < ky; ++a)
                {
                    a0 = bmax4(a0, *reinterpret_cast<const uint32_t *>(row + a * w));
                    a1 = bmax4(a1, *reinterpret_cast<const uint32_t *>(row + a * w + 4));
                }
                const uint32_t v = __byte_perm(bmax4(a0, a0 >> 8), bmax4(a1, a1 >> 8), 0x6420);
                unsigned char *o = reinterpret_cast<unsigned char *>(op) + pl * ohw + yo * ow + 4 * g;
                const int nv = min(4, ow - 4 * g);
                for (int q = 0; q < nv; ++q) o[q] = (unsigned char)(v >> (8 * q));
            }
        }
        else if constexpr (KIND == 3)
        {
            const uint32_t *sw = reinterpret_cast<const uint32_t *>(pool_smem + shift);
            const int words = hw >> 2;
            for (int pl = threadIdx.x; pl < np; pl += blockDim.x)
            {
                uint32_t v = 0;
                for (int q = 0; q < words; ++q) v = bmax4(v, sw[pl * words + q]);
                v = bmax4(v, v >> 16);
                v = bmax4(v, v >> 8);
                reinterpret_cast<unsigned char *>(op)[pl] = (unsigned char)(v & 0xFF);
            }
        }
        else if constexpr (!WARP)
        {
            for (int o = threadIdx.x; o < cnt; o += blockDim.x)
            {
                const int pl = o / ohw, r = o - pl * ohw, yo = r / ow, xo = r - yo * ow;
                const T *plane = sp + pl * hw;
                T m = Lowest<T>::v();
                for (int a = 0; a < ky; ++a)
                {
                    const int yy = yo * sy + a - top;
                    for (int b = 0; b < kx; ++b)
                    {
                        const int xx = xo * sx + b - left;
                        const T v = (yy >= 0 && yy < h && xx >= 0 && xx < w) ? plane[yy * w + xx] : T(0);
                        m = (m < v) ? v : m;
                    }
                }
                op[o] = m;
            }
        }
        else
        {
            static_assert(KIND == 1, "pool kind");
            const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
            for (int o = threadIdx.x >> 5; o < cnt; o += warps)
            {
                const int pl = o / ohw, r = o - pl * ohw, yo = r / ow, xo = r - yo * ow;
                const T *plane = sp + pl * hw;
                T m = Lowest<T>::v();
                for (int i = lane; i < ky * kx; i += 32)
                {
                    const int a = i / kx, b = i - a * kx;
                    const int yy = yo * sy + a - top, xx = xo * sx + b - left;
                    const T v = (yy >= 0 && yy < h && xx >= 0 && xx < w) ? plane[yy * w + xx] : T(0);
                    m = (m < v) ? v : m;
                }
                for (int q = 16; q > 0; q >>= 1)
                {
                    const T v = T(__shfl_xor_sync(0xffffffffu, (typename Wide<T>::type)(m), q));
                    m = (m < v) ? v : m;
                }
                if (lane == 0) op[o] = m;
            }
        }
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
// 2x2 windows of stride 2 on u8 planes straight from global memory: a
// thread reads the two input rows of 2 output columns as two 4-byte words
// (W % 4 == 0), for 7 output rows at once, and writes each pair of outputs
// as one 2-byte word (even output width); no staging.  Any odd last
// input row / column is outside every window (oh = H / 2, ow = W / 2).
__global__ void pool2x2_u8_kernel(const uint8_t *__restrict__ in, uint8_t *__restrict__ out, int64_t n, int h, int w,
                                  int oh, int ow)
{
    // a thread takes 2 output columns of RY consecutive output rows (the
    // 2 * RY input words of a column pair are all in flight together)
    constexpr int RY = 7;
    const int g2 = ow / 2;             // 2-output groups per output row
    const int ry = (oh + RY - 1) / RY;  // row blocks per plane
    const int64_t total = n * ry * g2;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        const int g = int(k % g2);
        const int64_t r = k / g2;
        const int64_t pl = r / ry;
        const int y0 = int(r - pl * ry) * RY;
        uint32_t a[RY][2];
#pragma unroll
        for (int q = 0; q < RY; ++q)
            if (y0 + q < oh)
            {
                const uint8_t *row = in + (pl * h + 2 * (y0 + q)) * w + 4 * g;
                a[q][0] = *reinterpret_cast<const uint32_t *>(row);
                a[q][1] = *reinterpret_cast<const uint32_t *>(row + w);
            }
#pragma unroll
        for (int q = 0; q < RY; ++q)
            if (y0 + q < oh)
            {
                const uint32_t m = bmax4(a[q][0], a[q][1]);
                const uint32_t v = bmax4(m, m >> 8);  // bytes 0 and 2 hold the two outputs
                *reinterpret_cast<uint16_t *>(out + (pl * oh + y0 + q) * ow + 2 * g) =
                    uint16_t((v & 0xFFu) | ((v >> 8) & 0xFF00u));
            }
    }
}

// The same for F32 with 4 neighbouring pixels per thread (16-byte loads
// and stores): a warp moves 512 contiguous bytes of every (step, channel)
// row instead of 128, and each thread keeps 4 independent max chains.
__global__ void inhibit_f32x4_kernel(float4 *__restrict__ data, int64_t b, int t, int c, int64_t x4, float thr)
{
    const int64_t total = b * x4;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t s = k / x4, j = k - s * x4;
        float4 *base = data + s * int64_t(t) * c * x4 + j;
        int sum[4] = {0, 0, 0, 0};
        for (int q = 0; q < t; ++q)
        {
            const float4 *row = base + int64_t(q) * c * x4;
            float4 m = row[0];
#pragma unroll 4
            for (int z = 1; z < c; ++z)
            {
                const float4 v = row[int64_t(z) * x4];
                m.x = (v.x > m.x) ? v.x : m.x, m.y = (v.y > m.y) ? v.y : m.y;
                m.z = (v.z > m.z) ? v.z : m.z, m.w = (v.w > m.w) ? v.w : m.w;
            }
            sum[0] += (m.x > thr), sum[1] += (m.y > thr), sum[2] += (m.z > thr), sum[3] += (m.w > thr);
        }
        int win[4];
        float best[4];
#pragma unroll
        for (int l = 0; l < 4; ++l) win[l] = 0;
        {
            int ts[4];
#pragma unroll
            for (int l = 0; l < 4; ++l) ts[l] = t - (sum[l] > 1 ? sum[l] : 1);
#pragma unroll
            for (int l = 0; l < 4; ++l)
                best[l] = reinterpret_cast<const float *>(base + int64_t(ts[l]) * c * x4)[l];
            for (int z = 1; z < c; ++z)
#pragma unroll
                for (int l = 0; l < 4; ++l)
                {
                    const float v = reinterpret_cast<const float *>(base + (int64_t(ts[l]) * c + z) * x4)[l];
                    if (v > best[l]) best[l] = v, win[l] = z;
                }
        }
        for (int q = 0; q < t; ++q)
        {
            float4 *r = base + int64_t(q) * c * x4;
#pragma unroll 4
            for (int z = 0; z < c; ++z)
            {
                float4 v = r[int64_t(z) * x4];
                if (z != win[0]) v.x = v.x * 0.0f;
                if (z != win[1]) v.y = v.y * 0.0f;
                if (z != win[2]) v.z = v.z * 0.0f;
                if (z != win[3]) v.w = v.w * 0.0f;
                r[int64_t(z) * x4] = v;
            }
        }
    }
}
// F32 inhibition with V neighbouring pixels per thread (V = 4 where the
// plane size and alignment allow, else 2 or 1) and 8 loads in flight per
// thread.  The per-step maximum only feeds the count of steps
// above the threshold, so it is taken over two interleaved chains: chain A
// starts at channel 0 and takes the even channels, chain B starts at -inf
// and takes the odd ones; the merged value is above the threshold exactly
// when the reference's sequential maximum is (a NaN in channel 0 stays NaN in
// A and the merge keeps it; other NaNs are skipped by both).  The winner at
// step T - max(count, 1) and the zeroing keep the reference's order.
template <int V>
struct F32Vec;
template <>
struct F32Vec<1>
{
    using T = float;
    static __device__ __forceinline__ float get(const float &v, int) { return v; }
    static __device__ __forceinline__ void set(float &v, int, float x) { v = x; }
};
template <>
struct F32Vec<2>
{
    using T = float2;
    static __device__ __forceinline__ float get(const float2 &v, int l) { return l ? v.y : v.x; }
    static __device__ __forceinline__ void set(float2 &v, int l, float x) { (l ? v.y : v.x) = x; }
};
template <>
struct F32Vec<4>
{
    using T = float4;
    static __device__ __forceinline__ float get(const float4 &v, int l)
    {
        return l == 0 ? v.x : (l == 1 ? v.y : (l == 2 ? v.z : v.w));
    }
    static __device__ __forceinline__ void set(float4 &v, int l, float x)
    {
        (l == 0 ? v.x : (l == 1 ? v.y : (l == 2 ? v.z : v.w))) = x;
    }
};

template <int V>
__global__ void __launch_bounds__(256) inhibit_f32v_kernel(float *__restrict__ data, int64_t b, int t, int c,
                                                           int64_t xv, float thr)
{
    using F = F32Vec<V>;
    using Vec = typename F::T;
    const int64_t total = b * xv;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t s = k / xv, j = k - s * xv;
        Vec *base = reinterpret_cast<Vec *>(data) + s * int64_t(t) * c * xv + j;
        int sum[V];
#pragma unroll
        for (int l = 0; l < V; ++l) sum[l] = 0;
        for (int q = 0; q < t; ++q)
        {
            const Vec *row = base + int64_t(q) * c * xv;
            float ma[V], mb[V];
            const Vec r0 = row[0];
#pragma unroll
            for (int l = 0; l < V; ++l) ma[l] = F::get(r0, l), mb[l] = -INFINITY;
            int z = 1;
#pragma unroll 4
            for (; z + 1 < c; z += 2)
            {
                const Vec u = row[int64_t(z) * xv], w = row[int64_t(z + 1) * xv];
#pragma unroll
                for (int l = 0; l < V; ++l)
                {
                    const float vu = F::get(u, l), vw = F::get(w, l);
                    mb[l] = vu > mb[l] ? vu : mb[l];
                    ma[l] = vw > ma[l] ? vw : ma[l];
                }
            }
            if (z < c)
            {
                const Vec u = row[int64_t(z) * xv];
#pragma unroll
                for (int l = 0; l < V; ++l)
                {
                    const float vu = F::get(u, l);
                    mb[l] = vu > mb[l] ? vu : mb[l];
                }
            }
#pragma unroll
            for (int l = 0; l < V; ++l)
            {
                const float m = mb[l] > ma[l] ? mb[l] : ma[l];
                sum[l] += (m > thr);
            }
        }
        int win[V];
#pragma unroll
        for (int l = 0; l < V; ++l)
        {
            const int ts = t - (sum[l] > 1 ? sum[l] : 1);
            const float *col = reinterpret_cast<const float *>(base + int64_t(ts) * c * xv) + l;
            float best = col[0];
            int w = 0;
#pragma unroll 4
            for (int z = 1; z < c; ++z)
            {
                const float v = col[int64_t(z) * xv * V];
                if (v > best) best = v, w = z;
            }
            win[l] = w;
        }
        for (int q = 0; q < t; ++q)
        {
            Vec *r = base + int64_t(q) * c * xv;
#pragma unroll 8
            for (int z = 0; z < c; ++z)
            {
                Vec v = r[int64_t(z) * xv];
#pragma unroll
                for (int l = 0; l < V; ++l)
                    if (z != win[l]) F::set(v, l, F::get(v, l) * 0.0f);
                r[int64_t(z) * xv] = v;
            }
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
        // a window larger than the padded plane has no output (the staged
        // kernels read whole windows inside the plane)
        SPK_REQUIRE(h + p.top + p.bottom >= ky && w + p.left + p.right >= kx,
                    "input and kernel shapes are not compatible");
        SPK_REQUIRE(oh == (h + p.top + p.bottom - ky) / sy + 1 && ow == (w + p.left + p.right - kx) / sx + 1,
                    "output shape is not compatible");
        SPK_REQUIRE(oh > 0 && ow > 0, "input and kernel shapes are not compatible");
        if (n == 0) return;
        dispatch(type, [&](auto z) {
            using T = decltype(z);
            const int64_t plane = h * w * int64_t(sizeof(T));
            // word kernels: u8, 4-byte aligned rows and planes, no padding
            const bool words = sizeof(T) == 1 && reinterpret_cast<uintptr_t>(in) % 4 == 0 && (h * w) % 4 == 0 &&
                               p.top == 0 && p.left == 0 && p.bottom == 0 && p.right == 0;
            const bool pairs = words && kx == 2 && sx == 2 && ky == sy && w % 4 == 0;
            const bool whole = words && ky == h && kx == w && oh == 1 && ow == 1;
            if (pairs && ky == 2 && ow % 2 == 0 && ow * 2 <= w && oh * 2 <= h &&
                reinterpret_cast<uintptr_t>(out) % 2 == 0)
            {
                pool2x2_u8_kernel<<<grid_for(n * ceil_div(oh, 7) * (ow / 2), 256), 256, 0, stream_of(stream)>>>(
                    (const uint8_t *)in, (uint8_t *)out, n, int(h), int(w), int(oh), int(ow));
                SPK_LAUNCHED();
                return;
            }
            const int64_t tile_bytes = whole ? 48 * 1024 : kPoolTileBytes;
            const int per_tile = int(std::max<int64_t>(1, std::min<int64_t>(tile_bytes / plane, n)));
            if (plane + 32 <= kPoolPlaneMax && per_tile * oh * ow < (int64_t(1) << 30))
            {
                const int smem = int(per_tile * plane + 32);  // + alignment shift and word over-reads
                const bool warp = ky * kx >= 64;
                auto k = pairs   ? pool_plane_kernel<T, 2>
                         : whole ? pool_plane_kernel<T, 3>
                         : warp  ? pool_plane_kernel<T, 1>
                                 : pool_plane_kernel<T, 0>;
                if (smem > 48 * 1024)
                    SPK_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
                int occ = 0;
                SPK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, 256, smem));
                const int64_t tiles = ceil_div(n, per_tile);
                const unsigned grid = unsigned(std::max<int64_t>(1, std::min<int64_t>(tiles, int64_t(sm_count()) * std::max(occ, 1))));
                k<<<grid, 256, smem, stream_of(stream)>>>((const T *)in, (T *)out, n, int(h), int(w), int(oh), int(ow),
                                                         int(ky), int(kx), int(sy), int(sx), int(p.top), int(p.left),
                                                         per_tile);
                SPK_LAUNCHED();
                return;
            }
            // the grid is capped, so thread indexes always fit in 32 bits
            const bool small = n * oh * ow < (int64_t(1) << 31) && n * h * w < (int64_t(1) << 31);
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
        if (type == SPK_F32)
        {
            // the widest vector that still leaves a block of threads per SM
            const int64_t waves2 = int64_t(sm_count()) * 256;
            const uintptr_t a = reinterpret_cast<uintptr_t>(data);
            const float th = scalar_to<float>(threshold);
            float *d = static_cast<float *>(data);
            if (x % 4 == 0 && a % 16 == 0 && b * x / 4 >= waves2)
                inhibit_f32v_kernel<4><<<grid_for(b * x / 4, 256), 256, 0, stream_of(stream)>>>(d, b, int(t), int(c),
                                                                                              x / 4, th);
            else if (x % 2 == 0 && a % 8 == 0 && b * x / 2 >= waves2)
                inhibit_f32v_kernel<2><<<grid_for(b * x / 2, 256), 256, 0, stream_of(stream)>>>(d, b, int(t), int(c),
                                                                                              x / 2, th);
            else
                inhibit_f32v_kernel<1><<<grid_for(b * x, 256), 256, 0, stream_of(stream)>>>(d, b, int(t), int(c), x,
                                                                                          th);
            SPK_LAUNCHED();
            return;
        }
        dispatch(type, [&](auto z) {
            using T = decltype(z);
            inhibit_kernel<T><<<grid_for(b * x, 128), 128, 0, stream_of(stream)>>>((T *)data, b, int(t), int(c), x,
                                                                                  scalar_to<T>(threshold));
            SPK_LAUNCHED();
        });
    });
}

}  // extern "C"
