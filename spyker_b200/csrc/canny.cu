// Canny edge detection (cpu/canny.cpp:9-214) and two-level quantize
// (cpu/fire.cpp:116-131) on the GPU.
//
// Canny of a u8 image [H, W], as the reference computes it:
//   1 blur:      5x5 Gaussian table (F32 constants), zero pad 2, FP64 sums
//                rounded once to F32 (the FP64 conv of the reference build)
//   2 gradient:  two 5x5 integer kernels on the blur, FP64 sums -> gx, gy
//   3 magnitude: sqrt(gx gx + gy gy) in F32, times 255 / (image max - 1e-5);
//                direction atan2(gy, gx) in F32, in degrees, + 180 if < 0
//   4 thinning:  interior pixels keep their normalised magnitude (truncated
//                to u8) when it is >= both neighbours along the direction
//                (4 bins at 22.5 / 67.5 / 112.5 / 157.5 degrees), else 0;
//                borders 0; then u8 * 255 / (image max - 1e-5), truncated
//   5 classes:   2 (strong) if high <= v, 1 (weak) if low <= v, else 0
//   6 one pass:  an interior weak pixel next to a strong one (8 neighbours,
//                classes of step 5) becomes strong
//   7 output:    max(strong ? 255 : 0, v of step 4)
// Four launches (after zeroing the maxima): blur; gradient + magnitude +
// direction + the image's max magnitude; thinning + the image's max thinned
// value; classes, one-pass hysteresis and output.  The maxima are atomics on the values' bit
// patterns (non-negative floats order as their bits).
#include "common.cuh"

namespace spk
{
namespace
{
constexpr int kTile = 16, kHalo = 2, kSpan = kTile + 2 * kHalo;

__constant__ float c_gauss[25] = {
    0.0030f, 0.0133f, 0.0219f, 0.0133f, 0.0030f,  //
    0.0133f, 0.0596f, 0.0983f, 0.0596f, 0.0133f,  //
    0.0219f, 0.0983f, 0.1621f, 0.0983f, 0.0219f,  //
    0.0133f, 0.0596f, 0.0983f, 0.0596f, 0.0133f,  //
    0.0030f, 0.0133f, 0.0219f, 0.0133f, 0.0030f,  //
};
__constant__ float c_gx[25] = {
    -1, -1, 0, 1, 1,  //
    -2, -2, 0, 2, 2,  //
    -3, -6, 0, 6, 3,  //
    -2, -2, 0, 2, 2,  //
    -1, -1, 0, 1, 1,  //
};
__constant__ float c_gy[25] = {
    1,  2,  3,  2,  1,   //
    1,  2,  6,  2,  1,   //
    0,  0,  0,  0,  0,   //
    -1, -2, -6, -2, -1,  //
    -1, -2, -3, -2, -1,  //
};

// A 16 x 16 output tile per CTA with its 2-pixel zero halo in shared memory;
// each output is an FP64 sum over the 5 x 5 taps in row-major order, every
// product and sum rounded separately (as the reference build's conv
// computes it), rounded once to F32.
template <typename T>
__device__ __forceinline__ void load_tile(const T *__restrict__ img, int h, int w, int y0, int x0,
                                          double (&tile)[kSpan][kSpan + 1])
{
    for (int i = threadIdx.x; i < kSpan * kSpan; i += blockDim.x)
    {
        const int ty = i / kSpan, tx = i % kSpan, y = y0 + ty - kHalo, x = x0 + tx - kHalo;
        tile[ty][tx] = (y >= 0 && y < h && x >= 0 && x < w) ? double(img[int64_t(y) * w + x]) : 0.0;
    }
}

__global__ void __launch_bounds__(256) canny_blur_kernel(const uint8_t *__restrict__ in, float *__restrict__ blur,
                                                         int h, int w)
{
    __shared__ double tile[kSpan][kSpan + 1];
    const int64_t img = blockIdx.z;
    const int y0 = blockIdx.y * kTile, x0 = blockIdx.x * kTile;
    load_tile(in + img * h * w, h, w, y0, x0, tile);
    __syncthreads();
    const int ly = threadIdx.x / kTile, lx = threadIdx.x % kTile, y = y0 + ly, x = x0 + lx;
    if (y >= h || x >= w) return;
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 5; ++i)
#pragma unroll
        for (int j = 0; j < 5; ++j) s = __dadd_rn(s, __dmul_rn(tile[ly + i][lx + j], double(c_gauss[i * 5 + j])));
    blur[img * h * w + int64_t(y) * w + x] = float(s);
}

__global__ void __launch_bounds__(256) canny_grad_kernel(const float *__restrict__ blur, float *__restrict__ mag,
                                                         float *__restrict__ ang, unsigned *__restrict__ mmax, int h,
                                                         int w)
{
    __shared__ double tile[kSpan][kSpan + 1];
    const int64_t img = blockIdx.z;
    const int y0 = blockIdx.y * kTile, x0 = blockIdx.x * kTile;
    load_tile(blur + img * h * w, h, w, y0, x0, tile);
    __syncthreads();
    const int ly = threadIdx.x / kTile, lx = threadIdx.x % kTile, y = y0 + ly, x = x0 + lx;
    float m = 0.f;
    if (y < h && x < w)
    {
        double sx = 0.0, sy = 0.0;
#pragma unroll
        for (int i = 0; i < 5; ++i)
#pragma unroll
            for (int j = 0; j < 5; ++j)
            {
                const double v = tile[ly + i][lx + j];
                sx = __dadd_rn(sx, __dmul_rn(v, double(c_gx[i * 5 + j])));
                sy = __dadd_rn(sy, __dmul_rn(v, double(c_gy[i * 5 + j])));
            }
        const float gx = float(sx), gy = float(sy);
        // x x + y y contracted as the reference's -O3 FMA build does it:
        // fma(x, x, y y)
        m = __fsqrt_rn(__fmaf_rn(gx, gx, __fmul_rn(gy, gy)));
        const int64_t o = img * h * w + int64_t(y) * w + x;
        mag[o] = m;
        ang[o] = atan2f(gy, gx);
    }
    // warp max, one atomic per warp (magnitudes are >= 0, so their bit
    // patterns order as the values)
    const unsigned bits = __reduce_max_sync(0xffffffffu, __float_as_uint(m));
    if ((threadIdx.x & 31) == 0) atomicMax(mmax + img, bits);
}

// Normalised magnitude: v * (255 / (max - 1e-5)) in F32 (cpu/canny.cpp:9-14).
__device__ __forceinline__ float norm_scale(float mx) { return __fdiv_rn(255.0f, __fsub_rn(mx, 1e-5f)); }

__device__ __forceinline__ uint8_t f2u8(float v)
{
    // float -> u8 as the x86-64 build lowers it: truncate to int32, low byte
    if (!(v > -2147483648.0f && v < 2147483648.0f)) return 0;
    return uint8_t(uint32_t(__float2int_rz(v)));
}

__global__ void canny_thin_kernel(const float *__restrict__ mag, const float *__restrict__ ang,
                                  const unsigned *__restrict__ mmax, uint8_t *__restrict__ thin,
                                  unsigned *__restrict__ tmax, int h, int w)
{
    const int64_t img = blockIdx.y;
    const int64_t hw = int64_t(h) * w;
    const float sc = norm_scale(__uint_as_float(mmax[img]));
    const float *m = mag + img * hw;
    unsigned best = 0;
    for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < hw; p += int64_t(gridDim.x) * blockDim.x)
    {
        const int i = int(p / w), j = int(p - int64_t(i) * w);
        uint8_t r = 0;
        if (i >= 1 && i < h - 1 && j >= 1 && j < w - 1)
        {
            float a = float(double(ang[img * hw + p]) * (180.0 / 3.14159265358979323846));
            if (a < 0) a = __fadd_rn(a, 180.0f);
            int di, dj;  // neighbour 1 at (i + di, j + dj), neighbour 2 opposite
            if (a < 22.5f || 157.5f <= a)
                di = 0, dj = 1;
            else if (a < 67.5f)
                di = 1, dj = -1;
            else if (a < 112.5f)
                di = 1, dj = 0;
            else
                di = -1, dj = -1;
            const float v = __fmul_rn(m[p], sc);
            const float v1 = __fmul_rn(m[int64_t(i + di) * w + j + dj], sc);
            const float v2 = __fmul_rn(m[int64_t(i - di) * w + j - dj], sc);
            r = (v >= v1 && v >= v2) ? f2u8(v) : 0;
        }
        thin[img * hw + p] = r;
        best = max(best, unsigned(r));
    }
    best = __reduce_max_sync(0xffffffffu, best);
    if ((threadIdx.x & 31) == 0) atomicMax(tmax + img, best);
}

__device__ __forceinline__ uint8_t thin_norm(uint8_t t, float sc) { return f2u8(__fmul_rn(float(t), sc)); }

__device__ __forceinline__ int canny_class(uint8_t v, int low, int high)
{
    return high <= v ? 2 : (low <= v ? 1 : 0);
}

__global__ void canny_final_kernel(const uint8_t *__restrict__ thin, const unsigned *__restrict__ tmax,
                                   uint8_t *__restrict__ out, int h, int w, int low, int high)
{
    const int64_t img = blockIdx.y;
    const int64_t hw = int64_t(h) * w;
    const float sc = norm_scale(float(tmax[img]));
    const uint8_t *t = thin + img * hw;
    for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < hw; p += int64_t(gridDim.x) * blockDim.x)
    {
        const int i = int(p / w), j = int(p - int64_t(i) * w);
        const uint8_t v = thin_norm(t[p], sc);
        int c = canny_class(v, low, high);
        if (c == 1 && i >= 1 && i < h - 1 && j >= 1 && j < w - 1)
        {
            for (int di = -1; di <= 1 && c == 1; ++di)
                for (int dj = -1; dj <= 1; ++dj)
                    if ((di | dj) != 0 && canny_class(thin_norm(t[int64_t(i + di) * w + j + dj], sc), low, high) == 2)
                    {
                        c = 2;
                        break;
                    }
        }
        const uint8_t s = c == 2 ? 255 : 0;
        out[img * hw + p] = s > v ? s : v;
    }
}

template <typename T>
__global__ void quantize_kernel(T *__restrict__ data, int64_t n, T lower, T middle, T upper)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        data[i] = data[i] < middle ? lower : upper;
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }
}  // namespace
}  // namespace spk

using namespace spk;

extern "C" {

int64_t spk_canny_workspace(int64_t n, int64_t h, int64_t w)
{
    if (n <= 0 || h <= 0 || w <= 0) return 0;
    const size_t px = size_t(n) * h * w;
    return int64_t(align256(px * 4) * 3 + align256(px) + align256(size_t(n) * 8));
}

spk_status spk_canny(const uint8_t *in, uint8_t *out, int64_t n, int64_t h, int64_t w, double low, double high,
                     void *ws, int64_t ws_bytes, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(n >= 0 && h >= 0 && w >= 0, "invalid dims");
        if (n * h * w == 0) return;
        SPK_REQUIRE(in && out && ws, "null pointer");
        SPK_REQUIRE(ws_bytes >= spk_canny_workspace(n, h, w), "workspace too small");
        SPK_REQUIRE(n <= 65535 && h < (int64_t(1) << 30) && w < (int64_t(1) << 30) &&
                        ceil_div(h, kTile) <= 65535 && ceil_div(w, kTile) <= INT32_MAX,
                    "image batch too large for one call");
        const size_t px = size_t(n) * h * w;
        char *p = static_cast<char *>(ws);
        float *blur = reinterpret_cast<float *>(p);
        float *mag = reinterpret_cast<float *>(p + align256(px * 4));
        float *ang = reinterpret_cast<float *>(p + 2 * align256(px * 4));
        uint8_t *thin = reinterpret_cast<uint8_t *>(p + 3 * align256(px * 4));
        unsigned *maxes = reinterpret_cast<unsigned *>(p + 3 * align256(px * 4) + align256(px));
        cudaStream_t s = stream_of(stream);
        SPK_CUDA(cudaMemsetAsync(maxes, 0, size_t(n) * 8, s));
        const dim3 tiles(unsigned(ceil_div(w, kTile)), unsigned(ceil_div(h, kTile)), unsigned(n));
        canny_blur_kernel<<<tiles, 256, 0, s>>>(in, blur, int(h), int(w));
        SPK_LAUNCHED();
        canny_grad_kernel<<<tiles, 256, 0, s>>>(blur, mag, ang, maxes, int(h), int(w));
        SPK_LAUNCHED();
        const int64_t hw = h * w;
        const dim3 per(unsigned(std::min<int64_t>(ceil_div(hw, 256), 1024)), unsigned(n));
        canny_thin_kernel<<<per, 256, 0, s>>>(mag, ang, maxes, thin, maxes + n, int(h), int(w));
        SPK_LAUNCHED();
        const int lo = scalar_to<uint8_t>(low), hi = scalar_to<uint8_t>(high);
        canny_final_kernel<<<per, 256, 0, s>>>(thin, maxes + n, out, int(h), int(w), lo, hi);
        SPK_LAUNCHED();
    });
}

spk_status spk_quantize(void *data, spk_dtype type, int64_t n, double lower, double middle, double upper,
                        spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(n >= 0, "negative size");
        if (n == 0) return;
        SPK_REQUIRE(data != nullptr, "null data");
        dispatch(type, [&](auto z) {
            using T = decltype(z);
            quantize_kernel<T><<<grid_for(n, 256), 256, 0, stream_of(stream)>>>(
                static_cast<T *>(data), n, scalar_to<T>(lower), scalar_to<T>(middle), scalar_to<T>(upper));
            SPK_LAUNCHED();
        });
    });
}

}  // extern "C"
