// Spike x weight convolution: the plain FP32 SIMT path and the dispatcher of
// spk_conv (Core::conv of src/spyker/impl.h:224; semantics shape.cpp:35-50).
//
// out[n, o, y, x] = sum_{c, ky, kx} in[n, c, y*sy + ky - top, x*sx + kx - left]
//                                   * kernel[o, c, ky, kx]     (zero pad)
// N folds batch and time (the reference reshapes [B, T, C, H, W] to
// [B*T, C, H, W], opers.cpp:419-420).  Spikes are read as u8 directly: there
// is no F32 copy of the spike tensor (the reference casts it, opers.cpp:410).
#include <algorithm>

#include "common.cuh"
#include "conv_tc.cuh"

namespace spk
{
namespace
{
constexpr int kTileW = 32, kTileH = 8, kGroup = 16;

// CTA: one image, an 8x32 tile of output pixels, 16 output channels; one
// output pixel per thread with 16 FP32 accumulators.  Input channel by input
// channel, the receptive-field patch and the 16 weight slices are staged in
// shared memory.  Summation order: c, ky, kx (fmaf).
template <typename I>
__global__ void __launch_bounds__(kTileW *kTileH)
    conv_fp32_kernel(const I *__restrict__ in, const float *__restrict__ kernel, float *__restrict__ out, int cin,
                     int h, int w, int cout, int kh, int kw, int oh, int ow, int sy, int sx, int top, int left,
                     int tiles_x)
{
    extern __shared__ __align__(16) float smem[];
    const int ph = (kTileH - 1) * sy + kh, pw = (kTileW - 1) * sx + kw;
    float *patch = smem;                 // [ph][pw]
    float *wsm = smem + ph * pw;         // [kGroup][kh*kw]
    const int n = blockIdx.z;
    const int tile = blockIdx.x;
    const int ty0 = (tile / tiles_x) * kTileH, tx0 = (tile % tiles_x) * kTileW;
    const int o0 = blockIdx.y * kGroup;
    const int lx = threadIdx.x % kTileW, ly = threadIdx.x / kTileW;
    const int oy = ty0 + ly, ox = tx0 + lx;
    const int iy0 = ty0 * sy - top, ix0 = tx0 * sx - left;
    const int taps = kh * kw;
    float acc[kGroup];
#pragma unroll
    for (int g = 0; g < kGroup; ++g) acc[g] = 0.f;

    for (int c = 0; c < cin; ++c)
    {
        const I *plane = in + (int64_t(n) * cin + c) * h * w;
        for (int i = threadIdx.x; i < ph * pw; i += blockDim.x)
        {
            int yy = iy0 + i / pw, xx = ix0 + i % pw;
            patch[i] = (yy >= 0 && yy < h && xx >= 0 && xx < w) ? float(plane[int64_t(yy) * w + xx]) : 0.f;
        }
        for (int i = threadIdx.x; i < kGroup * taps; i += blockDim.x)
        {
            int g = i / taps, r = i % taps;
            wsm[i] = (o0 + g < cout) ? kernel[(int64_t(o0 + g) * cin + c) * taps + r] : 0.f;
        }
        __syncthreads();
        for (int ky = 0; ky < kh; ++ky)
            for (int kx = 0; kx < kw; ++kx)
            {
                float v = patch[(ly * sy + ky) * pw + lx * sx + kx];
                const float *wp = wsm + ky * kw + kx;
#pragma unroll
                for (int g = 0; g < kGroup; ++g) acc[g] = fmaf(v, wp[g * taps], acc[g]);
            }
        __syncthreads();
    }
    if (oy < oh && ox < ow)
    {
#pragma unroll
        for (int g = 0; g < kGroup; ++g)
            if (o0 + g < cout) out[((int64_t(n) * cout + o0 + g) * oh + oy) * ow + ox] = acc[g];
    }
}

template <typename I>
void launch_fp32(const I *in, const float *kernel, float *out, int64_t n, int64_t cin, int64_t h, int64_t w,
                 int64_t cout, int64_t kh, int64_t kw, int64_t oh, int64_t ow, int64_t sy, int64_t sx, Pad4 p,
                 cudaStream_t s)
{
    const int tiles_x = int(ceil_div(ow, kTileW)), tiles_y = int(ceil_div(oh, kTileH));
    const int ph = (kTileH - 1) * int(sy) + int(kh), pw = (kTileW - 1) * int(sx) + int(kw);
    const size_t smem = size_t(ph * pw + kGroup * kh * kw) * 4;
    SPK_REQUIRE(smem <= 200 * 1024, "kernel or stride too large for the FP32 path");
    SPK_REQUIRE(n <= 65535, "N (batch x time) is limited to 65535 per call on the FP32 path");
    auto k = conv_fp32_kernel<I>;
    SPK_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    dim3 grid(unsigned(tiles_x * tiles_y), unsigned(ceil_div(cout, kGroup)), unsigned(n));
    k<<<grid, kTileW * kTileH, smem, s>>>(in, kernel, out, int(cin), int(h), int(w), int(cout), int(kh), int(kw),
                                          int(oh), int(ow), int(sy), int(sx), int(p.top), int(p.left), tiles_x);
    SPK_LAUNCHED();
}
}  // namespace
}  // namespace spk

using namespace spk;

extern "C" {

size_t spk_conv_workspace(int64_t n, int64_t cin, int64_t h, int64_t w, int64_t cout, int64_t kh, int64_t kw,
                          int precision)
{
    if (precision == SPK_CONV_FP32) return 0;
    return conv_tc_workspace(n, cin, h, w, cout, kh, kw, precision);
}

spk_status spk_conv(const void *in, spk_dtype itype, const float *kernel, float *out, int64_t n, int64_t cin, int64_t h,
                    int64_t w, int64_t cout, int64_t kh, int64_t kw, int64_t sy, int64_t sx, const int64_t *pad4,
                    int precision, void *ws, size_t ws_bytes, spk_stream stream)
{
    return guarded([&] {
        Pad4 p = pad_of(pad4);
        SPK_REQUIRE(sy >= 1 && sx >= 1, "stride items are incorrect");
        SPK_REQUIRE(n >= 0 && cin >= 1 && cout >= 1 && kh >= 1 && kw >= 1 && h >= 1 && w >= 1, "invalid dims");
        const int64_t oh = (h + p.top + p.bottom - kh) / sy + 1, ow = (w + p.left + p.right - kw) / sx + 1;
        SPK_REQUIRE(h + p.top + p.bottom >= kh && w + p.left + p.right >= kw && oh > 0 && ow > 0,
                    "input and kernel shapes are not compatible");
        if (n == 0) return;
        cudaStream_t s = stream_of(stream);
        if (precision == SPK_CONV_FP32)
        {
            for (int64_t n0 = 0; n0 < n; n0 += 65535)
            {
                int64_t nn = std::min<int64_t>(65535, n - n0);
                float *o = out + n0 * cout * oh * ow;
                if (itype == SPK_U8)
                    launch_fp32<uint8_t>((const uint8_t *)in + n0 * cin * h * w, kernel, o, nn, cin, h, w, cout, kh,
                                         kw, oh, ow, sy, sx, p, s);
                else if (itype == SPK_F32)
                    launch_fp32<float>((const float *)in + n0 * cin * h * w, kernel, o, nn, cin, h, w, cout, kh, kw, oh,
                                       ow, sy, sx, p, s);
                else
                    throw Error(SPK_ERR_UNSUPPORTED, "conv input must be U8 or F32");
            }
            return;
        }
        SPK_REQUIRE(precision == SPK_CONV_BF16X2 || precision == SPK_CONV_BF16X3, "unknown precision");
        conv_tc(in, itype, kernel, out, n, cin, h, w, cout, kh, kw, sy, sx, p, oh, ow, precision, ws, ws_bytes, s);
    });
}

}  // extern "C"
