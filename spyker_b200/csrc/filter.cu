// DoG / Gabor / LoG filter banks (src/spyker/cpu/dog.cpp:40-94) and the FC
// product (src/spyker/cpu/fc.cpp:140-171).
//
// Filters: every plane is correlated with every kernel in FP64 (one exact
// sum per output, rounded once to F32, matching an exact convolution), then
//   DoG  : out[f] = max(g1[f] - g2[f], 0)                (F32 arithmetic)
//   Gabor: out[f] = g[f]
//   LoG  : d = g1[f] - g2[f]; out[f] = max(d, 0); out[F + f] = max(-d, 0)
// The rank code that follows orders these values, so they are produced
// exactly rather than to a tolerance.
#include "common.cuh"

namespace spk
{
namespace
{
__device__ __forceinline__ double correlate(const float *__restrict__ plane, int h, int w, const float *__restrict__ k,
                                            int kh, int kw, int y, int x, int top, int left)
{
    double acc = 0.0;
    for (int a = 0; a < kh; ++a)
    {
        int yy = y + a - top;
        if (yy < 0 || yy >= h) continue;
        for (int b = 0; b < kw; ++b)
        {
            int xx = x + b - left;
            if (xx < 0 || xx >= w) continue;
            acc = fma(double(plane[yy * w + xx]), double(k[a * kw + b]), acc);
        }
    }
    return acc;
}

__global__ void filter_kernel(int which, const float *__restrict__ in, const float *__restrict__ kernel,
                              float *__restrict__ out, int64_t n, int h, int w, int f, int kh, int kw, int oh, int ow,
                              int top, int left)
{
    const int64_t plane_out = int64_t(oh) * ow;
    const int64_t total = n * f * plane_out;
    const int fo = which == 2 ? 2 * f : f;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        const int x = int(k % ow), y = int((k / ow) % oh), q = int((k / plane_out) % f);
        const int64_t p = k / (plane_out * f);
        const float *plane = in + p * h * w;
        float *o = out + p * fo * plane_out + int64_t(y) * ow + x;
        if (which == 1)
        {
            o[int64_t(q) * plane_out] = float(correlate(plane, h, w, kernel + q * kh * kw, kh, kw, y, x, top, left));
        }
        else
        {
            float g1 = float(correlate(plane, h, w, kernel + q * kh * kw, kh, kw, y, x, top, left));
            float g2 = float(correlate(plane, h, w, kernel + (f + q) * kh * kw, kh, kw, y, x, top, left));
            float d = __fsub_rn(g1, g2);
            if (which == 0)
                o[int64_t(q) * plane_out] = (d < 0.f) ? 0.f : d;  // std::max(d, 0)
            else
            {
                float nd = -d;
                o[int64_t(q) * plane_out] = (d < 0.f) ? 0.f : d;
                o[int64_t(f + q) * plane_out] = (nd < 0.f) ? 0.f : nd;
            }
        }
    }
}

// The same filters with the plane staged in shared memory as FP64 (zero
// halo) and the kernels as FP64: a CTA takes rows [r0, r0 + rows) of one
// plane for every filter; a thread computes kXB neighbouring outputs of a
// row, reusing each loaded input for kXB products.  Every output is still
// one FMA chain over (a, b) in row-major order, so the result equals
// filter_kernel's bit for bit (a zero-halo term adds +-0 to the chain, which
// leaves it unchanged).
constexpr int kXB = 4, kMaxKw = 16;

__global__ void __launch_bounds__(256) filter_tiled_kernel(int which, const float *__restrict__ in,
                                                           const float *__restrict__ kernel, float *__restrict__ out,
                                                           int h, int w, int f, int kh, int kw, int oh, int ow, int top,
                                                           int left, int rows)
{
    extern __shared__ double fsm[];
    const int nk = which == 1 ? f : 2 * f, kk = kh * kw;
    const int sw = ow + kw - 1 + kXB;  // staged row width (zero beyond the plane)
    const int srows = rows + kh - 1;
    double *sk = fsm, *sp = fsm + nk * kk;
    const int64_t p = blockIdx.y;
    const int r0 = blockIdx.x * rows, nr = min(rows, oh - r0);
    const float *plane = in + p * h * w;
    for (int i = threadIdx.x; i < nk * kk; i += blockDim.x) sk[i] = double(kernel[i]);
    for (int i = threadIdx.x; i < srows * sw; i += blockDim.x)
    {
        const int yy = r0 + i / sw - top, xx = i % sw - left;
        sp[i] = (yy >= 0 && yy < h && xx >= 0 && xx < w) ? double(plane[yy * w + xx]) : 0.0;
    }
    __syncthreads();
    const int fo = which == 2 ? 2 * f : f;
    const int64_t plane_out = int64_t(oh) * ow;
    const int xg = (ow + kXB - 1) / kXB;
    for (int it = threadIdx.x; it < f * nr * xg; it += blockDim.x)
    {
        const int q = it / (nr * xg), rem = it - q * nr * xg, ry = rem / xg, x0 = (rem - ry * xg) * kXB;
        double g1[kXB], g2[kXB];
#pragma unroll
        for (int i = 0; i < kXB; ++i) g1[i] = 0.0, g2[i] = 0.0;
        const double *k1 = sk + q * kk, *k2 = sk + (f + q) * kk;
        for (int a = 0; a < kh; ++a)
        {
            const double *row = sp + (ry + a) * sw + x0;
            double v[kMaxKw + kXB - 1];
#pragma unroll
            for (int j = 0; j < kMaxKw + kXB - 1; ++j)
                if (j < kw + kXB - 1) v[j] = row[j];
#pragma unroll
            for (int bb = 0; bb < kMaxKw; ++bb)
            {
                if (bb >= kw) break;
                const double c1 = k1[a * kw + bb];
#pragma unroll
                for (int i = 0; i < kXB; ++i) g1[i] = fma(v[i + bb], c1, g1[i]);
                if (which != 1)
                {
                    const double c2 = k2[a * kw + bb];
#pragma unroll
                    for (int i = 0; i < kXB; ++i) g2[i] = fma(v[i + bb], c2, g2[i]);
                }
            }
        }
        float *o = out + p * fo * plane_out + int64_t(r0 + ry) * ow;
#pragma unroll
        for (int i = 0; i < kXB; ++i)
        {
            const int x = x0 + i;
            if (x >= ow) break;
            if (which == 1)
                o[int64_t(q) * plane_out + x] = float(g1[i]);
            else
            {
                const float d = __fsub_rn(float(g1[i]), float(g2[i]));
                o[int64_t(q) * plane_out + x] = (d < 0.f) ? 0.f : d;
                if (which == 2)
                {
                    const float nd = -d;
                    o[int64_t(f + q) * plane_out + x] = (nd < 0.f) ? 0.f : nd;
                }
            }
        }
    }
}

template <typename I>
__global__ void fc_kernel(const I *__restrict__ in, const float *__restrict__ kernel, float *__restrict__ out, int64_t r,
                          int ni, int no, int sign)
{
    const int64_t total = r * no;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t row = k / no;
        const int o = int(k % no);
        const I *a = in + row * ni;
        const float *wr = kernel + int64_t(o) * ni;
        float acc = 0.f;
        for (int i = 0; i < ni; ++i)
        {
            float wv = wr[i];
            if (sign) wv = wv > 0.f ? 1.f : (wv < 0.f ? -1.f : 0.f);
            acc = fmaf(float(a[i]), wv, acc);
        }
        out[k] = acc;
    }
}
}  // namespace
}  // namespace spk

using namespace spk;

extern "C" {

spk_status spk_filter(int which, const float *in, const float *kernel, float *out, int64_t n, int64_t h, int64_t w,
                      int64_t f, int64_t kh, int64_t kw, int64_t oh, int64_t ow, const int64_t *pad4,
                      spk_stream stream)
{
    return guarded([&] {
        Pad4 p = pad_of(pad4);
        SPK_REQUIRE(which >= 0 && which <= 2, "unknown filter kind");
        SPK_REQUIRE(n >= 0 && h >= 1 && w >= 1 && f >= 1 && kh >= 1 && kw >= 1, "invalid dims");
        SPK_REQUIRE(oh == h + p.top + p.bottom - kh + 1 && ow == w + p.left + p.right - kw + 1 && oh > 0 && ow > 0,
                    "input and kernel shapes are not compatible");
        if (n == 0) return;
        // tiled: as many output rows per CTA as fit 48 KB of FP64 staging
        const int64_t nk = which == 1 ? f : 2 * f, sw = ow + kw - 1 + kXB;
        const int64_t avail = (48 * 1024) / 8 - nk * kh * kw;
        const int64_t rows = std::min<int64_t>(oh, avail / sw - (kh - 1));
        if (kw <= kMaxKw && rows >= 1 && n <= 65535 && h * w < (int64_t(1) << 31))
        {
            const size_t smem = size_t(nk * kh * kw + (rows + kh - 1) * sw) * 8;
            filter_tiled_kernel<<<dim3(unsigned(ceil_div(oh, rows)), unsigned(n)), 256, smem, stream_of(stream)>>>(
                which, in, kernel, out, int(h), int(w), int(f), int(kh), int(kw), int(oh), int(ow), int(p.top),
                int(p.left), int(rows));
        }
        else
            filter_kernel<<<grid_for(n * f * oh * ow, 256), 256, 0, stream_of(stream)>>>(
                which, in, kernel, out, n, int(h), int(w), int(f), int(kh), int(kw), int(oh), int(ow), int(p.top),
                int(p.left));
        SPK_LAUNCHED();
    });
}

spk_status spk_fc(const void *in, spk_dtype itype, const float *kernel, float *out, int64_t r, int64_t ni, int64_t no,
                  int sign, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(r >= 0 && ni >= 1 && no >= 1, "invalid dims");
        if (r == 0) return;
        if (itype == SPK_U8)
            fc_kernel<uint8_t><<<grid_for(r * no, 256), 256, 0, stream_of(stream)>>>((const uint8_t *)in, kernel, out,
                                                                                   r, int(ni), int(no), sign);
        else if (itype == SPK_F32)
            fc_kernel<float><<<grid_for(r * no, 256), 256, 0, stream_of(stream)>>>((const float *)in, kernel, out, r,
                                                                                 int(ni), int(no), sign);
        else
            throw Error(SPK_ERR_UNSUPPORTED, "fc input must be U8 or F32");
        SPK_LAUNCHED();
    });
}

}  // extern "C"
