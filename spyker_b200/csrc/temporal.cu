// Temporal backprop through first-spike layers.
//
// A rank-coded layer maps input first-spike times t_in to output first-spike
// times t_out (conv or fc over cumulative spikes, then the first step whose
// potential exceeds the threshold).  The reference trains such a layer with
// the rule of its fc backward (src/spyker/cpu/backprop.cpp:105-160):
//     select[j, i] = (t_in[i] < t_out[j]) * grad[j]            (:116-119)
//     kernel      -= lrate * select                            (:121-124)
//     next[i]      = sum_j kernel[j, i] * select[j, i]         (:140-144)
// with grad the target rule's (desired - actual) / T (:40-52).  Here the rule
// is written for a weight shared over the output positions of a convolution
// (the fc layer is the 1x1 case) and as a derivative in autograd's sign
// convention (grad_out = dL/dt_out = -grad):
//     dL/dW[z, c, ky, kx] = -sum_{b, oy, ox} grad_out[b, z, oy, ox]
//                            * [t_in[b, c, iy, ix] < t_out[b, z, oy, ox]]
//     dL/dt_in[b, c, iy, ix] = sum_{z, ky, kx} W[z, c, ky, kx] * grad_out[b, z, oy, ox]
//                            * [t_in[b, c, iy, ix] < t_out[b, z, oy, ox]]
// with (iy, ix) = (oy * sy - top + ky, ox * sx - left + kx); padding never
// spikes.  dL/dW is the exact derivative of the potential-level loss
// L = sum grad_out' * V(t_out - 1) (the potential one step before the output
// spike, times held fixed), which `spk_fst_conv_prespike` evaluates in FP64.
// Only first-spike times are kept between forward and backward (T times less
// memory than the potentials); nothing here needs the potentials.
#include "common.cuh"

namespace spk
{
namespace
{
__device__ __forceinline__ int floor_div(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

struct Geo
{
    int h, w, oh, ow, kh, kw, sy, sx, top, left;
};

// Earliest spike of each window (pool of cumulative spikes); padding never
// spikes (`never` = T).
__global__ void fst_pool_kernel(const float *__restrict__ in, float *__restrict__ out, int64_t planes, Geo g,
                                float never)
{
    const int64_t total = planes * g.oh * g.ow;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x)
    {
        const int ox = int(i % g.ow), oy = int((i / g.ow) % g.oh);
        const float *src = in + (i / (int64_t(g.oh) * g.ow)) * g.h * g.w;
        float m = never;
        for (int dy = 0; dy < g.kh; ++dy)
        {
            const int iy = oy * g.sy - g.top + dy;
            if (iy < 0 || iy >= g.h) continue;
            for (int dx = 0; dx < g.kw; ++dx)
            {
                const int ix = ox * g.sx - g.left + dx;
                if (ix >= 0 && ix < g.w) m = fminf(m, src[iy * g.w + ix]);
            }
        }
        out[i] = m;
    }
}

// The gradient of a window goes to its earliest in-range input, the first in
// raster order on ties (as a first-index argmax of the spikes would pick).
// One thread per input element sums the windows it wins: deterministic.
__global__ void fst_pool_backward_kernel(const float *__restrict__ in, const float *__restrict__ go,
                                         float *__restrict__ gi, int64_t planes, Geo g)
{
    const int64_t total = planes * g.h * g.w;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x)
    {
        const int ix = int(i % g.w), iy = int((i / g.w) % g.h);
        const int64_t pl = i / (int64_t(g.h) * g.w);
        const float *src = in + pl * g.h * g.w;
        const float *gp = go + pl * g.oh * g.ow;
        const int oy0 = max(0, -floor_div(-(iy + g.top - g.kh + 1), g.sy)), oy1 = min(g.oh - 1, floor_div(iy + g.top, g.sy));
        const int ox0 = max(0, -floor_div(-(ix + g.left - g.kw + 1), g.sx)), ox1 = min(g.ow - 1, floor_div(ix + g.left, g.sx));
        float acc = 0.f;
        for (int oy = oy0; oy <= oy1; ++oy)
            for (int ox = ox0; ox <= ox1; ++ox)
            {
                float best = INFINITY;
                int bi = -1;
                for (int dy = 0; dy < g.kh; ++dy)
                {
                    const int y = oy * g.sy - g.top + dy;
                    if (y < 0 || y >= g.h) continue;
                    for (int dx = 0; dx < g.kw; ++dx)
                    {
                        const int x = ox * g.sx - g.left + dx;
                        if (x < 0 || x >= g.w) continue;
                        const float v = src[y * g.w + x];
                        if (v < best) best = v, bi = y * g.w + x;
                    }
                }
                if (bi == iy * g.w + ix) acc += gp[oy * g.ow + ox];
            }
        gi[i] = acc;
    }
}

// dL/dt_in.  CTA = (sample, block of cb channels); thread items = (channel,
// input pixel), up to kItems per thread; the output times, gradients and
// weights of zc maps at a time are staged in shared memory.  Per item the
// maps and taps are summed in a fixed order (deterministic).  UNIT: stride 1
// (no divisibility tests).
constexpr int kItems = 4, kGiThreads = 256;

template <bool UNIT>
__global__ void __launch_bounds__(kGiThreads) fst_conv_grad_in_kernel(
    const float *__restrict__ tin, const float *__restrict__ kern, const float *__restrict__ tout,
    const float *__restrict__ go, float *__restrict__ gi, int cin, int cout, Geo g, int cb, int zc)
{
    extern __shared__ float sm[];
    const int P = g.oh * g.ow, HW = g.h * g.w, KK = g.kh * g.kw;
    float *s_to = sm, *s_go = sm + zc * P, *s_w = sm + 2 * zc * P;  // [zc][P], [zc][P], [zc][cb][KK]
    const int64_t b = blockIdx.y;
    const int c0 = blockIdx.x * cb;
    const int nc = min(cb, cin - c0), items = nc * HW;
    float acc[kItems], ti[kItems];
    int ic[kItems], iy[kItems], ix[kItems];
#pragma unroll
    for (int u = 0; u < kItems; ++u)
    {
        const int it = threadIdx.x + u * kGiThreads;
        acc[u] = 0.f;
        ic[u] = -1;
        if (it < items)
        {
            ic[u] = it / HW;
            const int q = it - ic[u] * HW;
            iy[u] = q / g.w, ix[u] = q - iy[u] * g.w;
            ti[u] = tin[(b * cin + c0 + ic[u]) * HW + q];
        }
    }
    for (int z0 = 0; z0 < cout; z0 += zc)
    {
        const int nz = min(zc, cout - z0);
        __syncthreads();
        for (int i = threadIdx.x; i < nz * P; i += kGiThreads)
        {
            const int64_t src = (b * cout + z0) * P + i;
            s_to[i] = tout[src];
            s_go[i] = go[src];
        }
        for (int i = threadIdx.x; i < nz * nc * KK; i += kGiThreads)
        {
            const int zz = i / (nc * KK), r = i - zz * nc * KK, cl = r / KK, k = r - cl * KK;
            s_w[(zz * cb + cl) * KK + k] = kern[((int64_t(z0 + zz) * cin) + c0 + cl) * KK + k];
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < kItems; ++u)
        {
            if (ic[u] < 0) continue;
            for (int zz = 0; zz < nz; ++zz)
            {
                const float *wz = s_w + (zz * cb + ic[u]) * KK;
                const float *to = s_to + zz * P, *gz = s_go + zz * P;
                for (int ky = 0; ky < g.kh; ++ky)
                {
                    int oy = iy[u] + g.top - ky;
                    if (UNIT)
                    {
                        if (oy < 0 || oy >= g.oh) continue;
                    }
                    else
                    {
                        if (oy < 0 || oy % g.sy) continue;
                        oy /= g.sy;
                        if (oy >= g.oh) continue;
                    }
                    for (int kx = 0; kx < g.kw; ++kx)
                    {
                        int ox = ix[u] + g.left - kx;
                        if (UNIT)
                        {
                            if (ox < 0 || ox >= g.ow) continue;
                        }
                        else
                        {
                            if (ox < 0 || ox % g.sx) continue;
                            ox /= g.sx;
                            if (ox >= g.ow) continue;
                        }
                        const int p = oy * g.ow + ox;
                        if (ti[u] < to[p]) acc[u] = __fmaf_rn(wz[ky * g.kw + kx], gz[p], acc[u]);
                    }
                }
            }
        }
    }
#pragma unroll
    for (int u = 0; u < kItems; ++u)
        if (ic[u] >= 0) gi[(b * cin + c0 + ic[u]) * HW + iy[u] * g.w + ix[u]] = acc[u];
}

// dL/dW, first pass.  CTA = (map z, group of sb samples, block of up to 2048
// weight elements).  Work pairs =
// (weight element, slice of the output rows): `slices` row slices per weight
// so that the pairs fill the CTA's threads; each pair walks its rows and
// columns (no divisions) and sums in FP64; the slices are then added in
// order.  The sample's input times (when they fit) and a chunk of rows of
// the map's output times and gradients are staged in shared memory.
// Per-group partials part[group][z][Cin*KH*KW]; the second pass adds the
// groups in order (deterministic).
constexpr int kGwThreads = 256, kGwRounds = 8;

__global__ void __launch_bounds__(kGwThreads) fst_conv_grad_w_kernel(const float *__restrict__ tin,
                                                                      const float *__restrict__ tout,
                                                                      const float *__restrict__ go,
                                                                      double *__restrict__ part, int64_t b, int cin,
                                                                      int cout, Geo g, int sb, int slices, int rows,
                                                                      int stage_in)
{
    extern __shared__ double gsm[];
    const int z = blockIdx.x, grp = blockIdx.y;
    const int KK = g.kh * g.kw, WK = cin * KK, HW = g.h * g.w;
    const int wk0 = blockIdx.z * (kGwThreads * kGwRounds), wkn = min(WK - wk0, kGwThreads * kGwRounds / slices);
    const int pairs = wkn * slices;
    double *s_red = gsm;                                              // [pairs]
    float *s_to = reinterpret_cast<float *>(s_red + pairs);          // [rows * ow]
    float *s_go = s_to + rows * g.ow;                                 // [rows * ow]
    float *s_in = s_go + rows * g.ow;                                 // [cin * HW] when staged
    const int64_t s0 = int64_t(grp) * sb, s1 = min(b, s0 + sb);
    double acc[kGwRounds];
    int pc[kGwRounds], pky[kGwRounds], pkx[kGwRounds], psl[kGwRounds];
#pragma unroll
    for (int r = 0; r < kGwRounds; ++r)
    {
        acc[r] = 0.0;
        const int pi = threadIdx.x + r * kGwThreads;
        psl[r] = -1;
        if (pi < pairs)
        {
            const int wk = wk0 + pi % wkn;
            psl[r] = pi / wkn;
            pc[r] = wk / KK, pky[r] = (wk % KK) / g.kw, pkx[r] = wk % g.kw;
        }
    }
    for (int64_t s = s0; s < s1; ++s)
    {
        if (stage_in)
        {
            __syncthreads();
            for (int i = threadIdx.x; i < cin * HW; i += kGwThreads) s_in[i] = tin[s * cin * HW + i];
        }
        for (int oy0 = 0; oy0 < g.oh; oy0 += rows)
        {
            const int nr = min(rows, g.oh - oy0);
            __syncthreads();
            for (int i = threadIdx.x; i < nr * g.ow; i += kGwThreads)
            {
                const int64_t src = (s * cout + z) * int64_t(g.oh) * g.ow + int64_t(oy0) * g.ow + i;
                s_to[i] = tout[src];
                s_go[i] = go[src];
            }
            __syncthreads();
#pragma unroll
            for (int r = 0; r < kGwRounds; ++r)
            {
                if (psl[r] < 0) continue;
                const float *ti = stage_in ? s_in + pc[r] * HW : tin + (s * cin + pc[r]) * HW;
                // rows oy0 + j with j = slice index mod slices
                for (int j = (psl[r] - oy0 % slices + slices) % slices; j < nr; j += slices)
                {
                    const int iy = (oy0 + j) * g.sy - g.top + pky[r];
                    if (iy < 0 || iy >= g.h) continue;
                    const float *trow = ti + iy * g.w;
                    const float *to = s_to + j * g.ow, *gr = s_go + j * g.ow;
                    int ix = pkx[r] - g.left;
                    for (int ox = 0; ox < g.ow; ++ox, ix += g.sx)
                        if (ix >= 0 && ix < g.w && trow[ix] < to[ox]) acc[r] += double(gr[ox]);
                }
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kGwRounds; ++r)
        if (psl[r] >= 0) s_red[threadIdx.x + r * kGwThreads] = acc[r];
    __syncthreads();
    for (int w = threadIdx.x; w < wkn; w += kGwThreads)
    {
        double sum = 0.0;
        for (int q = 0; q < slices; ++q) sum += s_red[q * wkn + w];
        part[(int64_t(grp) * cout + z) * WK + wk0 + w] = sum;
    }
}

__global__ void fst_conv_grad_w_reduce_kernel(const double *__restrict__ part, float *__restrict__ gk, int64_t n,
                                              int groups)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    {
        double s = 0.0;
        for (int q = 0; q < groups; ++q) s += part[int64_t(q) * n + i];
        gk[i] = float(-s);
    }
}

// Potential one step before each output spike, in FP64:
//   V[b, z, oy, ox] = sum_{c, ky, kx} W * [t_in < t_out]   (padding never spikes)
__global__ void fst_conv_prespike_kernel(const float *__restrict__ tin, const float *__restrict__ kern,
                                         const float *__restrict__ tout, double *__restrict__ out, int64_t b, int cin,
                                         int cout, Geo g)
{
    const int64_t P = int64_t(g.oh) * g.ow, total = b * cout * P;
    const int KK = g.kh * g.kw;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t s = i / (cout * P);
        const int z = int((i / P) % cout), p = int(i % P), oy = p / g.ow, ox = p - oy * g.ow;
        const float to = tout[i];
        double acc = 0.0;
        for (int c = 0; c < cin; ++c)
        {
            const float *ti = tin + (s * cin + c) * g.h * g.w;
            const float *wk = kern + (int64_t(z) * cin + c) * KK;
            for (int ky = 0; ky < g.kh; ++ky)
            {
                const int iy = oy * g.sy - g.top + ky;
                if (iy < 0 || iy >= g.h) continue;
                for (int kx = 0; kx < g.kw; ++kx)
                {
                    const int ix = ox * g.sx - g.left + kx;
                    if (ix >= 0 && ix < g.w && ti[iy * g.w + ix] < to) acc += double(wk[ky * g.kw + kx]);
                }
            }
        }
        out[i] = acc;
    }
}

Geo geometry(int64_t h, int64_t w, int64_t oh, int64_t ow, int64_t kh, int64_t kw, const int64_t *stride2,
             const int64_t *pad4)
{
    SPK_REQUIRE(stride2 != nullptr, "stride pointer is null");
    SPK_REQUIRE(stride2[0] >= 1 && stride2[1] >= 1, "stride items are incorrect");
    const Pad4 p = pad_of(pad4);
    SPK_REQUIRE(h >= 1 && w >= 1 && kh >= 1 && kw >= 1, "invalid dims");
    SPK_REQUIRE((h + p.top + p.bottom - kh) / stride2[0] + 1 == oh && (w + p.left + p.right - kw) / stride2[1] + 1 == ow &&
                    oh >= 1 && ow >= 1,
                "output shape does not match the input, kernel, stride and pad");
    SPK_REQUIRE(h * w < (int64_t(1) << 31) && oh * ow < (int64_t(1) << 31) && kh * kw < (1 << 20),
                "planes are too large");
    return Geo{int(h), int(w), int(oh), int(ow), int(kh), int(kw), int(stride2[0]), int(stride2[1]), int(p.top),
               int(p.left)};
}

constexpr int kGwSamples = 8;  // samples per first-pass CTA of dL/dW
}  // namespace
}  // namespace spk

using namespace spk;

extern "C" {

spk_status spk_fst_pool(const float *in, int64_t b, int64_t c, int64_t h, int64_t w, float *out, int64_t oh,
                        int64_t ow, const int64_t *kernel2, const int64_t *stride2, const int64_t *pad4, double time,
                        spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(kernel2 != nullptr, "kernel pointer is null");
        const Geo g = geometry(h, w, oh, ow, kernel2[0], kernel2[1], stride2, pad4);
        SPK_REQUIRE(b >= 0 && c >= 1, "invalid dims");
        if (b == 0) return;
        fst_pool_kernel<<<grid_for(b * c * oh * ow, 256), 256, 0, stream_of(stream)>>>(in, out, b * c, g,
                                                                                         float(time));
        SPK_LAUNCHED();
    });
}

spk_status spk_fst_pool_backward(const float *in, int64_t b, int64_t c, int64_t h, int64_t w, const float *grad_out,
                                 int64_t oh, int64_t ow, const int64_t *kernel2, const int64_t *stride2,
                                 const int64_t *pad4, float *grad_in, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(kernel2 != nullptr, "kernel pointer is null");
        const Geo g = geometry(h, w, oh, ow, kernel2[0], kernel2[1], stride2, pad4);
        SPK_REQUIRE(b >= 0 && c >= 1, "invalid dims");
        if (b == 0) return;
        fst_pool_backward_kernel<<<grid_for(b * c * h * w, 256), 256, 0, stream_of(stream)>>>(in, grad_out, grad_in,
                                                                                                b * c, g);
        SPK_LAUNCHED();
    });
}

size_t spk_fst_conv_backward_workspace(int64_t b, int64_t cin, int64_t cout, int64_t kh, int64_t kw)
{
    if (b <= 0 || cin <= 0 || cout <= 0 || kh <= 0 || kw <= 0) return 0;
    return size_t(ceil_div(b, kGwSamples)) * size_t(cout) * size_t(cin * kh * kw) * sizeof(double);
}

spk_status spk_fst_conv_backward(const float *t_in, int64_t b, int64_t cin, int64_t h, int64_t w,
                                 const float *kernel, int64_t cout, int64_t kh, int64_t kw, const float *t_out,
                                 const float *grad_out, int64_t oh, int64_t ow, const int64_t *stride2,
                                 const int64_t *pad4, float *grad_in, float *grad_kernel, void *workspace,
                                 size_t workspace_bytes, spk_stream stream)
{
    return guarded([&] {
        const Geo g = geometry(h, w, oh, ow, kh, kw, stride2, pad4);
        SPK_REQUIRE(b >= 0 && cin >= 1 && cout >= 1, "invalid dims");
        SPK_REQUIRE(cin * kh * kw < (int64_t(1) << 31) && cout < 65536, "kernel is too large");
        cudaStream_t s = stream_of(stream);
        if (b == 0)
        {
            if (grad_kernel) SPK_CUDA(cudaMemsetAsync(grad_kernel, 0, size_t(cout * cin * kh * kw) * 4, s));
            return;
        }
        if (grad_in)
        {
            SPK_REQUIRE(kernel != nullptr, "grad_in needs the kernel");
            const int HW = int(h * w), P = int(oh * ow), KK = int(kh * kw);
            const int cb = int(std::max<int64_t>(1, std::min<int64_t>(cin, (kItems * kGiThreads) / HW)));
            SPK_REQUIRE(int64_t(cb) * HW <= kItems * kGiThreads,
                        "input planes of more than 1024 pixels are not supported by the input gradient");
            // maps per staging round: their times, gradients and weights in 48 KB
            const int64_t per_z = 2 * int64_t(P) + int64_t(cb) * KK;
            SPK_REQUIRE(per_z <= 12288, "output planes are too large for the input gradient");
            const int zc = int(std::min<int64_t>(cout, 12288 / per_z));
            SPK_REQUIRE(b <= 65535, "batch too large for one call (split it)");
            const dim3 grid(unsigned(ceil_div(cin, cb)), unsigned(b));
            const size_t smem = size_t(zc) * per_z * 4;
            if (g.sy == 1 && g.sx == 1)
                fst_conv_grad_in_kernel<true><<<grid, kGiThreads, smem, s>>>(t_in, kernel, t_out, grad_out, grad_in,
                                                                               int(cin), int(cout), g, cb, zc);
            else
                fst_conv_grad_in_kernel<false><<<grid, kGiThreads, smem, s>>>(t_in, kernel, t_out, grad_out, grad_in,
                                                                                int(cin), int(cout), g, cb, zc);
            SPK_LAUNCHED();
        }
        if (grad_kernel)
        {
            const size_t need = spk_fst_conv_backward_workspace(b, cin, cout, kh, kw);
            SPK_REQUIRE(workspace != nullptr && workspace_bytes >= need, "workspace too small");
            const int groups = int(ceil_div(b, kGwSamples));
            SPK_REQUIRE(groups <= 65535, "batch too large for one call (split it)");
            double *part = static_cast<double *>(workspace);
            // row slices per weight: enough pairs to fill the threads, at most one per row
            const int64_t wk = cin * kh * kw, cap = int64_t(kGwThreads) * kGwRounds;
            int slices = 1;  // a power of two
            while (slices * 2 <= oh && wk * slices * 2 <= cap) slices *= 2;
            const int64_t wblocks = ceil_div(wk, cap / slices);
            SPK_REQUIRE(wblocks <= 65535, "kernel too large");
            SPK_REQUIRE(ow <= 2048, "output rows are too wide for the kernel gradient");
            const int rows = int(std::max<int64_t>(1, std::min<int64_t>(oh, 2048 / ow)));
            const size_t base = size_t(std::min(wk, cap / slices) * slices) * 8 + size_t(2 * rows * ow) * 4;
            const bool stage_in = base + size_t(cin * h * w) * 4 <= 48 * 1024;
            const size_t smem = base + (stage_in ? size_t(cin * h * w) * 4 : 0);
            fst_conv_grad_w_kernel<<<dim3(unsigned(cout), unsigned(groups), unsigned(wblocks)), kGwThreads, smem, s>>>(
                t_in, t_out, grad_out, part, b, int(cin), int(cout), g, kGwSamples, slices, rows, stage_in ? 1 : 0);
            SPK_LAUNCHED();
            const int64_t n = cout * cin * kh * kw;
            fst_conv_grad_w_reduce_kernel<<<grid_for(n, 256), 256, 0, s>>>(part, grad_kernel, n, groups);
            SPK_LAUNCHED();
        }
    });
}

spk_status spk_fst_conv_prespike(const float *t_in, int64_t b, int64_t cin, int64_t h, int64_t w,
                                 const float *kernel, int64_t cout, int64_t kh, int64_t kw, const float *t_out,
                                 int64_t oh, int64_t ow, const int64_t *stride2, const int64_t *pad4, double *out,
                                 spk_stream stream)
{
    return guarded([&] {
        const Geo g = geometry(h, w, oh, ow, kh, kw, stride2, pad4);
        SPK_REQUIRE(b >= 0 && cin >= 1 && cout >= 1, "invalid dims");
        if (b == 0) return;
        fst_conv_prespike_kernel<<<grid_for(b * cout * oh * ow, 256), 256, 0, stream_of(stream)>>>(
            t_in, kernel, t_out, out, b, int(cin), int(cout), g);
        SPK_LAUNCHED();
    });
}

}  // extern "C"
