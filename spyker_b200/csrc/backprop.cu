// Temporal-backprop helpers: target rule, labelize and the sign-weight FC
// backward (src/spyker/cpu/backprop.cpp:40-160).
#include "common.cuh"

namespace spk
{
namespace
{
// backprop.cpp:40-62: one warp per row.
__global__ void backward_kernel(const float *__restrict__ in, float *__restrict__ out,
                                const int64_t *__restrict__ target, int64_t b, int n, float time, float gamma)
{
    const int64_t row = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= b) return;
    const float *id = in + row * n;
    float *od = out + row * n;
    float mn = id[0];
    for (int i = lane; i < n; i += 32) mn = (id[i] < mn) ? id[i] : mn;
    for (int o = 16; o > 0; o >>= 1)
    {
        float v = __shfl_xor_sync(0xffffffffu, mn, o);
        mn = (v < mn) ? v : mn;
    }
    const float upper = __fadd_rn(mn, gamma);
    const float value = (upper < time) ? upper : time;  // std::min(T(time), upper)
    const bool spread = (mn != time);
    const int64_t tg = target[row];
    for (int i = lane; i < n; i += 32)
    {
        float v = id[i];
        if (spread) v = (v < upper) ? value : v;
        if (i == tg) v = (0.f < mn) ? mn : 0.f;  // std::max(T(0), min)
        od[i] = __fdiv_rn(__fsub_rn(v, id[i]), time);
    }
}

// backprop.cpp:68-99: one warp per sample.
template <typename T>
__global__ void labelize_kernel(const T *__restrict__ in, int64_t *__restrict__ out, int64_t b, int t, int n, T thr)
{
    const int64_t s = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (s >= b) return;
    const T *base = in + s * int64_t(t) * n;
    // argmin of first-spike times (first index), then fallback argmax of the last step.
    int best_t = 1 << 30;
    int best_i = 1 << 30;
    for (int i = lane; i < n; i += 32)
    {
        int ft = t;
        for (int q = 0; q < t; ++q)
            if (base[int64_t(q) * n + i] > thr)
            {
                ft = q;
                break;
            }
        if (ft < best_t || (ft == best_t && i < best_i)) best_t = ft, best_i = i;
    }
    for (int o = 16; o > 0; o >>= 1)
    {
        int ot = __shfl_xor_sync(0xffffffffu, best_t, o), oi = __shfl_xor_sync(0xffffffffu, best_i, o);
        if (ot < best_t || (ot == best_t && oi < best_i)) best_t = ot, best_i = oi;
    }
    int64_t label = best_i;
    if (best_t == t)
    {
        // First index of the maximum of the last step (std::max_element).
        const T *last = base + int64_t(t - 1) * n;
        T bv = T(0);
        int bi = -1;
        for (int i = lane; i < n; i += 32)
            if (bi < 0 || bv < last[i]) bv = last[i], bi = i;
        for (int o = 16; o > 0; o >>= 1)
        {
            T ov = __shfl_xor_sync(0xffffffffu, bv, o);
            int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            bool take = (oi >= 0) && (bi < 0 || bv < ov || (!(ov < bv) && oi < bi));
            if (take) bv = ov, bi = oi;
        }
        label = bi;
    }
    if (lane == 0) out[s] = label;
}

// backprop.cpp:105-160, one CTA, sequential over samples.  The kernel and
// the selection matrix stay in global memory (L2 resident).
__global__ void fcbackward_kernel(float *__restrict__ kernel, int no, int ni, const float *__restrict__ in,
                                  const float *__restrict__ out, const float *__restrict__ grad,
                                  float *__restrict__ next, int64_t b, float lrate, float lrf, float lambda,
                                  float *__restrict__ sign, float *__restrict__ select, float *__restrict__ sfactor)
{
    __shared__ float s_part[32];
    const int k = no * ni;
    for (int i = threadIdx.x; i < k; i += blockDim.x)
    {
        float v = kernel[i];
        sign[i] = v > 0.f ? 1.f : (v < 0.f ? -1.f : 0.f);
    }
    float sf = 0.f;
    if (threadIdx.x == 0) sf = sfactor[0];
    __syncthreads();
    const float mult = __fmul_rn(lrate, lambda);
    for (int64_t s = 0; s < b; ++s)
    {
        const float *id = in + s * ni;
        float part = 0.f;
        for (int i = threadIdx.x; i < k; i += blockDim.x)
        {
            const int j = i / ni, c = i % ni;
            const float o = out[s * no + j], g = grad[s * no + j];
            const float sel = float(id[c] < o) * g;
            select[i] = sel;
            float kv = __fmaf_rn(-lrate, sel, kernel[i]);
            kv = __fmaf_rn(-mult, kv, kv);
            kernel[i] = kv;
            part = __fmaf_rn(__fmul_rn(lrf, sel), sign[i], part);
        }
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = part;
        __syncthreads();
        if (threadIdx.x == 0)
        {
            float sum = 0.f;
            for (int q = 0; q < int(blockDim.x >> 5); ++q) sum += s_part[q];
            sf = __fsub_rn(sf, __fdiv_rn(sum, float(k)));
        }
        for (int c = threadIdx.x; c < ni; c += blockDim.x)
        {
            float acc = 0.f;
            for (int j = 0; j < no; ++j) acc = __fmaf_rn(kernel[j * ni + c], select[j * ni + c], acc);
            next[s * ni + c] = acc;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) sfactor[0] = sf;
}
}  // namespace
}  // namespace spk

using namespace spk;

extern "C" {

spk_status spk_backward(const float *in, float *out, const int64_t *target, int64_t b, int64_t n, int64_t time,
                        double gamma, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(time > 0, "time steps must be higher than zero");
        SPK_REQUIRE(b >= 0 && n >= 1, "invalid dims");
        if (b == 0) return;
        backward_kernel<<<unsigned(ceil_div(b * 32, 256)), 256, 0, stream_of(stream)>>>(in, out, target, b, int(n),
                                                                                      float(time), float(gamma));
        SPK_LAUNCHED();
    });
}

spk_status spk_labelize(const void *in, spk_dtype type, int64_t *out, int64_t b, int64_t t, int64_t n,
                        double threshold, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(b >= 0 && t >= 1 && n >= 1, "invalid dims");
        if (b == 0) return;
        unsigned grid = unsigned(ceil_div(b * 32, 256));
        if (type == SPK_F32)
            labelize_kernel<float><<<grid, 256, 0, stream_of(stream)>>>((const float *)in, out, b, int(t), int(n),
                                                                       float(threshold));
        else
            throw Error(SPK_ERR_UNSUPPORTED, "labelize supports F32 input");
        SPK_LAUNCHED();
    });
}

size_t spk_fcbackward_workspace(int64_t no, int64_t ni) { return size_t(no * ni) * 8 + 256; }

spk_status spk_fcbackward(float *kernel, int64_t no, int64_t ni, const float *in, const float *out, const float *grad,
                          float *next, int64_t b, float *bp, void *ws, size_t ws_bytes, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(bp != nullptr, "null config");
        SPK_REQUIRE(no >= 1 && ni >= 1 && b >= 0, "invalid dims");
        SPK_REQUIRE(ws != nullptr && ws_bytes >= spk_fcbackward_workspace(no, ni), "workspace is too small");
        float *sign = reinterpret_cast<float *>(ws);
        float *select = sign + no * ni;
        float *sf = select + no * ni;
        cudaStream_t s = stream_of(stream);
        SPK_CUDA(cudaMemcpyAsync(sf, &bp[0], sizeof(float), cudaMemcpyHostToDevice, s));
        fcbackward_kernel<<<1, 1024, 0, s>>>(kernel, int(no), int(ni), in, out, grad, next, b, bp[1], bp[2], bp[3], sign,
                                             select, sf);
        SPK_LAUNCHED();
        SPK_CUDA(cudaMemcpyAsync(&bp[0], sf, sizeof(float), cudaMemcpyDeviceToHost, s));
        SPK_CUDA(cudaStreamSynchronize(s));
    });
}

}  // extern "C"
