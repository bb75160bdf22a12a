/* C++ layer of spyker_b200: the reference's `Spyker::` API for the dense
 * spiking-CNN hot path (src/spyker/opers.h:130-760, src/spyker/utils.h:96-524),
 * header-only, over the C ABI of spyker_b200.h.
 *
 * Same names, argument order, defaults and error conditions as the reference
 * for: Tensor (device tensors only), Expand2 / Expand4, DoGFilter, DoG,
 * GaborFilter, Gabor, LoG, Conv (operator(), stdp), FC (operator(), stdp,
 * backward), STDPConfig, BPConfig, Winner / Winners, code, threshold,
 * infinite, fire, gather, scatter, pad, pool, inhibit, convwta, fcwta, conv,
 * fc, backward, labelize, and the event-list path: SparseTensor, Sparse::code,
 * conv, pad, gather, pool, inhibit, convwta, Conv on a SparseTensor and its
 * stdp.
 * Tensors live in the current CUDA device's memory; the reference's host
 * tensors become Tensor::from_host / Tensor::to_host.  Every call is queued on
 * Spyker::stream() (the legacy default stream unless set), so calls run in
 * program order; functions that return host data (convwta, fcwta, to_host)
 * wait for the stream.  Errors throw Spyker::Error with the library's message
 * (the reference's SpykerCompare / SpykerAssert throw std::runtime_error).
 *
 * Not a counterpart of the reference: conv_fire_wta, the fused layer
 * (conv -> threshold -> inhibit -> fire + convwta [+ pool]) of
 * spk_conv_fire_wta, with the op-by-op composition as its fallback.
 *
 * Link: -lspyker_b200 -lcudart (spyker_b200/lib). */
#ifndef SPYKER_B200_HPP
#define SPYKER_B200_HPP

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "spyker_b200.h"

namespace Spyker
{
using Size = int64_t;
using F64 = double;
using Shape = std::vector<Size>;

/* utils.h:96-120: the same order as spk_dtype. */
enum class Type : int32_t
{
    I8,
    I16,
    I32,
    I64,
    U8,
    U16,
    U32,
    U64,
    F16,
    F32,
    F64
};

struct Error : std::runtime_error
{
    using std::runtime_error::runtime_error;
};

namespace detail
{
inline cudaStream_t &stream_ref()
{
    static thread_local cudaStream_t s = nullptr;
    return s;
}

inline void check(spk_status s, const char *what)
{
    if (s != SPK_OK) throw Error(std::string(what) + ": " + spk_last_error());
}

inline void cuda(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) throw Error(std::string(what) + ": " + cudaGetErrorString(e));
}

inline void require(bool ok, const char *msg)
{
    if (!ok) throw Error(msg);
}

inline size_t type_size(Type t)
{
    static const size_t sz[] = {1, 2, 4, 8, 1, 2, 4, 8, 2, 4, 8};
    return sz[int(t)];
}

inline Size prod(const Shape &s, size_t from = 0, size_t to = size_t(-1))
{
    Size p = 1;
    for (size_t i = from; i < s.size() && i < to; ++i) p *= s[i];
    return p;
}

/* Stream-ordered scratch of one call (freed on the same stream). */
struct Scratch
{
    void *ptr = nullptr;
    size_t bytes = 0;
    explicit Scratch(size_t n) : bytes(n)
    {
        if (n > 0) cuda(cudaMallocAsync(&ptr, n, stream_ref()), "workspace allocation");
    }
    ~Scratch()
    {
        if (ptr) cudaFreeAsync(ptr, stream_ref());
    }
    Scratch(const Scratch &) = delete;
    Scratch &operator=(const Scratch &) = delete;
};
}  // namespace detail

/* The stream every call of this layer is queued on. */
inline cudaStream_t stream() { return detail::stream_ref(); }
inline void setStream(cudaStream_t s) { detail::stream_ref() = s; }
inline void synchronize() { detail::cuda(cudaStreamSynchronize(stream()), "synchronize"); }

/* opers.h:130-142: one value for both, or (y, x). */
class Expand2
{
    Shape data;

public:
    Expand2() : data{0, 0} {}
    Expand2(Size a) : data{a, a} {}
    Expand2(Size a, Size b) : data{a, b} {}
    Size operator[](Size i) const { return data[size_t(i)]; }
    Shape get() const { return data; }
};

/* opers.h:147-160: (top, left, bottom, right); two values = (y, x). */
class Expand4
{
    Shape data;

public:
    Expand4() : data{0, 0, 0, 0} {}
    Expand4(Size a) : data{a, a, a, a} {}
    Expand4(Size a, Size b) : data{a, b, a, b} {}
    Expand4(Size a, Size b, Size c, Size d) : data{a, b, c, d} {}
    Size operator[](Size i) const { return data[size_t(i)]; }
    Shape get() const { return data; }
};

/* A dense tensor in device memory (the reference's Tensor on a CUDA
 * device, utils.h / base.h).  Copies share the buffer, as there. */
class Tensor
{
    std::shared_ptr<void> _data;
    Shape _shape;
    Type _type = Type::F32;

public:
    Tensor() = default;
    Tensor(Type type, const Shape &shape) : _shape(shape), _type(type)
    {
        for (Size d : shape) detail::require(d >= 0, "Tensor shape can't be negative.");
        void *p = nullptr;
        const size_t n = size_t(detail::prod(shape)) * detail::type_size(type);
        detail::cuda(cudaMalloc(&p, n > 0 ? n : 1), "Tensor allocation");
        detail::cuda(cudaMemsetAsync(p, 0, n, stream()), "Tensor initialisation");
        _data = std::shared_ptr<void>(p, [](void *q) { cudaFree(q); });
    }
    explicit Tensor(const Shape &shape, Type type = Type::F32) : Tensor(type, shape) {}
    /* A view of caller-owned device memory (not freed here); the reference's
     * Tensor(data, device, type, shape) wrapping a raw pointer. */
    Tensor(void *device_data, Type type, const Shape &shape) : _shape(shape), _type(type)
    {
        for (Size d : shape) detail::require(d >= 0, "Tensor shape can't be negative.");
        detail::require(device_data != nullptr || detail::prod(shape) == 0, "Tensor data can't be null.");
        _data = std::shared_ptr<void>(device_data, [](void *) {});
    }

    static Tensor from_host(const void *host, Type type, const Shape &shape)
    {
        Tensor t(type, shape);
        detail::cuda(cudaMemcpyAsync(t.data(), host, t.bytes(), cudaMemcpyHostToDevice, stream()), "Tensor upload");
        detail::cuda(cudaStreamSynchronize(stream()), "Tensor upload");
        return t;
    }
    void to_host(void *host) const
    {
        detail::cuda(cudaMemcpyAsync(host, data(), bytes(), cudaMemcpyDeviceToHost, stream()), "Tensor download");
        detail::cuda(cudaStreamSynchronize(stream()), "Tensor download");
    }
    template <typename T>
    std::vector<T> to_vector() const
    {
        detail::require(sizeof(T) == detail::type_size(_type), "Tensor element size mismatch.");
        std::vector<T> v(static_cast<size_t>(numel()));
        if (!v.empty()) to_host(v.data());
        return v;
    }

    bool valid() const { return bool(_data); }
    void *data() const { return _data.get(); }
    template <typename T>
    T *data() const
    {
        return static_cast<T *>(_data.get());
    }
    Type type() const { return _type; }
    Shape shape() const { return _shape; }
    Size shape(Size i) const { return _shape[size_t(i)]; }
    Size dims() const { return Size(_shape.size()); }
    Size numel() const { return detail::prod(_shape); }
    size_t bytes() const { return size_t(numel()) * detail::type_size(_type); }
    Tensor reshape(const Shape &shape) const
    {
        detail::require(detail::prod(shape) == numel(), "Tensor reshape can't change the element count.");
        Tensor t = *this;
        t._shape = shape;
        return t;
    }
    Tensor copy() const
    {
        Tensor t(_type, _shape);
        detail::cuda(cudaMemcpyAsync(t.data(), data(), bytes(), cudaMemcpyDeviceToDevice, stream()), "Tensor copy");
        return t;
    }
};

/* utils.h:483-502. */
struct Winner
{
    Size c, t, z, y, x;
};
using Winners = std::vector<std::vector<Winner>>;

/* utils.h:505-524. */
struct STDPConfig
{
    F64 positive = 0, negative = 0;
    bool stabilize = true;
    F64 lower = 0, upper = 1;
    STDPConfig() {}
    STDPConfig(F64 positive, F64 negative, bool stabilize = true, F64 lower = 0, F64 upper = 1)
        : positive(positive), negative(negative), stabilize(stabilize), lower(lower), upper(upper)
    {
    }
};

/* opers.h:163-174. */
struct DoGFilter
{
    F64 std1, std2;
    DoGFilter(F64 std1, F64 std2) : std1(std1), std2(std2) {}
};

/* opers.h:176-206: theta given in degrees, kept in radians. */
struct GaborFilter
{
    F64 sigma, theta, gamma, lambda, psi;
    GaborFilter(F64 sigma, F64 theta, F64 gamma, F64 lambda, F64 psi)
        : sigma(sigma), theta(theta * 0.017453292519943295), gamma(gamma), lambda(lambda), psi(psi)
    {
    }
};

/* utils.h:525-547. */
struct BPConfig
{
    float sfactor = 1, lrate = 1, lrf = 1, lambda = 0;
    BPConfig() {}
    BPConfig(float sfactor, float lrate, float lrf, float lambda)
        : sfactor(sfactor), lrate(lrate), lrf(lrf), lambda(lambda)
    {
    }
};

namespace detail
{
inline spk_dtype dt(Type t) { return spk_dtype(int(t)); }

inline std::vector<int64_t> pad4(const Expand4 &p) { return {p[0], p[1], p[2], p[3]}; }

/* [B, count, 5] int32 records + counts [B] -> nested winners (one copy). */
inline Winners winners_from(const Tensor &records, const Tensor &counts, Size count)
{
    const Size b = counts.numel();
    std::vector<int32_t> rec = records.to_vector<int32_t>(), cnt = counts.to_vector<int32_t>();
    Winners w(static_cast<size_t>(b));
    for (Size i = 0; i < b; ++i)
        for (Size j = 0; j < cnt[size_t(i)] && j < count; ++j)
        {
            const int32_t *r = &rec[size_t((i * count + j) * 5)];
            w[size_t(i)].push_back(Winner{r[0], r[1], r[2], r[3], r[4]});
        }
    return w;
}

/* Nested winners -> device records [B, count, 5] and counts [B]. */
inline std::pair<Tensor, Tensor> winners_to(const Winners &w, Size batch, Size &count)
{
    require(Size(w.size()) == batch, "Winners count must match the input batch.");
    count = 1;
    for (const auto &v : w) count = std::max<Size>(count, Size(v.size()));
    std::vector<int32_t> rec(static_cast<size_t>(batch * count * 5), 0), cnt(static_cast<size_t>(batch), 0);
    for (Size i = 0; i < batch; ++i)
    {
        cnt[size_t(i)] = int32_t(w[size_t(i)].size());
        for (size_t j = 0; j < w[size_t(i)].size(); ++j)
        {
            const Winner &x = w[size_t(i)][j];
            int32_t *r = &rec[size_t((i * count + Size(j)) * 5)];
            r[0] = int32_t(x.c), r[1] = int32_t(x.t), r[2] = int32_t(x.z), r[3] = int32_t(x.y), r[4] = int32_t(x.x);
        }
    }
    return {Tensor::from_host(rec.data(), Type::I32, {batch, count, 5}),
            Tensor::from_host(cnt.data(), Type::I32, {batch})};
}

inline std::vector<F64> configs(const std::vector<STDPConfig> &c)
{
    std::vector<F64> v;
    for (const auto &x : c) v.insert(v.end(), {x.positive, x.negative, F64(x.stabilize), x.lower, x.upper});
    return v;
}
}  // namespace detail

/* ---- coding and elementwise (opers.h:598-700) ----------------------------- */

namespace detail
{
inline void require_shape(const Tensor &t, const Shape &s, const char *msg) { require(t.shape() == s, msg); }
}  // namespace detail

/* [B, ...] -> output [B, T, ...] cumulative spikes; sort: rank order
 * (opers.h:632, the output's type chosen by the caller). */
inline Tensor code(Tensor input, Tensor output, Size time, bool sort = true)
{
    detail::require(time > 0, "Input time can't be less than 1.");
    detail::require(input.dims() >= 2, "Input dimensions must be at least 2.");
    const Shape s = input.shape();
    Shape o{s[0], time};
    o.insert(o.end(), s.begin() + 1, s.end());
    detail::require_shape(output, o, "Output shape is not compatible with the input.");
    const Size x = detail::prod(s, 1);
    detail::Scratch ws(spk_rank_code_workspace(s[0], x, int(sort)));
    detail::check(spk_rank_code(input.data(), detail::dt(input.type()), output.data(), detail::dt(output.type()), s[0],
                                time, x, int(sort), ws.ptr, ws.bytes, stream()),
                  "code");
    return output;
}

/* [B, ...] -> [B, T, ...] cumulative spikes; sort: rank order (opers.h:621). */
inline Tensor code(Tensor input, Size time, bool sort = true, Type type = Type::U8)
{
    detail::require(input.dims() >= 2, "Input dimensions must be at least 2.");
    const Shape s = input.shape();
    Shape o{s[0], std::max<Size>(time, 0)};
    o.insert(o.end(), s.begin() + 1, s.end());
    return code(input, Tensor(type, o), time, sort);
}

inline Tensor threshold(Tensor input, F64 threshold, F64 value = 0, bool inplace = true)
{
    Tensor t = inplace ? input : input.copy();
    detail::check(spk_threshold(t.data(), detail::dt(t.type()), t.numel(), threshold, value, stream()), "threshold");
    return t;
}

/* [B, T, ...]: steps 0 .. T-2 set to value (cpu/fire.cpp). */
inline Tensor infinite(Tensor input, F64 value = 0, bool inplace = true)
{
    detail::require(input.dims() >= 3, "Input dimensions must be at least 3.");
    Tensor t = inplace ? input : input.copy();
    detail::check(spk_rank_infinite(t.data(), detail::dt(t.type()), t.shape(0), t.shape(1),
                                    detail::prod(t.shape(), 2), value, stream()),
                  "infinite");
    return t;
}

inline Tensor fire(Tensor input, Tensor output, F64 threshold = 0)
{
    detail::require_shape(output, input.shape(), "Output shape is not compatible with the input.");
    detail::check(spk_rank_fire(input.data(), detail::dt(input.type()), output.data(), detail::dt(output.type()),
                                input.numel(), threshold, stream()),
                  "fire");
    return output;
}

inline Tensor fire(Tensor input, F64 threshold = 0, Type type = Type::U8)
{
    return fire(input, Tensor(type, input.shape()), threshold);
}

/* [B, T, ...] -> [B, ...] first step above the threshold (T when none). */
inline Tensor gather(Tensor input, Tensor output, F64 threshold = 0)
{
    detail::require(input.dims() >= 3, "Input dimensions must be at least 3.");
    Shape o{input.shape(0)};
    const Shape s = input.shape();
    o.insert(o.end(), s.begin() + 2, s.end());
    detail::require_shape(output, o, "Output shape is not compatible with the input.");
    detail::check(spk_rank_gather(input.data(), detail::dt(input.type()), output.data(), detail::dt(output.type()), s[0],
                                  s[1], detail::prod(s, 2), threshold, stream()),
                  "gather");
    return output;
}

inline Tensor gather(Tensor input, F64 threshold = 0, Type type = Type::U8)
{
    detail::require(input.dims() >= 3, "Input dimensions must be at least 3.");
    Shape o{input.shape(0)};
    const Shape s = input.shape();
    o.insert(o.end(), s.begin() + 2, s.end());
    return gather(input, Tensor(type, o), threshold);
}

/* [B, ...] first-spike times -> [B, T, ...] cumulative spikes. */
inline Tensor scatter(Tensor input, Size time, Type type = Type::U8)
{
    detail::require(time > 0, "Input time can't be less than 1.");
    const Shape s = input.shape();
    Shape o{s[0], time};
    o.insert(o.end(), s.begin() + 1, s.end());
    Tensor out(type, o);
    detail::check(spk_rank_scatter(input.data(), detail::dt(input.type()), out.data(), detail::dt(type), s[0], time,
                                   detail::prod(s, 1), stream()),
                  "scatter");
    return out;
}

/* [..., H, W] -> [..., H + top + bottom, W + left + right]. */
inline Tensor pad(Tensor input, Expand4 pad, F64 value = 0)
{
    detail::require(input.dims() >= 2, "Input dimensions must be at least 2.");
    detail::require(pad[0] >= 0 && pad[1] >= 0 && pad[2] >= 0 && pad[3] >= 0, "Pad items are incorrect.");
    Shape o = input.shape();
    const Size h = o[o.size() - 2], w = o[o.size() - 1];
    o[o.size() - 2] = h + pad[0] + pad[2], o[o.size() - 1] = w + pad[1] + pad[3];
    Tensor out(input.type(), o);
    const auto p = detail::pad4(pad);
    detail::check(spk_pad(input.data(), out.data(), detail::dt(input.type()), input.numel() / (h * w), h, w, p.data(),
                          value, stream()),
                  "pad");
    return out;
}

/* Max pooling of the last two dimensions; stride 0 = the window
 * (opers.h:709, cpu/pool.cpp:53-86). */
inline Tensor pool(Tensor input, Tensor output, Expand2 kernel, Expand2 stride = 0, Expand4 pad = 0)
{
    detail::require(input.dims() >= 3, "Input dimensions must be at least 3.");
    detail::require(output.type() == input.type(), "Output type must be the input's.");
    if (stride[0] == 0 && stride[1] == 0) stride = kernel;
    detail::require(kernel[0] > 0 && kernel[1] > 0 && stride[0] > 0 && stride[1] > 0 && pad[0] >= 0 && pad[1] >= 0 &&
                        pad[2] >= 0 && pad[3] >= 0,
                    "Kernel, stride or pad items are incorrect.");
    Shape o = input.shape();
    const Size h = o[o.size() - 2], w = o[o.size() - 1];
    detail::require(h + pad[0] + pad[2] >= kernel[0] && w + pad[1] + pad[3] >= kernel[1],
                    "Input and kernel shapes are not compatible.");
    const Size oh = (h + pad[0] + pad[2] - kernel[0]) / stride[0] + 1;
    const Size ow = (w + pad[1] + pad[3] - kernel[1]) / stride[1] + 1;
    detail::require(oh > 0 && ow > 0, "Input and kernel shapes are not compatible.");
    o[o.size() - 2] = oh, o[o.size() - 1] = ow;
    detail::require_shape(output, o, "Output shape is not compatible with the input.");
    const auto p = detail::pad4(pad);
    detail::check(spk_rank_pool(input.data(), output.data(), detail::dt(input.type()), input.numel() / (h * w), h, w,
                                oh, ow, kernel[0], kernel[1], stride[0], stride[1], p.data(), stream()),
                  "pool");
    return output;
}

inline Tensor pool(Tensor input, Expand2 kernel, Expand2 stride = 0, Expand4 pad = 0)
{
    detail::require(input.dims() >= 3, "Input dimensions must be at least 3.");
    if (stride[0] == 0 && stride[1] == 0) stride = kernel;
    detail::require(kernel[0] > 0 && kernel[1] > 0 && stride[0] > 0 && stride[1] > 0 && pad[0] >= 0 && pad[1] >= 0 &&
                        pad[2] >= 0 && pad[3] >= 0,
                    "Kernel, stride or pad items are incorrect.");
    Shape o = input.shape();
    const Size h = o[o.size() - 2], w = o[o.size() - 1];
    detail::require(h + pad[0] + pad[2] >= kernel[0] && w + pad[1] + pad[3] >= kernel[1],
                    "Input and kernel shapes are not compatible.");
    const Size oh = (h + pad[0] + pad[2] - kernel[0]) / stride[0] + 1;
    const Size ow = (w + pad[1] + pad[3] - kernel[1]) / stride[1] + 1;
    detail::require(oh > 0 && ow > 0, "Input and kernel shapes are not compatible.");
    o[o.size() - 2] = oh, o[o.size() - 1] = ow;
    Tensor out(input.type(), o);
    const auto p = detail::pad4(pad);
    detail::check(spk_rank_pool(input.data(), out.data(), detail::dt(input.type()), input.numel() / (h * w), h, w, oh,
                                ow, kernel[0], kernel[1], stride[0], stride[1], p.data(), stream()),
                  "pool");
    return out;
}

/* [B, T, C, ...] lateral inhibition (cpu/inhibit.cpp:41-121). */
inline Tensor inhibit(Tensor input, F64 threshold = 0, bool inplace = true)
{
    detail::require(input.dims() >= 4, "Input dimensions must be at least 4.");
    Tensor t = inplace ? input : input.copy();
    const Shape s = t.shape();
    detail::check(spk_rank_inhibit(t.data(), detail::dt(t.type()), s[0], s[1], s[2], detail::prod(s, 3), threshold,
                                   stream()),
                  "inhibit");
    return t;
}

/* [B, T, C, H, W] -> up to count winners per sample (cpu/wta.cpp:123-152). */
inline Winners convwta(Tensor input, Expand2 radius, Size count, F64 threshold = 0)
{
    detail::require(input.dims() == 5, "Input dimensions must be 5.");
    detail::require(count >= 0 && radius[0] >= 0 && radius[1] >= 0, "Winners count or radius are incorrect.");
    const Shape s = input.shape();
    if (count == 0) return Winners(size_t(s[0]));
    Tensor rec(Type::I32, {s[0], count, 5}), cnt(Type::I32, {s[0]});
    detail::Scratch ws(spk_rank_convwta_workspace(s[0], s[1], s[2], s[3], s[4]));
    detail::check(spk_rank_convwta(input.data(), detail::dt(input.type()), s[0], s[1], s[2], s[3], s[4], radius[0],
                                   radius[1], count, threshold, rec.data<int32_t>(), cnt.data<int32_t>(), ws.ptr,
                                   ws.bytes, stream()),
                  "convwta");
    return detail::winners_from(rec, cnt, count);
}

/* [B, T, N] -> up to count winners per sample (cpu/wta.cpp:72-96). */
inline Winners fcwta(Tensor input, Size radius, Size count, F64 threshold = 0)
{
    detail::require(input.dims() == 3, "Input dimensions must be 3.");
    detail::require(count >= 0 && radius >= 0, "Winners count or radius are incorrect.");
    const Shape s = input.shape();
    if (count == 0) return Winners(size_t(s[0]));
    Tensor rec(Type::I32, {s[0], count, 5}), cnt(Type::I32, {s[0]});
    detail::Scratch ws(spk_rank_fcwta_workspace(s[0], s[1], s[2]));
    detail::check(spk_rank_fcwta(input.data(), detail::dt(input.type()), s[0], s[1], s[2], radius, count, threshold,
                                 rec.data<int32_t>(), cnt.data<int32_t>(), ws.ptr, ws.bytes, stream()),
                  "fcwta");
    return detail::winners_from(rec, cnt, count);
}

/* ---- convolution (opers.h:545-555) ------------------------------------------ */

/* [B, T, Cin, H, W] (or [N, Cin, H, W]) x [Cout, Cin, KH, KW] F32 ->
 * F32 potentials [B, T, Cout, OH, OW] written to output (opers.h:555). */
inline Tensor conv(Tensor input, Tensor kernel, Tensor output, Expand2 stride = 1, Expand4 pad = 0,
                   int precision = SPK_CONV_FP32)
{
    detail::require(input.dims() == 4 || input.dims() == 5, "Input dimensions must be 4 or 5.");
    detail::require(kernel.dims() == 4 && kernel.type() == Type::F32, "Kernel must be a 4D F32 tensor.");
    detail::require(output.type() == Type::F32, "Output must be F32.");
    detail::require(stride[0] > 0 && stride[1] > 0 && pad[0] >= 0 && pad[1] >= 0 && pad[2] >= 0 && pad[3] >= 0,
                    "Stride or pad items are incorrect.");
    const Shape s = input.shape();
    const size_t d = s.size();
    const Size cin = s[d - 3], h = s[d - 2], w = s[d - 1];
    const Size cout = kernel.shape(0), kh = kernel.shape(2), kw = kernel.shape(3);
    detail::require(kernel.shape(1) == cin, "Input and kernel channels are not compatible.");
    detail::require(h + pad[0] + pad[2] >= kh && w + pad[1] + pad[3] >= kw, "Input and kernel shapes are not compatible.");
    const Size oh = (h + pad[0] + pad[2] - kh) / stride[0] + 1, ow = (w + pad[1] + pad[3] - kw) / stride[1] + 1;
    detail::require(oh > 0 && ow > 0, "Input and kernel shapes are not compatible.");
    Shape o(s.begin(), s.end() - 3);
    o.insert(o.end(), {cout, oh, ow});
    detail::require_shape(output, o, "Output shape is not compatible with the input.");
    const Size n = detail::prod(s, 0, d - 3);
    const auto p = detail::pad4(pad);
    detail::Scratch ws(spk_conv_workspace(n, cin, h, w, cout, kh, kw, precision));
    detail::check(spk_conv(input.data(), detail::dt(input.type()), kernel.data<float>(), output.data<float>(), n, cin, h,
                           w, cout, kh, kw, stride[0], stride[1], p.data(), precision, ws.ptr, ws.bytes, stream()),
                  "conv");
    return output;
}

/* The same into a new F32 tensor (opers.h:545). */
inline Tensor conv(Tensor input, Tensor kernel, Expand2 stride = 1, Expand4 pad = 0,
                   int precision = SPK_CONV_FP32)
{
    detail::require(input.dims() == 4 || input.dims() == 5, "Input dimensions must be 4 or 5.");
    detail::require(kernel.dims() == 4 && kernel.type() == Type::F32, "Kernel must be a 4D F32 tensor.");
    detail::require(stride[0] > 0 && stride[1] > 0 && pad[0] >= 0 && pad[1] >= 0 && pad[2] >= 0 && pad[3] >= 0,
                    "Stride or pad items are incorrect.");
    const Shape s = input.shape();
    const size_t d = s.size();
    const Size cin = s[d - 3], h = s[d - 2], w = s[d - 1];
    const Size cout = kernel.shape(0), kh = kernel.shape(2), kw = kernel.shape(3);
    detail::require(kernel.shape(1) == cin, "Input and kernel channels are not compatible.");
    detail::require(h + pad[0] + pad[2] >= kh && w + pad[1] + pad[3] >= kw, "Input and kernel shapes are not compatible.");
    const Size oh = (h + pad[0] + pad[2] - kh) / stride[0] + 1, ow = (w + pad[1] + pad[3] - kw) / stride[1] + 1;
    detail::require(oh > 0 && ow > 0, "Input and kernel shapes are not compatible.");
    Shape o(s.begin(), s.end() - 3);
    o.insert(o.end(), {cout, oh, ow});
    Tensor out(Type::F32, o);
    const Size n = detail::prod(s, 0, d - 3);
    const auto p = detail::pad4(pad);
    detail::Scratch ws(spk_conv_workspace(n, cin, h, w, cout, kh, kw, precision));
    detail::check(spk_conv(input.data(), detail::dt(input.type()), kernel.data<float>(), out.data<float>(), n, cin, h, w,
                           cout, kh, kw, stride[0], stride[1], p.data(), precision, ws.ptr, ws.bytes, stream()),
                  "conv");
    return out;
}

/* ---- fully connected and temporal backprop (opers.h:560-580, 755-761) ------ */

/* input [B, T, I] (U8 or F32; [T, I] is one sample), kernel [O, I] F32 ->
 * output [B, T, O] F32; sign: the kernel's signs (cpu/fc.cpp). */
inline Tensor fc(Tensor input, Tensor kernel, Tensor output, bool sign = false)
{
    detail::require(input.dims() == 2 || input.dims() == 3, "Input dimensions couldn't be viewed as 3D.");
    detail::require(input.type() == Type::U8 || input.type() == Type::F32, "fc takes U8 or F32 input.");
    detail::require(kernel.dims() == 2 && kernel.type() == Type::F32, "Kernel must be a 2D F32 tensor.");
    Shape s = input.shape();
    if (s.size() == 2) s.insert(s.begin(), 1);
    detail::require(s[2] == kernel.shape(1), "Input and kernel shapes don't match.");
    detail::require(output.type() == Type::F32 && output.numel() == s[0] * s[1] * kernel.shape(0),
                    "Output shape is not compatible with the input.");
    detail::check(spk_fc(input.data(), detail::dt(input.type()), kernel.data<float>(), output.data<float>(), s[0] * s[1],
                         s[2], kernel.shape(0), int(sign), stream()),
                  "fc");
    return output;
}

inline Tensor fc(Tensor input, Tensor kernel, bool sign = false)
{
    Shape s = input.shape();
    detail::require(!s.empty(), "Input dimensions couldn't be viewed as 3D.");
    s.back() = kernel.dims() == 2 ? kernel.shape(0) : 0;
    Tensor out(Type::F32, s);
    return fc(input, kernel, out, sign);
}

/* Target-rule gradient of first-spike times: input / output [B, ...] F32,
 * target [B] I64 (cpu/backprop.cpp:40-62). */
inline Tensor backward(Tensor input, Tensor output, Tensor target, Size time, F64 gamma)
{
    detail::require(time > 0, "Time steps must be higher than zero.");
    detail::require(input.type() == Type::F32 && output.type() == Type::F32, "backward takes F32 tensors.");
    detail::require(target.type() == Type::I64, "Target type must have I64 type.");
    detail::require(input.dims() >= 1 && target.numel() == input.shape(0), "Input and target shapes are not compatible.");
    detail::require(output.shape() == input.shape(), "Output shape is not compatible with the input.");
    const Size b = input.shape(0);
    detail::check(spk_backward(input.data<float>(), output.data<float>(), target.data<int64_t>(), b,
                               b > 0 ? input.numel() / b : 0, time, gamma, stream()),
                  "backward");
    return output;
}

inline Tensor backward(Tensor input, Tensor target, Size time, F64 gamma)
{
    Tensor out(Type::F32, input.shape());
    return backward(input, out, target, time, gamma);
}

/* input [B, T, N, ...] F32 -> output [B] I64 labels (cpu/backprop.cpp:68-99). */
inline Tensor labelize(Tensor input, Tensor output, F64 threshold)
{
    detail::require(input.dims() >= 3, "Input dimensions must be at least 3.");
    detail::require(input.type() == Type::F32, "labelize takes F32 input.");
    detail::require(output.type() == Type::I64 && output.numel() == input.shape(0),
                    "Output shape is not compatible with the input.");
    const Size b = input.shape(0), t = input.shape(1);
    detail::check(spk_labelize(input.data(), detail::dt(input.type()), output.data<int64_t>(), b, t,
                               detail::prod(input.shape(), 2), threshold, stream()),
                  "labelize");
    return output;
}

inline Tensor labelize(Tensor input, F64 threshold)
{
    detail::require(input.dims() >= 3, "Input dimensions must be at least 3.");
    Tensor out(Type::I64, {input.shape(0)});
    return labelize(input, out, threshold);
}

/* ---- modules (opers.h:211-456) ---------------------------------------------- */

/* Difference-of-Gaussians bank, window 2 size + 1: [B, C, H, W] ->
 * [B, C F, OH, OW] (cpu/dog.cpp). */
class DoG
{
    Expand4 _pad;

public:
    Tensor kernel;  // F32 [2, F, 2 size + 1, 2 size + 1]

    DoG() {}
    DoG(Size size, const std::vector<DoGFilter> &filters, Expand4 pad = 0) : _pad(pad)
    {
        detail::require(size > 0, "Input size can't be less than 1.");
        detail::require(!filters.empty(), "Input filters count can't be less then 1.");
        detail::require(pad[0] >= 0 && pad[1] >= 0 && pad[2] >= 0 && pad[3] >= 0, "Pad items are incorrect.");
        const Size n = 2 * size + 1, f = Size(filters.size());
        std::vector<double> g(static_cast<size_t>(n * n));
        std::vector<float> k(static_cast<size_t>(2 * f * n * n));
        for (Size i = 0; i < f; ++i)
            for (int which = 0; which < 2; ++which)
            {
                detail::check(spk_gaussian_kernel(g.data(), n, which ? filters[size_t(i)].std2 : filters[size_t(i)].std1),
                              "DoG kernel");
                for (Size j = 0; j < n * n; ++j) k[size_t((which * f + i) * n * n + j)] = float(g[size_t(j)]);
            }
        kernel = Tensor::from_host(k.data(), Type::F32, {2, f, n, n});
    }

    Tensor operator()(Tensor input)
    {
        detail::require(kernel.valid(), "DoG is not initialized.");
        detail::require(input.dims() == 4, "Input dimensions must be 4.");
        detail::require(input.type() == Type::F32, "DoG takes F32 input.");
        const Tensor &x = input;
        const Shape s = x.shape();
        const Size f = kernel.shape(1), kh = kernel.shape(2), kw = kernel.shape(3);
        const Size oh = s[2] + _pad[0] + _pad[2] - kh + 1, ow = s[3] + _pad[1] + _pad[3] - kw + 1;
        detail::require(oh > 0 && ow > 0, "Input and kernel shapes are not compatible.");
        Tensor out(Type::F32, {s[0], s[1] * f, oh, ow});
        const auto p = detail::pad4(_pad);
        detail::check(spk_filter(0, x.data<float>(), kernel.data<float>(), out.data<float>(), s[0] * s[1], s[2], s[3], f,
                                 kh, kw, oh, ow, p.data(), stream()),
                      "DoG");
        return out;
    }
};

namespace detail
{
/* A filter bank's planes: [B, C, H, W] F32 -> [B, C fo, OH, OW] (spk_filter
 * kind `which`, `nk` kernels of the bank). */
inline Tensor filter_bank(int which, const Tensor &kernel, const Expand4 &pad, Tensor input, Size nk, Size fo,
                          const char *what)
{
    require(kernel.valid(), "Filter is not initialized.");
    require(input.dims() == 4, "Input dimensions must be 4.");
    require(input.type() == Type::F32, "Filters take F32 input.");
    const Shape s = input.shape();
    const Size kh = kernel.shape(kernel.dims() - 2), kw = kernel.shape(kernel.dims() - 1);
    const Size oh = s[2] + pad[0] + pad[2] - kh + 1, ow = s[3] + pad[1] + pad[3] - kw + 1;
    require(oh > 0 && ow > 0, "Input and kernel shapes are not compatible.");
    Tensor out(Type::F32, {s[0], s[1] * fo, oh, ow});
    const auto p = pad4(pad);
    check(spk_filter(which, input.data<float>(), kernel.data<float>(), out.data<float>(), s[0] * s[1], s[2], s[3], nk,
                     kh, kw, oh, ow, p.data(), stream()),
          what);
    return out;
}
}  // namespace detail

/* Gabor bank, window 2 size + 1: [B, C, H, W] -> [B, C F, OH, OW] raw
 * responses (opers.h:254-291, cpu/dog.cpp). */
class Gabor
{
    Expand4 _pad;

public:
    Tensor kernel;  // F32 [F, 2 size + 1, 2 size + 1]

    Gabor() {}
    Gabor(Size size, const std::vector<GaborFilter> &filters, Expand4 pad = 0) : _pad(pad)
    {
        detail::require(size > 0, "Input size can't be less than 1.");
        detail::require(!filters.empty(), "Input filters count can't be less then 1.");
        detail::require(pad[0] >= 0 && pad[1] >= 0 && pad[2] >= 0 && pad[3] >= 0, "Pad items are incorrect.");
        const Size n = 2 * size + 1, f = Size(filters.size());
        std::vector<double> g(static_cast<size_t>(n * n));
        std::vector<float> k(static_cast<size_t>(f * n * n));
        for (Size i = 0; i < f; ++i)
        {
            const GaborFilter &q = filters[size_t(i)];
            detail::check(spk_gabor_kernel(g.data(), n, q.sigma, q.theta, q.gamma, q.lambda, q.psi), "Gabor kernel");
            for (Size j = 0; j < n * n; ++j) k[size_t(i * n * n + j)] = float(g[size_t(j)]);
        }
        kernel = Tensor::from_host(k.data(), Type::F32, {f, n, n});
    }

    Tensor operator()(Tensor input)
    {
        const Size f = kernel.valid() ? kernel.shape(0) : 0;
        return detail::filter_bank(1, kernel, _pad, input, f, f, "Gabor");
    }
};

/* Laplacian-of-Gaussian bank as DoG(std / sqrt 2, std sqrt 2), on and off
 * parts: [B, C, H, W] -> [B, 2 C F, OH, OW] (opers.h:297-334, cpu/dog.cpp). */
class LoG
{
    Expand4 _pad;

public:
    Tensor kernel;  // F32 [2, F, 2 size + 1, 2 size + 1]

    LoG() {}
    LoG(Size size, const std::vector<F64> &stds, Expand4 pad = 0) : _pad(pad)
    {
        detail::require(size > 0, "Input size can't be less than 1.");
        detail::require(!stds.empty(), "Input stds count can't be less then 1.");
        detail::require(pad[0] >= 0 && pad[1] >= 0 && pad[2] >= 0 && pad[3] >= 0, "Pad items are incorrect.");
        const Size n = 2 * size + 1, f = Size(stds.size());
        std::vector<double> g(static_cast<size_t>(n * n));
        std::vector<float> k(static_cast<size_t>(2 * f * n * n));
        for (Size i = 0; i < f; ++i)
            for (int which = 0; which < 2; ++which)
            {
                const F64 sd = which ? stds[size_t(i)] * std::sqrt(2.0) : stds[size_t(i)] / std::sqrt(2.0);
                detail::check(spk_gaussian_kernel(g.data(), n, sd), "LoG kernel");
                for (Size j = 0; j < n * n; ++j) k[size_t((which * f + i) * n * n + j)] = float(g[size_t(j)]);
            }
        kernel = Tensor::from_host(k.data(), Type::F32, {2, f, n, n});
    }

    Tensor operator()(Tensor input)
    {
        const Size f = kernel.valid() ? kernel.shape(1) : 0;
        return detail::filter_bank(2, kernel, _pad, input, f, 2 * f, "LoG");
    }
};

/* Sparse binary spikes [U, T, C, H, W] as per-(sample, step) event lists
 * (utils.h:369-420): on the device one CSR array, offsets I64 [U T + 1] and
 * events I32 (x | y << 8 | z << 16), sized for the worst case so no call
 * waits for the host. */
class SparseTensor
{
public:
    Tensor offsets, events;
    Shape shape;

    SparseTensor() {}
    SparseTensor(const Shape &shape_, Size capacity)
        : offsets(Type::I64, {shape_[0] * shape_[1] + 1}), events(Type::I32, {std::max<Size>(capacity, 1)}),
          shape(shape_)
    {
    }
    /* An event at the first step whose value exceeds threshold, per position
     * of a dense [U, T, C, H, W] tensor (sparse/opers.cpp:59-86). */
    explicit SparseTensor(Tensor dense, F64 threshold = 0)
    {
        detail::require(dense.dims() == 5, "Input dimensions must be 5.");
        const Shape s = dense.shape();
        *this = SparseTensor(s, s[0] * s[2] * s[3] * s[4]);
        detail::Scratch ws(spk_sparse_from_dense_workspace(s[0], s[1], s[2], s[3], s[4]));
        detail::check(spk_sparse_from_dense(dense.data(), detail::dt(dense.type()), s[0], s[1], s[2], s[3], s[4],
                                            threshold, offsets.data<int64_t>(), events.data<uint32_t>(),
                                            capacity(), ws.ptr, ws.bytes, stream()),
                      "SparseTensor");
    }

    Size capacity() const { return events.numel(); }
    /* Number of events (waits for the stream). */
    Size numel() const
    {
        int64_t n = 0;
        detail::cuda(cudaMemcpyAsync(&n, offsets.data<int64_t>() + (offsets.numel() - 1), sizeof(n),
                                     cudaMemcpyDeviceToHost, stream()),
                     "SparseTensor::numel");
        detail::cuda(cudaStreamSynchronize(stream()), "SparseTensor::numel");
        return Size(n);
    }
    F64 sparsity() const { return F64(numel()) / F64(detail::prod(shape)); }
    /* Cumulative U8 spikes [U, T, C, H, W] (sparse/opers.cpp:88-104). */
    Tensor dense() const
    {
        Tensor out(Type::U8, shape);
        detail::Scratch ws(spk_sparse_dense_workspace(shape[0], shape[2], shape[3], shape[4]));
        detail::check(spk_sparse_to_dense(offsets.data<int64_t>(), events.data<uint32_t>(), shape[0], shape[1],
                                          shape[2], shape[3], shape[4], out.data(), SPK_U8, ws.ptr, ws.bytes,
                                          stream()),
                      "SparseTensor::dense");
        return out;
    }
};

/* The event-list path (opers.h:763-790, src/spyker/sparse/). */
namespace Sparse
{
/* Rank-order (sort) or latency code of [U, C, H, W] into event lists
 * (sparse/code.cpp:39-130). */
inline SparseTensor code(Tensor input, Size time, bool sort = true)
{
    detail::require(time > 0, "Input time can't be less than 1.");
    detail::require(input.dims() == 4, "Input dimensions must be 4.");
    const Shape s = input.shape();
    SparseTensor out({s[0], time, s[1], s[2], s[3]}, s[0] * s[1] * s[2] * s[3]);
    detail::Scratch ws(spk_sparse_code_workspace(s[0], time, s[1], s[2], s[3]));
    detail::check(spk_sparse_code(input.data(), detail::dt(input.type()), s[0], s[1], s[2], s[3], time, int(sort),
                                  out.offsets.data<int64_t>(), out.events.data<uint32_t>(), out.capacity(), ws.ptr,
                                  ws.bytes, stream()),
                  "Sparse::code");
    return out;
}

/* Incremental convolution and fire on event lists (sparse/conv.cpp:42-160). */
inline SparseTensor conv(SparseTensor input, Tensor kernel, F64 threshold, Expand2 stride = 1, Expand4 pad = 0)
{
    detail::require(kernel.dims() == 4 && kernel.type() == Type::F32, "Kernel must be a 4D F32 tensor.");
    const Shape &s = input.shape;
    const Size cout = kernel.shape(0), kh = kernel.shape(2), kw = kernel.shape(3);
    detail::require(kernel.shape(1) == s[2], "Input and kernel channels are not compatible.");
    const Size oh = s[3] + pad[0] + pad[2] - kh + 1, ow = s[4] + pad[1] + pad[3] - kw + 1;
    SparseTensor out({s[0], s[1], cout, oh, ow}, s[0] * cout * std::max<Size>(oh, 1) * std::max<Size>(ow, 1));
    const auto s2 = stride.get();
    const auto p = detail::pad4(pad);
    detail::Scratch ws(spk_sparse_conv_workspace(s[0], s[1], s[3], s[4], cout, kh, kw, p.data()));
    detail::check(spk_sparse_conv(input.offsets.data<int64_t>(), input.events.data<uint32_t>(), s[0], s[1], s[2],
                                  s[3], s[4], kernel.data<float>(), cout, kh, kw, threshold, s2.data(), p.data(),
                                  out.offsets.data<int64_t>(), out.events.data<uint32_t>(), out.capacity(), ws.ptr,
                                  ws.bytes, stream()),
                  "Sparse::conv");
    return out;
}

/* Every event shifted by (top, left) (sparse/pad.cpp:37-55). */
inline SparseTensor pad(SparseTensor input, Expand4 pad)
{
    detail::require(pad[0] >= 0 && pad[1] >= 0 && pad[2] >= 0 && pad[3] >= 0, "Pad items are incorrect.");
    const Shape &s = input.shape;
    SparseTensor out({s[0], s[1], s[2], s[3] + pad[0] + pad[2], s[4] + pad[1] + pad[3]}, input.capacity());
    const auto p = detail::pad4(pad);
    detail::check(spk_sparse_pad(input.offsets.data<int64_t>(), input.events.data<uint32_t>(), input.capacity(), s[0],
                                 s[1], s[2], s[3], s[4], p.data(), out.offsets.data<int64_t>(),
                                 out.events.data<uint32_t>(), out.capacity(), stream()),
                  "Sparse::pad");
    return out;
}

/* First event time per position [U, C, H, W], T when silent
 * (sparse/opers.cpp:106-118). */
inline Tensor gather(SparseTensor input, Tensor output)
{
    const Shape &s = input.shape;
    detail::require(output.shape() == Shape({s[0], s[2], s[3], s[4]}), "Output shape is not compatible with the input.");
    detail::Scratch ws(spk_sparse_dense_workspace(s[0], s[2], s[3], s[4]));
    detail::check(spk_sparse_gather(input.offsets.data<int64_t>(), input.events.data<uint32_t>(), s[0], s[1], s[2],
                                    s[3], s[4], output.data(), detail::dt(output.type()), ws.ptr, ws.bytes, stream()),
                  "Sparse::gather");
    return output;
}

inline Tensor gather(SparseTensor input, Type type = Type::U8)
{
    const Shape &s = input.shape;
    Tensor out(type, {s[0], s[2], s[3], s[4]});
    return gather(input, out);
}

/* The first event of every pooled cell; stride must equal the kernel
 * (sparse/pool.cpp:37-64). */
inline SparseTensor pool(SparseTensor input, Expand2 kernel, Expand2 stride = 0, Expand4 pad = 0)
{
    if (stride[0] == 0 && stride[1] == 0) stride = kernel;
    detail::require(kernel[0] >= 1 && kernel[1] >= 1 && stride[0] >= 1 && stride[1] >= 1 && pad[0] >= 0 &&
                        pad[1] >= 0 && pad[2] >= 0 && pad[3] >= 0,
                    "Kernel, stride or pad items are incorrect.");
    const Shape &s = input.shape;
    detail::require(s[3] + pad[0] + pad[2] >= kernel[0] && s[4] + pad[1] + pad[3] >= kernel[1],
                    "Input and kernel shapes are not compatible.");
    const Size oh = (s[3] + pad[0] + pad[2] - kernel[0]) / stride[0] + 1;
    const Size ow = (s[4] + pad[1] + pad[3] - kernel[1]) / stride[1] + 1;
    detail::require(oh > 0 && ow > 0, "Input and kernel shapes are not compatible.");
    const Size cap = std::max<Size>(1, std::min<Size>(input.capacity(), s[0] * s[2] * oh * ow));
    SparseTensor out({s[0], s[1], s[2], oh, ow}, cap);
    const auto k2 = kernel.get(), s2 = stride.get();
    const auto p = detail::pad4(pad);
    detail::Scratch ws(spk_sparse_pool_workspace(s[0], s[2], oh, ow, input.capacity()));
    detail::check(spk_sparse_pool(input.offsets.data<int64_t>(), input.events.data<uint32_t>(), input.capacity(), s[0],
                                  s[1], s[2], s[3], s[4], k2.data(), s2.data(), p.data(), oh, ow,
                                  out.offsets.data<int64_t>(), out.events.data<uint32_t>(), out.capacity(), ws.ptr,
                                  ws.bytes, stream()),
                  "Sparse::pool");
    return out;
}

/* Per pixel only the channel of its first event survives
 * (sparse/inhibit.cpp:37-65). */
inline SparseTensor inhibit(SparseTensor input)
{
    const Shape &s = input.shape;
    SparseTensor out(s, input.capacity());
    detail::Scratch ws(spk_sparse_inhibit_workspace(s[0], s[3], s[4], input.capacity()));
    detail::check(spk_sparse_inhibit(input.offsets.data<int64_t>(), input.events.data<uint32_t>(), input.capacity(),
                                     s[0], s[1], s[2], s[3], s[4], out.offsets.data<int64_t>(),
                                     out.events.data<uint32_t>(), out.capacity(), ws.ptr, ws.bytes, stream()),
                  "Sparse::inhibit");
    return out;
}

/* Winners in (step, list) order outside every accepted box
 * (sparse/wta.cpp:44-95; waits for the stream). */
inline Winners convwta(SparseTensor input, Expand2 radius, Size count)
{
    detail::require(radius[0] >= 0 && radius[1] >= 0, "Radius items are incorrect.");
    detail::require(count > 0, "Winners count can't be less than 1.");
    const Shape &s = input.shape;
    Tensor rec(Type::I32, {s[0], count, 5}), cnt(Type::I32, {s[0]});
    const auto r2 = radius.get();
    detail::check(spk_sparse_convwta(input.offsets.data<int64_t>(), input.events.data<uint32_t>(), s[0], s[1], s[2],
                                     s[3], s[4], r2.data(), count, rec.data<int32_t>(), cnt.data<int32_t>(), stream()),
                  "Sparse::convwta");
    return detail::winners_from(rec, cnt, count);
}
}  // namespace Sparse

/* 2D convolution module with STDP (opers.h:378-456, cpu/stdp.cpp:99-169). */
class Conv
{
    Expand2 _stride;
    Expand4 _pad;

public:
    Tensor kernel;  // F32 [Cout, Cin, KH, KW]
    std::vector<STDPConfig> stdpconfig;
    int precision = SPK_CONV_FP32;  // SPK_CONV_BF16X2 / X3: the tensor-core paths

    Conv() {}
    Conv(Size input, Size output, Expand2 kernel_, Expand2 stride = 1, Expand4 pad = 0, F64 mean = .5, F64 std = .02)
        : _stride(stride), _pad(pad)
    {
        detail::require(input > 0 && output > 0, "Input or output channels can't be less than 1.");
        detail::require(kernel_[0] > 0 && kernel_[1] > 0 && stride[0] > 0 && stride[1] > 0 && pad[0] >= 0 &&
                            pad[1] >= 0 && pad[2] >= 0 && pad[3] >= 0,
                        "Kernel, stride or pad items are incorrect.");
        const Size n = output * input * kernel_[0] * kernel_[1];
        std::vector<double> w(static_cast<size_t>(n));
        detail::check(spk_normal_kernel(w.data(), n, mean, std), "Conv kernel");
        std::vector<float> f(w.begin(), w.end());
        kernel = Tensor::from_host(f.data(), Type::F32, {output, input, kernel_[0], kernel_[1]});
    }

    Expand2 stride() const { return _stride; }
    Expand4 pad() const { return _pad; }

    Tensor operator()(Tensor input)
    {
        detail::require(kernel.valid(), "Conv is not initialized.");
        return conv(input, kernel, _stride, _pad, precision);
    }

    /* The event-list form: incremental convolution and fire (opers.h:436). */
    SparseTensor operator()(SparseTensor input, F64 threshold)
    {
        detail::require(kernel.valid(), "Conv is not initialized.");
        return Sparse::conv(input, kernel, threshold, _stride, _pad);
    }

    /* STDP from event lists, F32 update arithmetic (opers.h:450,
     * sparse/stdp.cpp:41-133). */
    void stdp(SparseTensor input, const Winners &winners)
    {
        detail::require(!stdpconfig.empty(), "At least one STDP Config must be given.");
        const Shape &s = input.shape;
        detail::require(kernel.shape(1) == s[2], "Input and kernel channels are not compatible.");
        for (const auto &v : winners)
            for (const auto &x : v)
                detail::require(x.c >= 0 && x.c < Size(stdpconfig.size()), "Winner STDP config index out of range.");
        Size count = 0;
        auto rc = detail::winners_to(winners, s[0], count);
        const auto cfg = detail::configs(stdpconfig);
        const auto p = detail::pad4(_pad);
        detail::Scratch ws(spk_sparse_stdp_workspace(s[0], count, s[2], s[3], s[4], kernel.shape(2), kernel.shape(3),
                                                     p.data()));
        detail::check(spk_sparse_stdp(input.offsets.data<int64_t>(), input.events.data<uint32_t>(), s[0], s[1], s[2],
                                      s[3], s[4], kernel.data<float>(), kernel.shape(0), kernel.shape(2),
                                      kernel.shape(3), cfg.data(), Size(stdpconfig.size()), rc.first.data<int32_t>(),
                                      rc.second.data<int32_t>(), count, p.data(), ws.ptr, ws.bytes, stream()),
                      "Conv::stdp");
        synchronize();  // the host winner arrays are freed on return
    }

    /* input [B, T, Cin, H, W] spikes, output [B, T, Cout, OH, OW] spikes. */
    void stdp(Tensor input, const Winners &winners, Tensor output)
    {
        detail::require(!stdpconfig.empty(), "At least one STDP Config must be given.");
        detail::require(input.dims() == 5 && output.dims() == 5, "Input and output dimensions must be 5.");
        const Shape s = input.shape(), o = output.shape();
        for (const auto &v : winners)
            for (const auto &x : v)
                detail::require(x.c >= 0 && x.c < Size(stdpconfig.size()), "Winner STDP config index out of range.");
        Size count = 0;
        auto rc = detail::winners_to(winners, s[0], count);
        const auto cfg = detail::configs(stdpconfig);
        const auto p = detail::pad4(_pad);
        detail::Scratch ws(spk_rank_convstdp_workspace(s[0], count, s[2], s[3], s[4], kernel.shape(2), kernel.shape(3)));
        detail::check(spk_rank_convstdp(input.data(), detail::dt(input.type()), s[0], s[1], s[2], s[3], s[4],
                                        kernel.data<float>(), kernel.shape(0), kernel.shape(2), kernel.shape(3),
                                        output.data(), o[3], o[4], cfg.data(), Size(stdpconfig.size()),
                                        rc.first.data<int32_t>(), rc.second.data<int32_t>(), count, _stride[0],
                                        _stride[1], p.data(), ws.ptr, ws.bytes, stream()),
                      "Conv::stdp");
        synchronize();  // the host winner arrays are freed on return
    }
};

/* Fully connected module with STDP and the target-rule backward
 * (opers.h:457-518, cpu/fc.cpp, cpu/stdp.cpp:42-97, cpu/backprop.cpp:105-160). */
class FC
{
public:
    Tensor kernel;  // F32 [O, I]
    std::vector<STDPConfig> stdpconfig;
    BPConfig bpconfig;

    FC() {}
    FC(Size input, Size output, F64 mean = .5, F64 std = .02)
    {
        detail::require(input > 0 && output > 0, "Input and output sizes can't be less than 1.");
        const Size n = output * input;
        std::vector<double> w(static_cast<size_t>(n));
        detail::check(spk_normal_kernel(w.data(), n, mean, std), "FC kernel");
        std::vector<float> f(w.begin(), w.end());
        kernel = Tensor::from_host(f.data(), Type::F32, {output, input});
    }

    Tensor operator()(Tensor input, Tensor output, bool sign = false)
    {
        detail::require(kernel.valid(), "FC is not initialized.");
        return fc(input, kernel, output, sign);
    }
    Tensor operator()(Tensor input, bool sign = false)
    {
        detail::require(kernel.valid(), "FC is not initialized.");
        return fc(input, kernel, sign);
    }

    /* input [B, T, I] spikes, output [B, T, O] spikes. */
    void stdp(Tensor input, const Winners &winners, Tensor output)
    {
        detail::require(!stdpconfig.empty(), "At least one STDP Config must be given.");
        detail::require(input.dims() == 3 && output.dims() == 3, "Input and output dimensions must be 3.");
        const Shape s = input.shape(), o = output.shape();
        detail::require(o[0] == s[0] && o[1] == s[1] && o[2] == kernel.shape(0) && s[2] == kernel.shape(1),
                        "Tensor shapes are not compatible.");
        for (const auto &v : winners)
            for (const auto &x : v)
                detail::require(x.c >= 0 && x.c < Size(stdpconfig.size()), "Winner STDP config index out of range.");
        Size count = 0;
        auto rc = detail::winners_to(winners, s[0], count);
        const auto cfg = detail::configs(stdpconfig);
        detail::Scratch ws(spk_rank_fcstdp_workspace(s[0], s[1], s[2]));
        detail::check(spk_rank_fcstdp(input.data(), detail::dt(input.type()), s[0], s[1], s[2], kernel.data<float>(),
                                      kernel.shape(0), output.data(), cfg.data(), Size(stdpconfig.size()),
                                      rc.first.data<int32_t>(), rc.second.data<int32_t>(), count, ws.ptr, ws.bytes,
                                      stream()),
                      "FC::stdp");
        synchronize();  // the host winner arrays are freed on return
    }

    /* input [B, I], output and grad [B, O] F32: updates the kernel and
     * bpconfig.sfactor and writes next [B, I], the gradient for the layer
     * below (waits for the stream). */
    Tensor backward(Tensor input, Tensor output, Tensor grad, Tensor next)
    {
        detail::require(kernel.valid(), "FC is not initialized.");
        const Size no = kernel.shape(0), ni = kernel.shape(1);
        detail::require(input.type() == Type::F32 && output.type() == Type::F32 && grad.type() == Type::F32 &&
                            next.type() == Type::F32,
                        "FC::backward takes F32 tensors.");
        const Size b = input.dims() > 0 ? input.shape(0) : 0;
        detail::require(input.numel() == b * ni && output.numel() == b * no && grad.numel() == b * no &&
                            next.numel() == b * ni,
                        "Tensor shapes are not compatible.");
        float bp[4] = {bpconfig.sfactor, bpconfig.lrate, bpconfig.lrf, bpconfig.lambda};
        detail::Scratch ws(spk_fcbackward_workspace(no, ni));
        detail::check(spk_fcbackward(kernel.data<float>(), no, ni, input.data<float>(), output.data<float>(),
                                     grad.data<float>(), next.data<float>(), b, bp, ws.ptr, ws.bytes, stream()),
                      "FC::backward");
        bpconfig.sfactor = bp[0];
        return next;
    }
    Tensor backward(Tensor input, Tensor output, Tensor grad)
    {
        Tensor next(Type::F32, input.shape());
        return backward(input, output, grad, next);
    }
};

/* ---- the fused layer (spyker_b200 only) ------------------------------------ */

struct LayerOutput
{
    Tensor spikes;    // U8 [B, T, Cout, OH, OW]
    Winners winners;  // convwta of the inhibited potentials
    Tensor pooled;    // U8 [B, T, Cout, OH / py, OW / px] when a pool window is given
};

/* spikes = fire(out), winners = convwta(out, radius, count) and, with a pool
 * window, pooled = pool(spikes, window) for out = inhibit(threshold(conv(input),
 * threshold)): one tensor-core kernel on the BF16 precisions (the potentials
 * never reach memory), else the ops one by one. */
inline LayerOutput conv_fire_wta(Tensor input, Conv &layer, F64 threshold, Expand2 radius, Size count,
                                 Expand2 pool_window = 0)
{
    detail::require(input.dims() == 5, "Input dimensions must be 5.");
    detail::require(count >= 0 && radius[0] >= 0 && radius[1] >= 0, "Winners count or radius are incorrect.");
    const Shape s = input.shape();
    const Size cout = layer.kernel.shape(0), cin = s[2], kh = layer.kernel.shape(2), kw = layer.kernel.shape(3);
    const Expand2 st = layer.stride();
    const Expand4 pd = layer.pad();
    const auto p = detail::pad4(pd);
    const bool pooled = pool_window[0] > 0 && pool_window[1] > 0;
    size_t nb = 0;
    bool fused = layer.precision != SPK_CONV_FP32 && input.type() == Type::U8 && s[1] <= 32 && cout >= 2;
    if (fused)
    {
        Size tp = 1;
        while (tp < s[1]) tp <<= 1;
        nb = spk_conv_fire_wta_workspace(s[0], s[1], cin, s[3], s[4], cout, kh, kw, st[0], st[1], p.data(),
                                         layer.precision);
        fused = nb > 0 && s[1] * cout * (128 / tp) <= 32768;
    }
    LayerOutput r;
    if (!fused)
    {
        Tensor out = inhibit(Spyker::threshold(layer(input), threshold));
        r.spikes = fire(out);
        r.winners = count > 0 ? convwta(out, radius, count) : Winners(size_t(s[0]));
        if (pooled) r.pooled = pool(r.spikes, pool_window);
        return r;
    }
    const Size oh = (s[3] + pd[0] + pd[2] - kh) / st[0] + 1, ow = (s[4] + pd[1] + pd[3] - kw) / st[1] + 1;
    r.spikes = Tensor(Type::U8, {s[0], s[1], cout, oh, ow});
    if (pooled) r.pooled = Tensor(Type::U8, {s[0], s[1], cout, oh / pool_window[0], ow / pool_window[1]});
    Tensor rec, cnt;
    if (count > 0) rec = Tensor(Type::I32, {s[0], count, 5}), cnt = Tensor(Type::I32, {s[0]});
    detail::Scratch ws(nb);
    detail::check(spk_conv_fire_wta(input.data(), SPK_U8, layer.kernel.data<float>(), s[0], s[1], cin, s[3], s[4], cout,
                                    kh, kw, st[0], st[1], p.data(), threshold, 0.0, 0.0, 0.0, radius[0], radius[1],
                                    count, 0.0, r.spikes.data<uint8_t>(),
                                    count > 0 ? rec.data<int32_t>() : nullptr, count > 0 ? cnt.data<int32_t>() : nullptr,
                                    pooled ? pool_window[0] : 0, pooled ? pool_window[1] : 0,
                                    pooled ? r.pooled.data<uint8_t>() : nullptr, layer.precision, ws.ptr, ws.bytes,
                                    stream()),
                  "conv_fire_wta");
    r.winners = count > 0 ? detail::winners_from(rec, cnt, count) : Winners(size_t(s[0]));
    return r;
}
}  // namespace Spyker

#endif
