// Test infrastructure, not product code.
//
// C-ABI shim over the UNMODIFIED reference CPU backend (Spyker's
// src/spyker/cpu/*.cpp and src/spyker/sparse/*.cpp), compiled from the
// reference sources by oracle/Makefile into oracle/_ref/libspyker_ref.so.
// It exposes exactly the same `orc_*` entry points as the restatement in
// oracle/spyker_oracle.cpp, so the two can be compared call for call.
//
// The reference's DNNL/BLAS submodules are empty, so its cpu/conv.cpp and
// cpu/fc.cpp cannot produce numbers (they throw, cpu/conv.cpp:235-240,
// cpu/fc.cpp:132-136).  This file therefore supplies `cpu_conv`, `cpu_fc`,
// `cpu_signfc` and their cache-clear hooks as FP64 direct loops (the
// semantics of shape.cpp:35-50 and cpu/conv.cpp:58-75: NCHW
// cross-correlation, zero pad (top, left, bottom, right), stride), result
// rounded once to the output type.  Every other op runs the reference code.

#include <spyker/impl.h>
#include <spyker/cpu/base.h>
#include <spyker/helper/csv.h>
#include <spyker/helper/mnist.h>
#include <spyker/shape.h>

#include <omp.h>

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace Spyker;
using namespace Spyker::Core;

namespace
{
thread_local std::string g_error;

template <typename F>
int guard(F &&f)
{
    try
    {
        f();
        return 0;
    }
    catch (const std::exception &e)
    {
        g_error = e.what();
        return 1;
    }
}

Type ty(int code) { return Type(code); }

template <typename T>
double load(const void *p, int64_t i)
{
    return double(((const T *)p)[i]);
}

double loadd(const void *p, Type t, int64_t i)
{
    switch (t)
    {
    case Type::U8: return load<uint8_t>(p, i);
    case Type::I8: return load<int8_t>(p, i);
    case Type::U16: return load<uint16_t>(p, i);
    case Type::I16: return load<int16_t>(p, i);
    case Type::I32: return load<int32_t>(p, i);
    case Type::U32: return load<uint32_t>(p, i);
    case Type::I64: return load<int64_t>(p, i);
    case Type::U64: return double(((const uint64_t *)p)[i]);
    case Type::F32: return load<float>(p, i);
    case Type::F64: return load<double>(p, i);
    default: throw std::runtime_error("unsupported type in FP64 shim");
    }
}

void stored(void *p, Type t, int64_t i, double v)
{
    switch (t)
    {
    case Type::F32: ((float *)p)[i] = float(v); break;
    case Type::F64: ((double *)p)[i] = v; break;
    default: throw std::runtime_error("FP64 shim writes only F32/F64 outputs");
    }
}

Winners to_winners(const int64_t *w, const int64_t *counts, int64_t b, int64_t count)
{
    Winners out(b);
    for (int64_t i = 0; i < b; ++i)
        for (int64_t j = 0; j < counts[i]; ++j)
        {
            const int64_t *e = w + (i * count + j) * 5;
            out[i].push_back(Winner{e[0], e[1], e[2], e[3], e[4]});
        }
    return out;
}

void from_winners(const Winners &ws, int64_t count, int64_t *w, int64_t *counts)
{
    for (size_t i = 0; i < ws.size(); ++i)
    {
        counts[i] = int64_t(ws[i].size());
        for (size_t j = 0; j < ws[i].size() && int64_t(j) < count; ++j)
        {
            int64_t *e = w + (int64_t(i) * count + j) * 5;
            e[0] = ws[i][j].c, e[1] = ws[i][j].t, e[2] = ws[i][j].z, e[3] = ws[i][j].y, e[4] = ws[i][j].x;
        }
    }
}

std::vector<STDPConfig> to_configs(const double *c, int64_t n)
{
    std::vector<STDPConfig> out;
    for (int64_t i = 0; i < n; ++i)
        out.push_back(STDPConfig(c[i * 5 + 0], c[i * 5 + 1], c[i * 5 + 2] != 0, c[i * 5 + 3], c[i * 5 + 4]));
    return out;
}

// Event lists cross the C boundary as offsets[u*t+1] (int64) plus packed
// (z, y, x) u8 triples.
Sparse5 to_sparse(const int64_t *offsets, const uint8_t *zyx, int64_t u, int64_t t, int64_t z, int64_t y, int64_t x)
{
    Sparse5 s = sparse_alloc(Len5(u, t, z, y, x));
    for (int64_t i = 0; i < u * t; ++i)
        for (int64_t k = offsets[i]; k < offsets[i + 1]; ++k)
            s.data[i].add(Spridx(zyx[k * 3 + 0], zyx[k * 3 + 1], zyx[k * 3 + 2]));
    return s;
}

void from_sparse(Sparse5 s, int64_t **offsets, uint8_t **zyx)
{
    int64_t n = s.u * s.t, total = 0;
    *offsets = (int64_t *)malloc(sizeof(int64_t) * (n + 1));
    for (int64_t i = 0; i < n; ++i) (*offsets)[i] = total, total += s.data[i].size;
    (*offsets)[n] = total;
    *zyx = (uint8_t *)malloc(total * 3 + 1);
    for (int64_t i = 0; i < n; ++i)
        for (int64_t k = 0; k < s.data[i].size; ++k)
        {
            Spridx e = s.data[i].data[k];
            uint8_t *d = *zyx + ((*offsets)[i] + k) * 3;
            d[0] = e.z, d[1] = e.y, d[2] = e.x;
        }
}
}  // namespace

// ---------------------------------------------------------------------------
// FP64 replacements for the oneDNN/BLAS-only entry points of the reference.
// ---------------------------------------------------------------------------
namespace Spyker
{
namespace Core
{
void cpu_conv(Dyn4 input, Dyn4 kernel, Dyn4 output, Len2 stride, Len4 pad)
{
    const int64_t N = input.t, C = input.z, H = input.y, W = input.x;
    const int64_t O = kernel.t, KH = kernel.y, KW = kernel.x;
    const int64_t OH = output.y, OW = output.x;
#pragma omp parallel for collapse(2)
    for (int64_t n = 0; n < N; ++n)
        for (int64_t o = 0; o < O; ++o)
            for (int64_t i = 0; i < OH; ++i)
                for (int64_t j = 0; j < OW; ++j)
                {
                    double acc = 0;
                    for (int64_t c = 0; c < C; ++c)
                        for (int64_t ky = 0; ky < KH; ++ky)
                        {
                            int64_t yy = i * stride.y + ky - pad.t;
                            if (yy < 0 || yy >= H) continue;
                            for (int64_t kx = 0; kx < KW; ++kx)
                            {
                                int64_t xx = j * stride.x + kx - pad.z;
                                if (xx < 0 || xx >= W) continue;
                                acc += loadd(input.data, input.type, ((n * C + c) * H + yy) * W + xx) *
                                       loadd(kernel.data, kernel.type, ((o * C + c) * KH + ky) * KW + kx);
                            }
                        }
                    stored(output.data, output.type, ((n * O + o) * OH + i) * OW + j, acc);
                }
}
void cpu_conv_clear() {}

static void fc64(Dyn3 input, Dyn2 kernel, Dyn3 output, bool sign)
{
    const int64_t B = input.z * input.y, I = input.x, O = kernel.y;
#pragma omp parallel for
    for (int64_t b = 0; b < B; ++b)
        for (int64_t o = 0; o < O; ++o)
        {
            double acc = 0;
            for (int64_t i = 0; i < I; ++i)
            {
                double w = loadd(kernel.data, kernel.type, o * I + i);
                if (sign) w = w > 0 ? 1 : (w < 0 ? -1 : 0);
                acc += loadd(input.data, input.type, b * I + i) * w;
            }
            stored(output.data, output.type, b * O + o, acc);
        }
}
void cpu_fc(Dyn3 input, Dyn2 kernel, Dyn3 output) { fc64(input, kernel, output, false); }
void cpu_signfc(Dyn3 input, Dyn2 kernel, Dyn3 output) { fc64(input, kernel, output, true); }
void cpu_fc_clear() {}
}  // namespace Core
}  // namespace Spyker

// ---------------------------------------------------------------------------
// orc_* entry points (identical ABI to oracle/spyker_oracle.cpp).
// ---------------------------------------------------------------------------
extern "C" {

const char *orc_last_error() { return g_error.c_str(); }
const char *orc_kind() { return "reference"; }
void orc_free(void *p) { free(p); }

int orc_rank_code(const void *in, int itype, void *out, int otype, int64_t b, int64_t t, int64_t x, int sort)
{
    return guard([&] { cpu_rank_code(Dyn2((void *)in, ty(itype), b, x), Dyn3(out, ty(otype), b, t, x), sort != 0); });
}

int orc_threshold(void *data, int type, int64_t n, double thr, double value)
{
    return guard([&] { cpu_threshold(Dyn1(data, ty(type), n), Scalar(thr), Scalar(value)); });
}

int orc_rank_infinite(void *data, int type, int64_t b, int64_t t, int64_t x, double value)
{
    return guard([&] { cpu_rank_infinite(Dyn3(data, ty(type), b, t, x), Scalar(value)); });
}

int orc_rank_fire(const void *in, int itype, void *out, int otype, int64_t n, double thr)
{
    return guard([&] { cpu_rank_fire(Dyn1((void *)in, ty(itype), n), Dyn1(out, ty(otype), n), Scalar(thr)); });
}

int orc_rank_gather(const void *in, int itype, void *out, int otype, int64_t b, int64_t t, int64_t x, double thr)
{
    return guard(
        [&] { cpu_rank_gather(Dyn3((void *)in, ty(itype), b, t, x), Dyn2(out, ty(otype), b, x), Scalar(thr)); });
}

int orc_rank_scatter(const void *in, int itype, void *out, int otype, int64_t b, int64_t t, int64_t x)
{
    return guard([&] { cpu_rank_scatter(Dyn2((void *)in, ty(itype), b, x), Dyn3(out, ty(otype), b, t, x)); });
}

int orc_pad(const void *in, void *out, int type, int64_t n, int64_t h, int64_t w, const int64_t *pad4, double value)
{
    return guard([&] {
        int64_t oh = h + pad4[0] + pad4[2], ow = w + pad4[1] + pad4[3];
        cpu_pad(Dyn3((void *)in, ty(type), n, h, w), Dyn3(out, ty(type), n, oh, ow),
                Len4(pad4[0], pad4[1], pad4[2], pad4[3]), Scalar(value));
    });
}

int orc_rank_pool(const void *in, void *out, int type, int64_t n, int64_t c, int64_t h, int64_t w, int64_t oh,
                  int64_t ow, const int64_t *kernel2, const int64_t *stride2, const int64_t *pad4)
{
    return guard([&] {
        cpu_rank_pool(Dyn4((void *)in, ty(type), n, c, h, w), Dyn4(out, ty(type), n, c, oh, ow),
                      Len2(kernel2[0], kernel2[1]), Len2(stride2[0], stride2[1]),
                      Len4(pad4[0], pad4[1], pad4[2], pad4[3]));
    });
}

int orc_rank_inhibit(void *data, int type, int64_t b, int64_t t, int64_t c, int64_t x, double thr)
{
    return guard([&] { cpu_rank_inhibit(Dyn4(data, ty(type), b, t, c, x), Scalar(thr)); });
}

int orc_rank_convwta(const void *in, int type, int64_t b, int64_t t, int64_t c, int64_t h, int64_t w,
                     const int64_t *radius2, int64_t count, double thr, int64_t *winners, int64_t *counts)
{
    return guard([&] {
        Winners ws = cpu_rank_convwta(Dyn5((void *)in, ty(type), b, t, c, h, w), Len2(radius2[0], radius2[1]), count,
                                      Scalar(thr));
        from_winners(ws, count, winners, counts);
    });
}

int orc_rank_fcwta(const void *in, int type, int64_t b, int64_t t, int64_t n, int64_t radius, int64_t count,
                   double thr, int64_t *winners, int64_t *counts)
{
    return guard([&] {
        Winners ws = cpu_rank_fcwta(Dyn3((void *)in, ty(type), b, t, n), radius, count, Scalar(thr));
        from_winners(ws, count, winners, counts);
    });
}

int orc_rank_convstdp(const void *in, int itype, int64_t b, int64_t t, int64_t cin, int64_t h, int64_t w,
                      void *kernel, int ktype, int64_t cout, int64_t kh, int64_t kw, const void *out, int64_t oh,
                      int64_t ow, const double *configs, int64_t nconf, const int64_t *winners,
                      const int64_t *counts, int64_t count, const int64_t *stride2, const int64_t *pad4)
{
    return guard([&] {
        cpu_rank_convstdp(Dyn5((void *)in, ty(itype), b, t, cin, h, w), Dyn4(kernel, ty(ktype), cout, cin, kh, kw),
                          Dyn5((void *)out, ty(itype), b, t, cout, oh, ow), to_configs(configs, nconf),
                          to_winners(winners, counts, b, count), Len2(stride2[0], stride2[1]),
                          Len4(pad4[0], pad4[1], pad4[2], pad4[3]));
    });
}

int orc_rank_fcstdp(const void *in, int itype, int64_t b, int64_t t, int64_t i, void *kernel, int ktype, int64_t o,
                    const void *out, const double *configs, int64_t nconf, const int64_t *winners,
                    const int64_t *counts, int64_t count)
{
    return guard([&] {
        cpu_rank_fcstdp(Dyn3((void *)in, ty(itype), b, t, i), Dyn2(kernel, ty(ktype), o, i),
                        Dyn3((void *)out, ty(itype), b, t, o), to_configs(configs, nconf),
                        to_winners(winners, counts, b, count));
    });
}

int orc_conv(const void *in, int itype, const void *kernel, int ktype, void *out, int otype, int64_t n, int64_t cin,
             int64_t h, int64_t w, int64_t cout, int64_t kh, int64_t kw, int64_t oh, int64_t ow,
             const int64_t *stride2, const int64_t *pad4)
{
    return guard([&] {
        cpu_conv(Dyn4((void *)in, ty(itype), n, cin, h, w), Dyn4((void *)kernel, ty(ktype), cout, cin, kh, kw),
                 Dyn4(out, ty(otype), n, cout, oh, ow), Len2(stride2[0], stride2[1]),
                 Len4(pad4[0], pad4[1], pad4[2], pad4[3]));
    });
}

int orc_fc(const void *in, int itype, const void *kernel, int ktype, void *out, int otype, int64_t b, int64_t t,
           int64_t i, int64_t o, int sign)
{
    return guard([&] {
        Dyn3 a((void *)in, ty(itype), b, t, i);
        Dyn2 k((void *)kernel, ty(ktype), o, i);
        Dyn3 c(out, ty(otype), b, t, o);
        if (sign)
            cpu_signfc(a, k, c);
        else
            cpu_fc(a, k, c);
    });
}

// DoG/LoG kernels are [2, F, KH, KW]; Gabor kernels are [F, KH, KW].
// Input [N, H, W] single-channel planes (the caller folds channels into N,
// as opers.cpp:251-255 does); output [N, F (or 2F for LoG), OH, OW].
int orc_filter(int which, const void *in, const void *kernel, void *out, int type, int64_t n, int64_t h, int64_t w,
               int64_t f, int64_t kh, int64_t kw, int64_t oh, int64_t ow, const int64_t *pad4)
{
    return guard([&] {
        Dyn4 a((void *)in, ty(type), n, 1, h, w);
        Len4 p(pad4[0], pad4[1], pad4[2], pad4[3]);
        if (which == 0) cpu_dog(a, Dyn4((void *)kernel, ty(type), 2 * f, 1, kh, kw), Dyn4(out, ty(type), n, f, oh, ow), p);
        if (which == 1) cpu_gabor(a, Dyn4((void *)kernel, ty(type), f, 1, kh, kw), Dyn4(out, ty(type), n, f, oh, ow), p);
        if (which == 2)
            cpu_log(a, Dyn4((void *)kernel, ty(type), 2 * f, 1, kh, kw), Dyn4(out, ty(type), n, 2 * f, oh, ow), p);
    });
}

int orc_gaussian_kernel(double *kernel, int64_t size, double std)
{
    return guard([&] { gaussian_kernel(Vec2<F64>(kernel, size, size), std); });
}

int orc_gabor_kernel(double *kernel, int64_t size, double sigma, double theta, double gamma, double lambda, double psi)
{
    return guard([&] { gabor_kernel(Vec2<F64>(kernel, size, size), sigma, theta, gamma, lambda, psi); });
}

int orc_log_kernel(double *kernel, int64_t size, double std)
{
    return guard([&] { log_kernel(Vec2<F64>(kernel, size, size), std); });
}

int orc_backward(const void *in, void *out, int type, const int64_t *target, int64_t b, int64_t n, int64_t time,
                 double gamma)
{
    return guard([&] {
        cpu_backward(Dyn2((void *)in, ty(type), b, n), Dyn2(out, ty(type), b, n),
                     Dyn1((void *)target, Type::I64, b), time, Scalar(gamma));
    });
}

int orc_labelize(const void *in, int type, int64_t *out, int64_t b, int64_t t, int64_t n, double thr)
{
    return guard(
        [&] { cpu_labelize(Dyn3((void *)in, ty(type), b, t, n), Dyn1(out, Type::I64, b), Scalar(thr)); });
}

int orc_fcbackward(float *kernel, int64_t o, int64_t i, const void *in, const void *out, const void *grad, void *next,
                   int type, int64_t b, float *bp)
{
    return guard([&] {
        BPConfig config(bp[0], bp[1], bp[2], bp[3]);
        cpu_fcbackward(Dyn2(kernel, Type::F32, o, i), Dyn2((void *)in, ty(type), b, i), Dyn2((void *)out, ty(type), b, o),
                       Dyn2((void *)grad, ty(type), b, o), Dyn2(next, ty(type), b, i), config);
        bp[0] = config.sfactor;
    });
}

// ----------------------------- sparse path ---------------------------------

int orc_sparse_code(const void *in, int itype, int64_t u, int64_t c, int64_t h, int64_t w, int64_t t, int sort,
                    int64_t **offsets, uint8_t **zyx)
{
    return guard([&] {
        Sparse5 s = sparse_alloc(Len5(u, t, c, h, w));
        sparse_code(Dyn4((void *)in, ty(itype), u, c, h, w), s, sort != 0);
        from_sparse(s, offsets, zyx);
        sparse_dealloc(s);
    });
}

int orc_sparse_from_dense(const void *in, int itype, int64_t u, int64_t t, int64_t c, int64_t h, int64_t w,
                          double thr, int64_t **offsets, uint8_t **zyx)
{
    return guard([&] {
        Sparse5 s = sparse_alloc(Len5(u, t, c, h, w));
        sparse_convert(Dyn5((void *)in, ty(itype), u, t, c, h, w), s, Scalar(thr));
        from_sparse(s, offsets, zyx);
        sparse_dealloc(s);
    });
}

int orc_sparse_to_dense(const int64_t *offsets, const uint8_t *zyx, int64_t u, int64_t t, int64_t c, int64_t h,
                        int64_t w, void *out, int otype)
{
    return guard([&] {
        Sparse5 s = to_sparse(offsets, zyx, u, t, c, h, w);
        sparse_convert(s, Dyn5(out, ty(otype), u, t, c, h, w));
        sparse_dealloc(s);
    });
}

int orc_sparse_gather(const int64_t *offsets, const uint8_t *zyx, int64_t u, int64_t t, int64_t c, int64_t h,
                      int64_t w, void *out, int otype)
{
    return guard([&] {
        Sparse5 s = to_sparse(offsets, zyx, u, t, c, h, w);
        sparse_gather(s, Dyn4(out, ty(otype), u, c, h, w));
        sparse_dealloc(s);
    });
}

int orc_sparse_conv(const int64_t *offsets, const uint8_t *zyx, int64_t u, int64_t t, int64_t c, int64_t h, int64_t w,
                    const float *kernel, int64_t cout, int64_t kh, int64_t kw, double thr, const int64_t *stride2,
                    const int64_t *pad4, int64_t oh, int64_t ow, int64_t **ooff, uint8_t **ozyx)
{
    return guard([&] {
        Sparse5 s = to_sparse(offsets, zyx, u, t, c, h, w);
        Sparse5 o = sparse_alloc(Len5(u, t, cout, oh, ow));
        sparse_conv(s, Dyn4((void *)kernel, Type::F32, cout, c, kh, kw), Scalar(thr), o, Len2(stride2[0], stride2[1]),
                    Len4(pad4[0], pad4[1], pad4[2], pad4[3]));
        from_sparse(o, ooff, ozyx);
        sparse_dealloc(s), sparse_dealloc(o);
    });
}

int orc_sparse_pad(const int64_t *offsets, const uint8_t *zyx, int64_t u, int64_t t, int64_t c, int64_t h, int64_t w,
                   const int64_t *pad4, int64_t **ooff, uint8_t **ozyx)
{
    return guard([&] {
        Sparse5 s = to_sparse(offsets, zyx, u, t, c, h, w);
        Sparse5 o = sparse_alloc(Len5(u, t, c, h + pad4[0] + pad4[2], w + pad4[1] + pad4[3]));
        sparse_pad(s, o, Len4(pad4[0], pad4[1], pad4[2], pad4[3]));
        from_sparse(o, ooff, ozyx);
        sparse_dealloc(s), sparse_dealloc(o);
    });
}

int orc_sparse_pool(const int64_t *offsets, const uint8_t *zyx, int64_t u, int64_t t, int64_t c, int64_t h, int64_t w,
                    const int64_t *kernel2, const int64_t *stride2, const int64_t *pad4, int64_t oh, int64_t ow,
                    int64_t **ooff, uint8_t **ozyx)
{
    return guard([&] {
        Sparse5 s = to_sparse(offsets, zyx, u, t, c, h, w);
        Sparse5 o = sparse_alloc(Len5(u, t, c, oh, ow));
        sparse_pool(s, o, Len2(kernel2[0], kernel2[1]), Len2(stride2[0], stride2[1]),
                    Len4(pad4[0], pad4[1], pad4[2], pad4[3]));
        from_sparse(o, ooff, ozyx);
        sparse_dealloc(s), sparse_dealloc(o);
    });
}

int orc_sparse_inhibit(const int64_t *offsets, const uint8_t *zyx, int64_t u, int64_t t, int64_t c, int64_t h,
                       int64_t w, int64_t **ooff, uint8_t **ozyx)
{
    return guard([&] {
        Sparse5 s = to_sparse(offsets, zyx, u, t, c, h, w);
        Sparse5 o = sparse_alloc(Len5(u, t, c, h, w));
        sparse_inhibit(s, o);
        from_sparse(o, ooff, ozyx);
        sparse_dealloc(s), sparse_dealloc(o);
    });
}

int orc_sparse_convwta(const int64_t *offsets, const uint8_t *zyx, int64_t u, int64_t t, int64_t c, int64_t h,
                       int64_t w, const int64_t *radius2, int64_t count, int64_t *winners, int64_t *counts)
{
    return guard([&] {
        Sparse5 s = to_sparse(offsets, zyx, u, t, c, h, w);
        Winners ws = sparse_convwta(s, Len2(radius2[0], radius2[1]), count);
        from_winners(ws, count, winners, counts);
        sparse_dealloc(s);
    });
}

int orc_sparse_stdp(const int64_t *offsets, const uint8_t *zyx, int64_t u, int64_t t, int64_t c, int64_t h, int64_t w,
                    float *kernel, int64_t cout, int64_t kh, int64_t kw, const double *configs, int64_t nconf,
                    const int64_t *winners, const int64_t *counts, int64_t count, const int64_t *pad4)
{
    return guard([&] {
        Sparse5 s = to_sparse(offsets, zyx, u, t, c, h, w);
        sparse_stdp(s, Dyn4(kernel, Type::F32, cout, c, kh, kw), to_configs(configs, nconf),
                    to_winners(winners, counts, u, count), Len4(pad4[0], pad4[1], pad4[2], pad4[3]));
        sparse_dealloc(s);
    });
}


// ---- rate coding (cpu/code.cpp:134-243, fire.cpp:84-113, time.cpp:87-92,
// pool.cpp:88-137, init.cpp:120-149) ----
int orc_rate_code(const void *in, int itype, void *out, int otype, int64_t b, int64_t t, int64_t x, int sort)
{
    return guard([&] { cpu_rate_code(Dyn2((void *)in, ty(itype), b, x), Dyn3(out, ty(otype), b, t, x), sort != 0); });
}

int orc_rate_fire(const void *in, int itype, void *out, int otype, int64_t b, int64_t t, int64_t x, double thr)
{
    return guard(
        [&] { cpu_rate_fire(Dyn3((void *)in, ty(itype), b, t, x), Dyn3(out, ty(otype), b, t, x), Scalar(thr)); });
}

int orc_rate_gather(const void *in, int itype, void *out, int otype, int64_t b, int64_t t, int64_t x)
{
    return guard(
        [&] { cpu_rate_gather(Dyn3((void *)in, ty(itype), b, t, x), Dyn2(out, ty(otype), b, x), Scalar(0.0)); });
}

int orc_rate_pool(const void *in, const void *rates, int type, int rtype, void *out, int64_t b, int64_t t, int64_t c,
                  int64_t h, int64_t w, int64_t oh, int64_t ow, const int64_t *kernel2, const int64_t *stride2)
{
    return guard([&] {
        cpu_rate_pool(Dyn5((void *)in, ty(type), b, t, c, h, w), Dyn4((void *)rates, ty(rtype), b, c, h, w),
                      Dyn5(out, ty(type), b, t, c, oh, ow), Len2(kernel2[0], kernel2[1]), Len2(stride2[0], stride2[1]),
                      Len4(0, 0, 0, 0));
    });
}

// The interval table [time][bins] (rows in the reference's shuffled order).
int orc_poisson_table(int64_t time, int64_t bins, uint16_t *out)
{
    return guard([&] {
        auto v = poisson_create(time, bins);
        std::memcpy(out, v.data, size_t(time * bins) * sizeof(uint16_t));
        CPU::deinit(v);
    });
}

// ---- reference-only: the data helpers (helper/csv.cpp, helper/mnist.cpp) ----
// CSV rows read by Helper::CSV after skip(skip): fields joined by 0x1f, each
// row ended by 0x1e, copied into out when cap allows; *len = bytes needed.
int orc_ref_csv(const char *path, const char *delim, int64_t skip, int64_t max_rows, char *out, int64_t cap,
                int64_t *len, int64_t *skipped)
{
    return guard([&] {
        Helper::CSV csv(path, delim);
        *skipped = int64_t(csv.skip(Size(skip)));
        std::string buf;
        std::vector<std::string> row;
        for (int64_t r = 0; r < max_rows && csv.readline(row); ++r)
        {
            for (size_t i = 0; i < row.size(); ++i) buf += (i ? "\x1f" : "") + row[i];
            buf += '\x1e';
        }
        *len = int64_t(buf.size());
        if (*len <= cap) std::memcpy(out, buf.data(), buf.size());
    });
}

// An IDX file through Helper::mnistLabel / mnistData: *ndim = 0 for the
// empty tensor they return on failure, else the shape and (when cap allows)
// the bytes.
int orc_ref_idx(const char *path, int64_t labels, uint8_t *out, int64_t cap, int64_t *shape, int64_t *ndim)
{
    return guard([&] {
        Tensor t = labels ? Helper::mnistLabel(path) : Helper::mnistData(path);
        if (!t)
        {
            *ndim = 0;
            return;
        }
        auto s = t.shape();
        *ndim = int64_t(s.size());
        for (size_t i = 0; i < s.size(); ++i) shape[i] = int64_t(s[i]);
        if (int64_t(t.numel()) <= cap) std::memcpy(out, t.data(), size_t(t.numel()));
    });
}

// ---- reference-only: Canny and quantize (cpu/canny.cpp, cpu/fire.cpp) ----
// Canny runs on one OpenMP thread: cpu/canny.cpp:190-214 views u8 scratch
// planes of image i at byte offset i*H*W of the F32 buffers, which hold the
// F32 planes of image i/8, so images processed at once on several threads
// overwrite one another's gradients and magnitudes (the result then depends
// on the schedule); in order on one thread every overwritten plane has
// already been used.
int orc_ref_canny(const uint8_t *in, uint8_t *out, int64_t n, int64_t h, int64_t w, double low, double high)
{
    return guard([&] {
        const int threads = omp_get_max_threads();
        omp_set_num_threads(1);
        try
        {
            cpu_canny(Dyn3((void *)in, Type::U8, n, h, w), Dyn3(out, Type::U8, n, h, w), Scalar(low),
                      Scalar(high));
        }
        catch (...)
        {
            omp_set_num_threads(threads);
            throw;
        }
        omp_set_num_threads(threads);
    });
}

// cpu/zca.cpp:67-118 (ZCA fit, with the in-place transform when `transform`)
// on input [n, d] F32/F64, mean [d] and trans [d, d] of the same type.
int orc_ref_zca_fit(void *in, int type, int64_t n, int64_t d, void *mean, void *trans, double epsilon,
                    int transform)
{
    return guard([&] {
        cpu_zca_fit(Dyn2(in, ty(type), n, d), Dyn1(mean, ty(type), d), Dyn2(trans, ty(type), d, d),
                    Scalar(epsilon), transform != 0);
    });
}

// cpu/zca.cpp:107-118 (in-place ZCA transform of input [n, d])
int orc_ref_zca_trans(void *in, int type, int64_t n, int64_t d, void *mean, void *trans)
{
    return guard([&] { cpu_zca_trans(Dyn2(in, ty(type), n, d), Dyn1(mean, ty(type), d), Dyn2(trans, ty(type), d, d)); });
}

// cpu/zca.cpp:139-155 (split [n, d] -> [n, 2, d])
int orc_ref_zca_split(void *in, int type, int64_t n, int64_t d, void *out)
{
    return guard([&] { cpu_zca_split(Dyn2(in, ty(type), n, d), Dyn3(out, ty(type), n, 2, d)); });
}

int orc_ref_quantize(void *data, int type, int64_t n, double lower, double middle, double upper)
{
    return guard([&] { cpu_quantize(Dyn1(data, ty(type), n), Scalar(lower), Scalar(middle), Scalar(upper)); });
}
}  // extern "C"
