// ORACLE — test infrastructure only.  Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg may load this library, and only as the
// checker; the product never calls it.
//
// A CPU restatement, written for this project, of the algorithms of
// Spyker's CPU backend for the spiking-CNN hot path.  Every entry point
// cites the reference file:line it follows (paths inside the Spyker
// project).  Parity of this restatement is pinned by the test suite against
// the reference itself, compiled here from its own sources
// (oracle/ref_capi.cpp + oracle/Makefile -> oracle/_ref/libspyker_ref.so),
// call for call, on seeded inputs; the golden fixtures under tests/golden/
// are outputs of that reference build.
//
// Convolution / FC have no usable reference arithmetic (oneDNN and BLAS are
// absent from the reference tree), so they are computed exactly in FP64 and
// rounded once to the output type: this is the FP64 oracle for potentials.
//
// ABI: identical to oracle/ref_capi.cpp (`orc_*`), 0 = success.

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

namespace
{
thread_local std::string g_error;

// Type codes follow the reference's `enum class Type` (utils.h:96-120).
enum Ty
{
    I8 = 0,
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

// Dispatch a generic lambda over the element types the hot path uses.
template <typename F>
void dispatch(int t, F &&f)
{
    switch (t)
    {
    case I8: f(int8_t()); break;
    case I16: f(int16_t()); break;
    case I32: f(int32_t()); break;
    case I64: f(int64_t()); break;
    case U8: f(uint8_t()); break;
    case U16: f(uint16_t()); break;
    case U32: f(uint32_t()); break;
    case U64: f(uint64_t()); break;
    case F32: f(float()); break;
    case F64: f(double()); break;
    default: throw std::runtime_error("oracle: unsupported data type");
    }
}

// Reduced dispatch for multi-type kernels (spikes/potentials/weights).
template <typename F>
void dispatchR(int t, F &&f)
{
    switch (t)
    {
    case U8: f(uint8_t()); break;
    case I32: f(int32_t()); break;
    case F32: f(float()); break;
    case F64: f(double()); break;
    default: throw std::runtime_error("oracle: unsupported data type");
    }
}

template <typename T>
T lowest()
{
    return std::numeric_limits<T>::lowest();  // Limits<T>::min() of base.h:759-774
}

// Scalar conversion: the reference stores the scalar as F64 and converts with
// a C cast to the data type (utils.cpp:290-295).
template <typename T>
T scal(double v)
{
    return T(v);
}

// float -> U16 exactly as x86-64 GCC lowers `U16 x = f` (cvttss2si to int32,
// keep the low 16 bits; NaN and out-of-range give 0x80000000 -> 0).
inline uint16_t f2u16(float v)
{
    if (!(v > -2147483648.0f && v < 2147483648.0f)) return 0;
    return uint16_t(uint32_t(int32_t(v)));
}

// std::max_element semantics: first index of the maximum, NaN never
// replaces the running maximum (cpu/base.h:137-141).
template <typename T>
int64_t maxidx(const T *v, int64_t n)
{
    int64_t best = 0;
    for (int64_t i = 1; i < n; ++i)
        if (v[best] < v[i]) best = i;
    return best;
}

template <typename T>
int64_t minidx(const T *v, int64_t n)
{
    int64_t best = 0;
    for (int64_t i = 1; i < n; ++i)
        if (v[i] < v[best]) best = i;
    return best;
}

struct W5
{
    int64_t c, t, z, y, x;
};

void put_winners(const std::vector<std::vector<W5>> &ws, int64_t count, int64_t *w, int64_t *counts)
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

struct Cfg
{
    double pos, neg;
    bool stab;
    double lo, hi;
};

std::vector<Cfg> get_cfgs(const double *c, int64_t n)
{
    std::vector<Cfg> out;
    for (int64_t i = 0; i < n; ++i) out.push_back({c[i * 5], c[i * 5 + 1], c[i * 5 + 2] != 0, c[i * 5 + 3], c[i * 5 + 4]});
    return out;
}

// ------------------------------------------------------------------------
// Rank-order coding (cpu/code.cpp:42-132).  Per row of X values:
//  sort=True : order indices by value descending with std::sort (the same
//              libstdc++ algorithm as the reference, so ties resolve
//              identically); cnt = number of values strictly above the row
//              minimum (lower_bound of the last sorted element); scale =
//              F32(T + 1e-5) / cnt; time[idx[i]] = U16(i * scale).
//  sort=False: time = U16(end - scale * (x - min)), end = T + 1e-5,
//              scale = end / (max - min), F32 arithmetic.
// ------------------------------------------------------------------------
template <typename T>
void code_times(const T *in, int64_t x, int64_t time, bool sort, uint16_t *temp, std::vector<uint32_t> &index)
{
    if (sort)
    {
        index.resize(x);
        for (int64_t i = 0; i < x; ++i) index[i] = uint32_t(i);
        auto comp = [in](uint32_t i, uint32_t j) { return in[i] > in[j]; };
        std::sort(index.begin(), index.end(), comp);
        int64_t cnt = std::distance(index.begin(), std::lower_bound(index.begin(), index.end(), index[x - 1], comp));
        float scale = float(float(time) + 1e-5f) / float(cnt);
        for (int64_t i = 0; i < x; ++i) temp[index[i]] = f2u16(float(i) * scale);
    }
    else
    {
        T mn = in[0], mx = in[0];
        for (int64_t i = 0; i < x; ++i) mn = std::min(mn, in[i]), mx = std::max(mx, in[i]);
        float end = float(time) + 1e-5f;
        float scale = end / float(mx - mn);
        for (int64_t i = 0; i < x; ++i) temp[i] = f2u16(std::fma(-scale, float(in[i] - mn), end));
    }
}

template <typename I, typename O>
void rank_code(const I *in, O *out, int64_t b, int64_t t, int64_t x, bool sort)
{
#pragma omp parallel
    {
        std::vector<uint16_t> temp(x);
        std::vector<uint32_t> index;
#pragma omp for
        for (int64_t i = 0; i < b; ++i)
        {
            code_times(in + i * x, x, t, sort, temp.data(), index);
            for (int64_t s = 0; s < t; ++s)
            {
                O *od = out + (i * t + s) * x;
                for (int64_t j = 0; j < x; ++j) od[j] = O(temp[j] <= uint16_t(s));
            }
        }
    }
}

// ------------------------------------------------------------------------
// First-spike time of one neuron over a [T, stride] block: smallest t with a
// non-zero entry, T when none (cpu/stdp.cpp:42-64,99-118).
// ------------------------------------------------------------------------
template <typename T>
uint16_t first_nonzero(const T *base, int64_t t, int64_t stride)
{
    uint16_t v = uint16_t(t);
    for (int64_t i = t - 1; i >= 0; --i)
        if (base[i * stride]) v = uint16_t(i);
    return v;
}

// Soft-bound STDP update of one weight in FP64 (cpu/stdp.cpp:122-137),
// written with the fused multiply-add that GCC forms for
// `old + rate * value` under -ffp-contract=fast.
template <typename K>
void stdp_weight(K &w, bool pre_first, const Cfg &c)
{
    double old = double(w);
    double m = c.stab ? (old - c.lo) * (c.hi - old) : 1.0;
    double v = std::fma(pre_first ? c.pos : c.neg, m, old);
    w = K(std::max(c.lo, std::min(v, c.hi)));
}

// ------------------------------------------------------------------------
// WTA key (cpu/wta.cpp:40-85): per sample over a [T, X] block.
// ------------------------------------------------------------------------
template <typename T>
void wta_keys(const T *in, int64_t t, int64_t x, double thr, std::vector<float> &keyf, std::vector<uint16_t> &keyi)
{
    if (std::is_floating_point<T>::value)
    {
        T mn = in[0], mx = in[0];
        for (int64_t i = 0; i < t * x; ++i) mn = std::min(mn, in[i]), mx = std::max(mx, in[i]);
        T diff = (mx - mn) * T(2);
        T th = scal<T>(thr);
        keyf.assign(x, -FLT_MAX);
        for (int64_t i = t - 1; i >= 0; --i)
        {
            T level = T(t - i - 1);
            const T *id = in + i * x;
            for (int64_t j = 0; j < x; ++j)
                if (id[j] > th) keyf[j] = float(level + (id[j] - mn) / diff);
        }
    }
    else
    {
        keyi.assign(x, 0);
        for (int64_t i = t - 1; i >= 0; --i)
        {
            const T *id = in + i * x;
            for (int64_t j = 0; j < x; ++j)
                if (id[j]) keyi[j] = uint16_t(t - i);
        }
    }
}

template <typename S>
bool is_sentinel(S v);
template <>
bool is_sentinel<float>(float v)
{
    return std::abs(v - (-FLT_MAX)) < 1e-5f;
}
template <>
bool is_sentinel<uint16_t>(uint16_t v)
{
    return float(std::abs(int(v) - 0)) < 1e-5f;
}

template <typename S>
void convwta_rounds(std::vector<S> &key, S low, int64_t c, int64_t h, int64_t w, int64_t ry, int64_t rx, int64_t count,
                    std::vector<W5> &out)
{
    for (int64_t r = 0; r < count; ++r)
    {
        int64_t idx = maxidx(key.data(), int64_t(key.size()));
        if (is_sentinel<S>(key[idx])) break;
        int64_t len = h * w, z = idx / len, y = (idx % len) / w, x = (idx % len) % w;
        int64_t sj = std::max<int64_t>(0, y - ry), ej = std::min(h, y + ry + 1);
        int64_t sk = std::max<int64_t>(0, x - rx), ek = std::min(w, x + rx + 1);
        for (int64_t i = 0; i < c; ++i)
            for (int64_t j = sj; j < ej; ++j)
                for (int64_t k = sk; k < ek; ++k) key[(i * h + j) * w + k] = low;
        for (int64_t i = 0; i < len; ++i) key[z * len + i] = low;
        out.push_back({0, 0, z, y, x});
    }
}

template <typename S>
void fcwta_rounds(std::vector<S> &key, S low, int64_t radius, int64_t count, std::vector<W5> &out)
{
    int64_t n = int64_t(key.size());
    for (int64_t r = 0; r < count; ++r)
    {
        int64_t idx = maxidx(key.data(), n);
        if (is_sentinel<S>(key[idx])) break;
        int64_t s = std::max<int64_t>(0, idx - radius), e = std::min(n, idx + radius + 1);
        for (int64_t i = s; i < e; ++i) key[i] = low;
        out.push_back({0, 0, 0, 0, idx});
    }
}

// ------------------------------------------------------------------------
// Sparse event lists: per (sample, t) vectors of (z, y, x) u8 triples
// (base.h:493-528).
// ------------------------------------------------------------------------
struct Ev
{
    uint8_t z, y, x;
};
using Lists = std::vector<std::vector<Ev>>;

Lists get_lists(const int64_t *off, const uint8_t *zyx, int64_t n)
{
    Lists l(n);
    for (int64_t i = 0; i < n; ++i)
        for (int64_t k = off[i]; k < off[i + 1]; ++k) l[i].push_back({zyx[k * 3], zyx[k * 3 + 1], zyx[k * 3 + 2]});
    return l;
}

void put_lists(const Lists &l, int64_t **off, uint8_t **zyx)
{
    int64_t n = int64_t(l.size()), total = 0;
    *off = (int64_t *)malloc(sizeof(int64_t) * (n + 1));
    for (int64_t i = 0; i < n; ++i) (*off)[i] = total, total += int64_t(l[i].size());
    (*off)[n] = total;
    *zyx = (uint8_t *)malloc(total * 3 + 1);
    for (int64_t i = 0; i < n; ++i)
        for (size_t k = 0; k < l[i].size(); ++k)
        {
            uint8_t *d = *zyx + ((*off)[i] + int64_t(k)) * 3;
            d[0] = l[i][k].z, d[1] = l[i][k].y, d[2] = l[i][k].x;
        }
}

// Emit one event per pixel at its first-spike time, (z, y, x) order
// (sparse/code.cpp:52-61, sparse/opers.cpp:59-69).
void times_to_events(const uint16_t *tm, int64_t c, int64_t h, int64_t w, int64_t t, Lists &l, int64_t sample)
{
    for (int64_t j = 0; j < c; ++j)
        for (int64_t k = 0; k < h; ++k)
            for (int64_t q = 0; q < w; ++q)
            {
                uint16_t v = tm[(j * h + k) * w + q];
                if (v < t) l[sample * t + v].push_back({uint8_t(j), uint8_t(k), uint8_t(q)});
            }
}
}  // namespace

extern "C" {

const char *orc_last_error() { return g_error.c_str(); }
const char *orc_kind() { return "port"; }
void orc_free(void *p) { free(p); }

// cpu/code.cpp:68-132
int orc_rank_code(const void *in, int itype, void *out, int otype, int64_t b, int64_t t, int64_t x, int sort)
{
    return guard([&] {
        dispatch(itype, [&](auto i) {
            dispatch(otype, [&](auto o) {
                using I = decltype(i);
                using O = decltype(o);
                rank_code<I, O>((const I *)in, (O *)out, b, t, x, sort != 0);
            });
        });
    });
}

// cpu/fire.cpp:41-57 (in place, `x <= threshold -> value`)
int orc_threshold(void *data, int type, int64_t n, double thr, double value)
{
    return guard([&] {
        dispatch(type, [&](auto z) {
            using T = decltype(z);
            T *d = (T *)data;
            T th = scal<T>(thr), v = scal<T>(value);
            for (int64_t i = 0; i < n; ++i)
                if (d[i] <= th) d[i] = v;
        });
    });
}

// cpu/fire.cpp:59-65 (steps 0..T-2 of every sample set to value)
int orc_rank_infinite(void *data, int type, int64_t b, int64_t t, int64_t x, double value)
{
    return guard([&] {
        dispatch(type, [&](auto z) {
            using T = decltype(z);
            T v = scal<T>(value);
            for (int64_t i = 0; i < b; ++i) std::fill((T *)data + i * t * x, (T *)data + (i * t + t - 1) * x, v);
        });
    });
}

// cpu/fire.cpp:67-82 (`out = in > threshold`)
int orc_rank_fire(const void *in, int itype, void *out, int otype, int64_t n, double thr)
{
    return guard([&] {
        dispatch(itype, [&](auto i) {
            dispatch(otype, [&](auto o) {
                using I = decltype(i);
                using O = decltype(o);
                I th = scal<I>(thr);
                for (int64_t k = 0; k < n; ++k) ((O *)out)[k] = O(((const I *)in)[k] > th);
            });
        });
    });
}

// cpu/time.cpp:40-58 (first t with in > threshold, T if never)
int orc_rank_gather(const void *in, int itype, void *out, int otype, int64_t b, int64_t t, int64_t x, double thr)
{
    return guard([&] {
        dispatch(itype, [&](auto i) {
            dispatch(otype, [&](auto o) {
                using I = decltype(i);
                using O = decltype(o);
                I th = scal<I>(thr);
                for (int64_t s = 0; s < b; ++s)
                    for (int64_t j = 0; j < x; ++j)
                    {
                        O v = O(t);
                        for (int64_t k = t - 1; k >= 0; --k)
                            if (((const I *)in)[(s * t + k) * x + j] > th) v = O(k);
                        ((O *)out)[s * x + j] = v;
                    }
            });
        });
    });
}

// cpu/time.cpp:60-78 (`out[t] = U32(t) >= in`)
int orc_rank_scatter(const void *in, int itype, void *out, int otype, int64_t b, int64_t t, int64_t x)
{
    return guard([&] {
        dispatch(itype, [&](auto i) {
            dispatch(otype, [&](auto o) {
                using I = decltype(i);
                using O = decltype(o);
                for (int64_t s = 0; s < b; ++s)
                    for (int64_t k = 0; k < t; ++k)
                        for (int64_t j = 0; j < x; ++j)
                            ((O *)out)[(s * t + k) * x + j] = O(uint32_t(k) >= ((const I *)in)[s * x + j]);
            });
        });
    });
}

// cpu/pool.cpp:41-51 (pad order: top, left, bottom, right)
int orc_pad(const void *in, void *out, int type, int64_t n, int64_t h, int64_t w, const int64_t *p, double value)
{
    return guard([&] {
        dispatch(type, [&](auto z) {
            using T = decltype(z);
            int64_t oh = h + p[0] + p[2], ow = w + p[1] + p[3];
            T v = scal<T>(value);
            for (int64_t i = 0; i < n; ++i)
            {
                T *od = (T *)out + i * oh * ow;
                std::fill(od, od + oh * ow, v);
                for (int64_t j = 0; j < h; ++j)
                    std::copy((const T *)in + (i * h + j) * w, (const T *)in + (i * h + j + 1) * w,
                              od + (j + p[0]) * ow + p[1]);
            }
        });
    });
}

// cpu/pool.cpp:53-86 (zero pad, then max over the window; init Limits::min)
int orc_rank_pool(const void *in, void *out, int type, int64_t n, int64_t c, int64_t h, int64_t w, int64_t oh,
                  int64_t ow, const int64_t *k2, const int64_t *s2, const int64_t *p)
{
    return guard([&] {
        dispatch(type, [&](auto z) {
            using T = decltype(z);
            for (int64_t i = 0; i < n * c; ++i)
                for (int64_t y = 0; y < oh; ++y)
                    for (int64_t x = 0; x < ow; ++x)
                    {
                        T m = lowest<T>();
                        for (int64_t ky = 0; ky < k2[0]; ++ky)
                            for (int64_t kx = 0; kx < k2[1]; ++kx)
                            {
                                int64_t yy = y * s2[0] + ky - p[0], xx = x * s2[1] + kx - p[1];
                                T v = (yy >= 0 && yy < h && xx >= 0 && xx < w) ? ((const T *)in)[(i * h + yy) * w + xx]
                                                                              : T(0);
                                m = std::max(m, v);
                            }
                        ((T *)out)[(i * oh + y) * ow + x] = m;
                    }
        });
    });
}

// cpu/inhibit.cpp:41-121 over [B, T, C, X] in place.
int orc_rank_inhibit(void *data, int type, int64_t b, int64_t t, int64_t c, int64_t x, double thr)
{
    return guard([&] {
        dispatch(type, [&](auto z) {
            using T = decltype(z);
            T th = scal<T>(thr);
            for (int64_t s = 0; s < b; ++s)
            {
                T *d = (T *)data + s * t * c * x;
                for (int64_t j = 0; j < x; ++j)
                {
                    std::vector<uint16_t> ch(t);
                    uint16_t sum = 0;
                    for (int64_t k = 0; k < t; ++k)
                    {
                        T m = d[(k * c) * x + j];
                        uint16_t mc = 0;
                        for (int64_t q = 1; q < c; ++q)
                            if (d[(k * c + q) * x + j] > m) m = d[(k * c + q) * x + j], mc = uint16_t(q);
                        ch[k] = mc;
                        sum = uint16_t(sum + (m > th));
                    }
                    uint16_t win = ch[t - std::max<int64_t>(sum, 1)];
                    for (int64_t k = 0; k < t; ++k)
                        for (int64_t q = 0; q < c; ++q) d[(k * c + q) * x + j] *= T(uint16_t(q) == win);
                }
            }
        });
    });
}

// cpu/wta.cpp:123-152,159-162
int orc_rank_convwta(const void *in, int type, int64_t b, int64_t t, int64_t c, int64_t h, int64_t w,
                     const int64_t *r2, int64_t count, double thr, int64_t *winners, int64_t *counts)
{
    return guard([&] {
        std::vector<std::vector<W5>> ws(b);
        dispatch(type, [&](auto z) {
            using T = decltype(z);
#pragma omp parallel for
            for (int64_t s = 0; s < b; ++s)
            {
                std::vector<float> kf;
                std::vector<uint16_t> ki;
                wta_keys<T>((const T *)in + s * t * c * h * w, t, c * h * w, thr, kf, ki);
                if (std::is_floating_point<T>::value)
                    convwta_rounds<float>(kf, -FLT_MAX, c, h, w, r2[0], r2[1], count, ws[s]);
                else
                    convwta_rounds<uint16_t>(ki, 0, c, h, w, r2[0], r2[1], count, ws[s]);
            }
        });
        put_winners(ws, count, winners, counts);
    });
}

// cpu/wta.cpp:72-96,155-158
int orc_rank_fcwta(const void *in, int type, int64_t b, int64_t t, int64_t n, int64_t radius, int64_t count,
                   double thr, int64_t *winners, int64_t *counts)
{
    return guard([&] {
        std::vector<std::vector<W5>> ws(b);
        dispatch(type, [&](auto z) {
            using T = decltype(z);
            for (int64_t s = 0; s < b; ++s)
            {
                std::vector<float> kf;
                std::vector<uint16_t> ki;
                wta_keys<T>((const T *)in + s * t * n, t, n, thr, kf, ki);
                if (std::is_floating_point<T>::value)
                    fcwta_rounds<float>(kf, -FLT_MAX, radius, count, ws[s]);
                else
                    fcwta_rounds<uint16_t>(ki, 0, radius, count, ws[s]);
            }
        });
        put_winners(ws, count, winners, counts);
    });
}

// cpu/stdp.cpp:99-169.  Sequential over (sample, winner); the input window
// is read on the zero-padded grid, so taps outside the image never spike.
int orc_rank_convstdp(const void *in, int itype, int64_t b, int64_t t, int64_t cin, int64_t h, int64_t w,
                      void *kernel, int ktype, int64_t cout, int64_t kh, int64_t kw, const void *out, int64_t oh,
                      int64_t ow, const double *configs, int64_t nconf, const int64_t *winners,
                      const int64_t *counts, int64_t count, const int64_t *s2, const int64_t *p)
{
    return guard([&] {
        auto cfgs = get_cfgs(configs, nconf);
        dispatchR(itype, [&](auto iz) {
            dispatchR(ktype, [&](auto kz) {
                using T = decltype(iz);
                using K = decltype(kz);
                const T *I = (const T *)in;
                const T *O = (const T *)out;
                std::vector<uint16_t> isum(cin * kh * kw);
                for (int64_t s = 0; s < b; ++s)
                    for (int64_t j = 0; j < counts[s]; ++j)
                    {
                        const int64_t *e = winners + (s * count + j) * 5;
                        int64_t wc = e[0], wz = e[2], wy = e[3], wx = e[4];
                        if (wc < 0) continue;
                        if (wc >= nconf) throw std::runtime_error("STDP configuration index is out of range.");
                        for (int64_t c = 0; c < cin; ++c)
                            for (int64_t ky = 0; ky < kh; ++ky)
                                for (int64_t kx = 0; kx < kw; ++kx)
                                {
                                    int64_t yy = wy * s2[0] + ky - p[0], xx = wx * s2[1] + kx - p[1];
                                    uint16_t v = uint16_t(t);
                                    if (yy >= 0 && yy < h && xx >= 0 && xx < w)
                                        v = first_nonzero(I + ((s * t * cin + c) * h + yy) * w + xx, t, cin * h * w);
                                    isum[(c * kh + ky) * kw + kx] = v;
                                }
                        uint16_t osum = first_nonzero(O + ((s * t * cout + wz) * oh + wy) * ow + wx, t, cout * oh * ow);
                        K *kd = (K *)kernel + wz * cin * kh * kw;
                        for (int64_t i = 0; i < cin * kh * kw; ++i) stdp_weight(kd[i], isum[i] <= osum, cfgs[wc]);
                    }
            });
        });
    });
}

// cpu/stdp.cpp:42-97
int orc_rank_fcstdp(const void *in, int itype, int64_t b, int64_t t, int64_t ni, void *kernel, int ktype, int64_t no,
                    const void *out, const double *configs, int64_t nconf, const int64_t *winners,
                    const int64_t *counts, int64_t count)
{
    return guard([&] {
        auto cfgs = get_cfgs(configs, nconf);
        dispatchR(itype, [&](auto iz) {
            dispatchR(ktype, [&](auto kz) {
                using T = decltype(iz);
                using K = decltype(kz);
                std::vector<uint16_t> isum(ni);
                for (int64_t s = 0; s < b; ++s)
                {
                    for (int64_t j = 0; j < ni; ++j) isum[j] = first_nonzero((const T *)in + s * t * ni + j, t, ni);
                    for (int64_t j = 0; j < counts[s]; ++j)
                    {
                        const int64_t *e = winners + (s * count + j) * 5;
                        if (e[0] < 0) continue;
                        if (e[0] >= nconf) throw std::runtime_error("STDP configuration index is out of range.");
                        uint16_t osum = first_nonzero((const T *)out + s * t * no + e[4], t, no);
                        K *kd = (K *)kernel + e[4] * ni;
                        for (int64_t i = 0; i < ni; ++i) stdp_weight(kd[i], isum[i] <= osum, cfgs[e[0]]);
                    }
                }
            });
        });
    });
}

// FP64 oracle for the spike x weight contraction: cross-correlation with
// zero pad (top, left, bottom, right) and stride (shape.cpp:35-50,
// cpu/conv.cpp:58-75); exact FP64 sum, rounded once to the output type.
int orc_conv(const void *in, int itype, const void *kernel, int ktype, void *out, int otype, int64_t n, int64_t cin,
             int64_t h, int64_t w, int64_t cout, int64_t kh, int64_t kw, int64_t oh, int64_t ow, const int64_t *s2,
             const int64_t *p)
{
    return guard([&] {
        dispatchR(itype, [&](auto iz) {
            dispatchR(ktype, [&](auto kz) {
                dispatchR(otype, [&](auto oz) {
                    using I = decltype(iz);
                    using K = decltype(kz);
                    using O = decltype(oz);
                    const I *A = (const I *)in;
                    const K *B = (const K *)kernel;
#pragma omp parallel for collapse(2)
                    for (int64_t i = 0; i < n; ++i)
                        for (int64_t o = 0; o < cout; ++o)
                            for (int64_t y = 0; y < oh; ++y)
                                for (int64_t x = 0; x < ow; ++x)
                                {
                                    double acc = 0;
                                    for (int64_t c = 0; c < cin; ++c)
                                        for (int64_t ky = 0; ky < kh; ++ky)
                                        {
                                            int64_t yy = y * s2[0] + ky - p[0];
                                            if (yy < 0 || yy >= h) continue;
                                            for (int64_t kx = 0; kx < kw; ++kx)
                                            {
                                                int64_t xx = x * s2[1] + kx - p[1];
                                                if (xx < 0 || xx >= w) continue;
                                                acc += double(A[((i * cin + c) * h + yy) * w + xx]) *
                                                       double(B[((o * cin + c) * kh + ky) * kw + kx]);
                                            }
                                        }
                                    ((O *)out)[((i * cout + o) * oh + y) * ow + x] = O(acc);
                                }
                });
            });
        });
    });
}

// FC (cpu/fc.cpp:140-171): out[b,t,o] = sum_i in[b,t,i] * W[o,i]; sign
// variant uses sign(W).  Exact FP64 sum rounded once.
int orc_fc(const void *in, int itype, const void *kernel, int ktype, void *out, int otype, int64_t b, int64_t t,
           int64_t ni, int64_t no, int sign)
{
    return guard([&] {
        dispatchR(itype, [&](auto iz) {
            dispatchR(ktype, [&](auto kz) {
                dispatchR(otype, [&](auto oz) {
                    using I = decltype(iz);
                    using K = decltype(kz);
                    using O = decltype(oz);
                    for (int64_t r = 0; r < b * t; ++r)
                        for (int64_t o = 0; o < no; ++o)
                        {
                            double acc = 0;
                            for (int64_t i = 0; i < ni; ++i)
                            {
                                double wv = double(((const K *)kernel)[o * ni + i]);
                                if (sign) wv = wv > 0 ? 1.0 : (wv < 0 ? -1.0 : 0.0);
                                acc += double(((const I *)in)[r * ni + i]) * wv;
                            }
                            ((O *)out)[r * no + o] = O(acc);
                        }
                });
            });
        });
    });
}

// Filter banks (cpu/dog.cpp:40-94): each plane is convolved with every
// kernel (FP64 sum, rounded to the data type), then
//   DoG  : out = max(g1 - g2, 0)                  kernel [2, F, KH, KW]
//   Gabor: out = raw response                     kernel [F, KH, KW]
//   LoG  : on = max(d, 0), off = max(-d, 0) -> 2F kernel [2, F, KH, KW]
int orc_filter(int which, const void *in, const void *kernel, void *out, int type, int64_t n, int64_t h, int64_t w,
               int64_t f, int64_t kh, int64_t kw, int64_t oh, int64_t ow, const int64_t *p)
{
    return guard([&] {
        dispatch(type, [&](auto z) {
            using T = decltype(z);
            const T *A = (const T *)in;
            const T *K = (const T *)kernel;
            int64_t nk = (which == 1) ? f : 2 * f;
            std::vector<T> mid(nk * oh * ow);
            for (int64_t i = 0; i < n; ++i)
            {
                for (int64_t q = 0; q < nk; ++q)
                    for (int64_t y = 0; y < oh; ++y)
                        for (int64_t x = 0; x < ow; ++x)
                        {
                            double acc = 0;
                            for (int64_t ky = 0; ky < kh; ++ky)
                            {
                                int64_t yy = y + ky - p[0];
                                if (yy < 0 || yy >= h) continue;
                                for (int64_t kx = 0; kx < kw; ++kx)
                                {
                                    int64_t xx = x + kx - p[1];
                                    if (xx < 0 || xx >= w) continue;
                                    acc += double(A[(i * h + yy) * w + xx]) * double(K[(q * kh + ky) * kw + kx]);
                                }
                            }
                            mid[(q * oh + y) * ow + x] = T(acc);
                        }
                T *od = (T *)out + i * (which == 2 ? 2 * f : f) * oh * ow;
                int64_t plane = f * oh * ow;
                if (which == 1)
                    std::copy(mid.begin(), mid.end(), od);
                else if (which == 0)
                    for (int64_t k = 0; k < plane; ++k) od[k] = std::max<T>(mid[k] - mid[plane + k], T(0));
                else
                    for (int64_t k = 0; k < plane; ++k)
                    {
                        T d = mid[k] - mid[plane + k];
                        od[k] = std::max<T>(d, T(0));
                        od[plane + k] = std::max<T>(-d, T(0));
                    }
            }
        });
    });
}

// cpu/init.cpp:38-62 (normalised Gaussian)
int orc_gaussian_kernel(double *kernel, int64_t size, double std)
{
    return guard([&] {
        int64_t s = size / 2;
        double sum = 0;
        for (int64_t i = -s; i <= s; ++i)
            for (int64_t j = -s; j <= s; ++j)
            {
                double dist = std::sqrt(double(i * i + j * j));
                double v = std::exp(-.5 * std::pow(dist / std, 2));
                kernel[(i + s) * size + (j + s)] = v;
            }
        for (int64_t i = 0; i < size * size; ++i) sum += kernel[i];
        for (int64_t i = 0; i < size * size; ++i) kernel[i] /= sum;
    });
}

// cpu/init.cpp:64-77 (normalised Gabor, theta in radians here)
int orc_gabor_kernel(double *kernel, int64_t size, double sigma, double theta, double gamma, double lambda, double psi)
{
    return guard([&] {
        const double pi = 3.14159265358979323846;
        int64_t s = size / 2;
        double sum = 0;
        for (int64_t i = -s; i <= s; ++i)
            for (int64_t j = -s; j <= s; ++j)
            {
                double x = i * std::cos(theta) + j * std::sin(theta);
                double y = -i * std::sin(theta) + j * std::cos(theta);
                double a = std::exp(-(x * x + gamma * gamma * y * y) / (2 * sigma * sigma));
                double c = std::cos(2 * pi * x / lambda + psi);
                kernel[(i + s) * size + (j + s)] = a * c;
            }
        for (int64_t i = 0; i < size * size; ++i) sum += kernel[i];
        for (int64_t i = 0; i < size * size; ++i) kernel[i] /= sum;
    });
}

// cpu/init.cpp:79-90 (LoG kernel, not normalised)
int orc_log_kernel(double *kernel, int64_t size, double std)
{
    return guard([&] {
        const double pi = 3.14159265358979323846;
        int64_t s = size / 2;
        double div = -pi * std::pow(std, 4);
        for (int64_t i = -s; i <= s; ++i)
            for (int64_t j = -s; j <= s; ++j)
            {
                double a = (i * i + j * j) / (-2 * std * std);
                kernel[(i + s) * size + (j + s)] = (1 + a) * std::exp(a) / div;
            }
    });
}

// cpu/backprop.cpp:40-62 (temporal-backprop target rule)
int orc_backward(const void *in, void *out, int type, const int64_t *target, int64_t b, int64_t n, int64_t time,
                 double gamma)
{
    return guard([&] {
        dispatch(type, [&](auto z) {
            using T = decltype(z);
            T g = scal<T>(gamma);
            for (int64_t s = 0; s < b; ++s)
            {
                const T *id = (const T *)in + s * n;
                T *od = (T *)out + s * n;
                std::copy(id, id + n, od);
                T mn = od[0];
                for (int64_t i = 0; i < n; ++i) mn = std::min(mn, od[i]);
                T upper = mn + g, value = std::min(T(time), upper);
                if (mn != time)
                    for (int64_t i = 0; i < n; ++i) od[i] = (od[i] < upper) ? value : od[i];
                od[target[s]] = std::max(T(0), mn);
                for (int64_t i = 0; i < n; ++i) od[i] = (od[i] - id[i]) / T(time);
            }
        });
    });
}

// cpu/backprop.cpp:68-99 (label = earliest-spiking neuron, else the
// last-step argmax)
int orc_labelize(const void *in, int type, int64_t *out, int64_t b, int64_t t, int64_t n, double thr)
{
    return guard([&] {
        dispatch(type, [&](auto z) {
            using T = decltype(z);
            T th = scal<T>(thr);
            std::vector<uint16_t> mid(n);
            for (int64_t s = 0; s < b; ++s)
            {
                const T *id = (const T *)in + s * t * n;
                for (int64_t j = 0; j < n; ++j)
                {
                    uint16_t v = uint16_t(t);
                    for (int64_t k = t - 1; k >= 0; --k)
                        if (id[k * n + j] > th) v = uint16_t(k);
                    mid[j] = v;
                }
                int64_t m = minidx(mid.data(), n);
                if (mid[m] == t) m = maxidx(id + (t - 1) * n, n);
                out[s] = m;
            }
        });
    });
}

// cpu/backprop.cpp:105-160 (sign-weight FC rule; updates the kernel and
// the scale factor inside backward).  Multiply-adds are fused as GCC does
// under -ffp-contract=fast.
int orc_fcbackward(float *kernel, int64_t no, int64_t ni, const void *in, const void *out, const void *grad,
                   void *next, int type, int64_t b, float *bp)
{
    return guard([&] {
        dispatch(type, [&](auto z) {
            using T = decltype(z);
            std::vector<float> sign(no * ni), select(no * ni);
            for (int64_t i = 0; i < no * ni; ++i) sign[i] = kernel[i] > 0 ? 1.f : (kernel[i] < 0 ? -1.f : 0.f);
            float lrate = bp[1], lrf = bp[2], lambda = bp[3];
            for (int64_t s = 0; s < b; ++s)
            {
                const T *id = (const T *)in + s * ni;
                for (int64_t j = 0; j < no; ++j)
                {
                    T o = ((const T *)out)[s * no + j], g = ((const T *)grad)[s * no + j];
                    for (int64_t i = 0; i < ni; ++i) select[j * ni + i] = float(T(id[i] < o) * g);
                }
                for (int64_t i = 0; i < no * ni; ++i) kernel[i] = std::fma(-lrate, select[i], kernel[i]);
                float mult = lrate * lambda;
                for (int64_t i = 0; i < no * ni; ++i) kernel[i] = std::fma(-mult, kernel[i], kernel[i]);
                float sum = 0;
                for (int64_t i = 0; i < no * ni; ++i) sum = std::fma(lrf * select[i], sign[i], sum);
                bp[0] -= sum / float(no * ni);
                T *nd = (T *)next + s * ni;
                std::fill(nd, nd + ni, T(0));
                for (int64_t j = 0; j < no; ++j)
                    for (int64_t i = 0; i < ni; ++i) nd[i] = T(std::fma(kernel[j * ni + i], select[j * ni + i], float(nd[i])));
            }
        });
    });
}

// ------------------------------- sparse ----------------------------------

// sparse/code.cpp:39-100
int orc_sparse_code(const void *in, int itype, int64_t u, int64_t c, int64_t h, int64_t w, int64_t t, int sort,
                    int64_t **offsets, uint8_t **zyx)
{
    return guard([&] {
        Lists l(u * t);
        dispatch(itype, [&](auto z) {
            using T = decltype(z);
            std::vector<uint16_t> tm(c * h * w);
            std::vector<uint32_t> index;
            for (int64_t i = 0; i < u; ++i)
            {
                code_times((const T *)in + i * c * h * w, c * h * w, t, sort != 0, tm.data(), index);
                times_to_events(tm.data(), c, h, w, t, l, i);
            }
        });
        put_lists(l, offsets, zyx);
    });
}

// sparse/opers.cpp:59-86 (SparseTensor(Tensor, threshold))
int orc_sparse_from_dense(const void *in, int itype, int64_t u, int64_t t, int64_t c, int64_t h, int64_t w,
                          double thr, int64_t **offsets, uint8_t **zyx)
{
    return guard([&] {
        Lists l(u * t);
        dispatch(itype, [&](auto z) {
            using T = decltype(z);
            T th = scal<T>(thr);
            int64_t x = c * h * w;
            std::vector<uint16_t> tm(x);
            for (int64_t i = 0; i < u; ++i)
            {
                const T *id = (const T *)in + i * t * x;
                for (int64_t j = 0; j < x; ++j)
                {
                    uint16_t v = uint16_t(t);
                    for (int64_t k = t - 1; k >= 0; --k)
                        if (id[k * x + j] > th) v = uint16_t(k);
                    tm[j] = v;
                }
                times_to_events(tm.data(), c, h, w, t, l, i);
            }
        });
        put_lists(l, offsets, zyx);
    });
}

// sparse/opers.cpp:88-104 (cumulative dense spikes)
int orc_sparse_to_dense(const int64_t *offsets, const uint8_t *zyx, int64_t u, int64_t t, int64_t c, int64_t h,
                        int64_t w, void *out, int otype)
{
    return guard([&] {
        Lists l = get_lists(offsets, zyx, u * t);
        dispatch(otype, [&](auto z) {
            using T = decltype(z);
            int64_t x = c * h * w;
            for (int64_t i = 0; i < u; ++i)
                for (int64_t j = 0; j < t; ++j)
                {
                    T *od = (T *)out + (i * t + j) * x;
                    if (j == 0)
                        std::fill(od, od + x, T(0));
                    else
                        std::copy(od - x, od, od);
                    for (const Ev &e : l[i * t + j]) od[(e.z * h + e.y) * w + e.x] = T(1);
                }
        });
    });
}

// sparse/opers.cpp:106-118 (first-spike time map, T when silent)
int orc_sparse_gather(const int64_t *offsets, const uint8_t *zyx, int64_t u, int64_t t, int64_t c, int64_t h,
                      int64_t w, void *out, int otype)
{
    return guard([&] {
        Lists l = get_lists(offsets, zyx, u * t);
        dispatch(otype, [&](auto z) {
            using T = decltype(z);
            int64_t x = c * h * w;
            for (int64_t i = 0; i < u; ++i)
            {
                T *od = (T *)out + i * x;
                std::fill(od, od + x, T(t));
                for (int64_t j = t - 1; j >= 0; --j)
                    for (const Ev &e : l[i * t + j]) od[(e.z * h + e.y) * w + e.x] = T(j);
            }
        });
    });
}

// sparse/conv.cpp:42-130: incremental conv + fire.  Per (sample, output
// channel) an F32 potential plane accumulates, in event order, the kernel
// taps of every newly arrived input event; at each step that had input
// events, every neuron above threshold emits one event and is parked at
// -FLT_MAX.  Output events per step are channel-major.
int orc_sparse_conv(const int64_t *offsets, const uint8_t *zyx, int64_t u, int64_t t, int64_t c, int64_t h, int64_t w,
                    const float *kernel, int64_t cout, int64_t kh, int64_t kw, double thr, const int64_t *s2,
                    const int64_t *p, int64_t oh, int64_t ow, int64_t **ooff, uint8_t **ozyx)
{
    return guard([&] {
        if (s2[0] != 1 || s2[1] != 1) throw std::runtime_error("Stride must be 1 in sparse conv.");
        Lists l = get_lists(offsets, zyx, u * t), o(u * t);
        float th = float(thr);
        std::vector<float> pot(oh * ow);
        for (int64_t i = 0; i < u; ++i)
            for (int64_t q = 0; q < cout; ++q)
            {
                std::fill(pot.begin(), pot.end(), 0.f);
                for (int64_t j = 0; j < t; ++j)
                {
                    const auto &ev = l[i * t + j];
                    for (const Ev &e : ev)
                    {
                        const float *kd = kernel + (q * c + e.z) * kh * kw;
                        int64_t yy = e.y + p[0], xx = e.x + p[1];
                        for (int64_t y = 0; y < oh; ++y)
                        {
                            int64_t ky = yy - y;
                            if (ky < 0 || ky >= kh) continue;
                            for (int64_t x = 0; x < ow; ++x)
                            {
                                int64_t kx = xx - x;
                                if (kx < 0 || kx >= kw) continue;
                                pot[y * ow + x] += kd[ky * kw + kx];
                            }
                        }
                    }
                    if (!ev.empty())
                        for (int64_t y = 0; y < oh; ++y)
                            for (int64_t x = 0; x < ow; ++x)
                                if (pot[y * ow + x] > th)
                                {
                                    o[i * t + j].push_back({uint8_t(q), uint8_t(y), uint8_t(x)});
                                    pot[y * ow + x] = -FLT_MAX;
                                }
                }
            }
        // Per step, events were produced channel by channel already.
        put_lists(o, ooff, ozyx);
    });
}

// sparse/pad.cpp:37-55 (shift by (top, left); u8 coordinates wrap)
int orc_sparse_pad(const int64_t *offsets, const uint8_t *zyx, int64_t u, int64_t t, int64_t c, int64_t h, int64_t w,
                   const int64_t *p, int64_t **ooff, uint8_t **ozyx)
{
    return guard([&] {
        Lists l = get_lists(offsets, zyx, u * t);
        for (auto &v : l)
            for (auto &e : v) e.y = uint8_t(e.y + p[0]), e.x = uint8_t(e.x + p[1]);
        put_lists(l, ooff, ozyx);
    });
}

// sparse/pool.cpp:37-64 (first event per pooled cell; stride == kernel)
int orc_sparse_pool(const int64_t *offsets, const uint8_t *zyx, int64_t u, int64_t t, int64_t c, int64_t h, int64_t w,
                    const int64_t *k2, const int64_t *s2, const int64_t *p, int64_t oh, int64_t ow, int64_t **ooff,
                    uint8_t **ozyx)
{
    return guard([&] {
        if (s2[0] != k2[0] || s2[1] != k2[1]) throw std::runtime_error("Stride must be equal to kernel in sparse pool.");
        Lists l = get_lists(offsets, zyx, u * t), o(u * t);
        std::vector<uint8_t> seen(c * oh * ow);
        for (int64_t i = 0; i < u; ++i)
        {
            std::fill(seen.begin(), seen.end(), 0);
            for (int64_t j = 0; j < t; ++j)
                for (Ev e : l[i * t + j])
                {
                    uint8_t y = uint8_t((p[0] + e.y) / k2[0]), x = uint8_t((p[1] + e.x) / k2[1]);
                    if (y >= oh || x >= ow) continue;
                    uint8_t &s = seen[(e.z * oh + y) * ow + x];
                    if (s) continue;
                    s = 1;
                    o[i * t + j].push_back({e.z, y, x});
                }
        }
        put_lists(o, ooff, ozyx);
    });
}

// sparse/inhibit.cpp:37-65 (per pixel keep the channel of its first event)
int orc_sparse_inhibit(const int64_t *offsets, const uint8_t *zyx, int64_t u, int64_t t, int64_t c, int64_t h,
                       int64_t w, int64_t **ooff, uint8_t **ozyx)
{
    return guard([&] {
        Lists l = get_lists(offsets, zyx, u * t), o(u * t);
        std::vector<uint16_t> ch(h * w);
        for (int64_t i = 0; i < u; ++i)
        {
            std::fill(ch.begin(), ch.end(), uint16_t(0xFFFF));
            for (int64_t j = 0; j < t; ++j)
                for (const Ev &e : l[i * t + j])
                    if (ch[e.y * w + e.x] == 0xFFFF) ch[e.y * w + e.x] = e.z;
            for (int64_t j = 0; j < t; ++j)
                for (const Ev &e : l[i * t + j])
                    if (ch[e.y * w + e.x] == e.z) o[i * t + j].push_back(e);
        }
        put_lists(o, ooff, ozyx);
    });
}

// sparse/wta.cpp:44-95 (accept events in (t, list) order that hit neither
// a taken channel nor an accepted box)
int orc_sparse_convwta(const int64_t *offsets, const uint8_t *zyx, int64_t u, int64_t t, int64_t c, int64_t h,
                       int64_t w, const int64_t *r2, int64_t count, int64_t *winners, int64_t *counts)
{
    return guard([&] {
        Lists l = get_lists(offsets, zyx, u * t);
        std::vector<std::vector<W5>> ws(u);
        struct Box
        {
            int64_t z, ys, ye, xs, xe;
        };
        for (int64_t i = 0; i < u; ++i)
        {
            std::vector<Box> boxes;
            for (int64_t j = 0; j < t && int64_t(ws[i].size()) < count; ++j)
                for (const Ev &e : l[i * t + j])
                {
                    bool ok = true;
                    for (const Box &b : boxes)
                    {
                        if (e.z == b.z) { ok = false; break; }
                        if (e.y < b.ys || b.ye < e.y) continue;
                        if (e.x < b.xs || b.xe < e.x) continue;
                        ok = false;
                        break;
                    }
                    if (!ok) continue;
                    ws[i].push_back({0, j, e.z, e.y, e.x});
                    if (int64_t(ws[i].size()) >= count) break;
                    boxes.push_back({e.z, std::max<int64_t>(0, e.y - r2[0]), std::min<int64_t>(h - 1, e.y + r2[0]),
                                     std::max<int64_t>(0, e.x - r2[1]), std::min<int64_t>(w - 1, e.x + r2[1])});
                }
        }
        put_winners(ws, count, winners, counts);
    });
}

// sparse/stdp.cpp:41-133.  For every winner (global order) the window of
// kh x kw inputs starting at (winner.y, winner.x) on the padded grid is
// marked "pre-before-post" when the LAST event written at a position has
// time <= winner.t; updates use F32 storage with F64 bound arithmetic.
int orc_sparse_stdp(const int64_t *offsets, const uint8_t *zyx, int64_t u, int64_t t, int64_t c, int64_t h, int64_t w,
                    float *kernel, int64_t cout, int64_t kh, int64_t kw, const double *configs, int64_t nconf,
                    const int64_t *winners, const int64_t *counts, int64_t count, const int64_t *p)
{
    return guard([&] {
        Lists l = get_lists(offsets, zyx, u * t);
        auto cfgs = get_cfgs(configs, nconf);
        int64_t wsize = c * kh * kw;
        std::vector<std::vector<uint16_t>> direct;
        std::vector<const int64_t *> order;
        for (int64_t i = 0; i < u; ++i)
        {
            size_t first = direct.size();
            for (int64_t j = 0; j < counts[i]; ++j)
            {
                direct.emplace_back(wsize, uint16_t(t));
                order.push_back(winners + (i * count + j) * 5);
            }
            for (int64_t j = 0; j < t; ++j)
                for (Ev e : l[i * t + j])
                {
                    int64_t ey = e.y + p[0], ex = e.x + p[1];
                    for (size_t k = first; k < direct.size(); ++k)
                    {
                        const int64_t *b = order[k];
                        if (b[3] <= ey && ey <= b[3] + kh - 1 && b[4] <= ex && ex <= b[4] + kw - 1)
                            direct[k][(e.z * kh + (ey - b[3])) * kw + (ex - b[4])] = uint16_t(j);
                    }
                }
            for (size_t k = first; k < direct.size(); ++k)
                for (auto &v : direct[k]) v = uint16_t(v <= order[k][1]);
        }
        for (size_t k = 0; k < direct.size(); ++k)
        {
            const int64_t *b = order[k];
            if (b[0] < 0) continue;
            if (b[0] >= nconf) throw std::runtime_error("STDP config index is out of range.");
            const Cfg &cf = cfgs[b[0]];
            float *kd = kernel + b[2] * wsize;
            for (int64_t i = 0; i < wsize; ++i)
            {
                float mult = float(cf.stab ? (double(kd[i]) - cf.lo) * (cf.hi - double(kd[i])) : 1.0);
                kd[i] = float(std::fma(direct[k][i] ? cf.pos : cf.neg, double(mult), double(kd[i])));
                kd[i] = float(std::max(cf.lo, std::min(double(kd[i]), cf.hi)));
            }
        }
    });
}


// ------------------------------------------------------------------------
// Rate coding.  Interval table (cpu/init.cpp:120-149): row i, lambda = i + 1,
// r = ceil(scale sqrt(lambda)) (5 for row 0, else 4), each j in
// [max(1, lambda - r), lambda + r] nearbyint(ztp(j, lambda) bins) times, the
// rest lambda; the reference then std::random_shuffle-s each row (order
// implementation-defined) -- here Fisher-Yates with std::mt19937(i + 1).
// ------------------------------------------------------------------------
int orc_poisson_table(int64_t time, int64_t bins, uint16_t *out)
{
    return guard([&] {
        auto ztp = [](uint16_t k, float a) {
            float p = 1 / (std::exp(a) - 1);
            for (int64_t i = 1; i <= k; ++i) p *= a / i;
            return p;
        };
        for (int64_t i = 0; i < time; ++i)
        {
            float scale = i < 1 ? 5 : 4;
            uint16_t lambda = uint16_t(i + 1), range = uint16_t(std::ceil(scale * std::sqrt(lambda)));
            uint16_t start = uint16_t(std::max(1, lambda - range)), end = uint16_t(lambda + range);
            uint16_t *row = out + i * bins;
            int64_t index = 0;
            for (uint16_t j = start; j <= end; ++j)
            {
                int64_t count = int64_t(std::nearbyint(ztp(j, lambda) * bins));
                if (index + count > bins) count = bins - index;
                std::fill(row + index, row + index + count, j);
                index += count;
                if (j == 65535) break;
            }
            std::fill(row + index, row + bins, lambda);
            std::mt19937 rng(static_cast<std::mt19937::result_type>(i + 1));
            for (int64_t k = bins - 1; k > 0; --k) std::swap(row[k], row[rng() % uint32_t(k + 1)]);
        }
    });
}

// cpu/code.cpp:177-217: per position the Poisson process of its time's row
// (rows past the table: never); one std::mt19937 per sample seeded seed + i.
int orc_rate_code_seeded(const void *in, int itype, void *out, int otype, int64_t b, int64_t t, int64_t x, int sort,
                         uint64_t seed)
{
    return guard([&] {
        const int64_t bins = 1024;
        std::vector<uint16_t> table(size_t(t * bins));
        orc_poisson_table(t, bins, table.data());
        dispatch(itype, [&](auto zi) {
            dispatch(otype, [&](auto zo) {
                using I = decltype(zi);
                using O = decltype(zo);
                std::vector<uint16_t> temp(x), times(x), values(x);
                std::vector<uint32_t> index;
                for (int64_t i = 0; i < b; ++i)
                {
                    std::mt19937 random(static_cast<std::mt19937::result_type>(seed + uint64_t(i)));
                    code_times((const I *)in + i * x, x, t, sort != 0, temp.data(), index);
                    auto draw = [&](int64_t j) -> uint32_t {
                        const uint32_t idx = random() & uint32_t(bins - 1);
                        return temp[j] < t ? table[size_t(temp[j]) * bins + idx] : uint32_t(0);
                    };
                    std::fill(values.begin(), values.end(), uint16_t(0));
                    for (int64_t j = 0; j < x; ++j) times[j] = temp[j] < t ? uint16_t(draw(j)) : uint16_t(65535);
                    for (int64_t s = 0; s < t; ++s)
                    {
                        O *od = (O *)out + (i * t + s) * x;
                        for (int64_t j = 0; j < x; ++j)
                        {
                            if (times[j] == s) values[j] += 1, times[j] = uint16_t(times[j] + draw(j));
                            od[j] = O(values[j]);
                        }
                    }
                }
            });
        });
    });
}

int orc_rate_code(const void *in, int itype, void *out, int otype, int64_t b, int64_t t, int64_t x, int sort)
{
    return orc_rate_code_seeded(in, itype, out, otype, b, t, x, sort, 1);
}

// cpu/fire.cpp:84-113: a spike when the input exceeds the value at the last
// spike by more than the threshold; outputs are the running counts.
int orc_rate_fire(const void *in, int itype, void *out, int otype, int64_t b, int64_t t, int64_t x, double thr)
{
    return guard([&] {
        dispatch(itype, [&](auto zi) {
            dispatch(otype, [&](auto zo) {
                using I = decltype(zi);
                using O = decltype(zo);
                I th = scal<I>(thr);
                for (int64_t i = 0; i < b; ++i)
                    for (int64_t j = 0; j < x; ++j)
                    {
                        I value = I(0);
                        O spikes = O(0);
                        for (int64_t s = 0; s < t; ++s)
                        {
                            I v = ((const I *)in)[(i * t + s) * x + j];
                            if (value + th < v) spikes = O(spikes + O(1)), value = v;
                            ((O *)out)[(i * t + s) * x + j] = spikes;
                        }
                    }
            });
        });
    });
}

// cpu/time.cpp:87-92: the last step.
int orc_rate_gather(const void *in, int itype, void *out, int otype, int64_t b, int64_t t, int64_t x)
{
    return guard([&] {
        dispatch(itype, [&](auto zi) {
            dispatch(otype, [&](auto zo) {
                using I = decltype(zi);
                using O = decltype(zo);
                for (int64_t i = 0; i < b; ++i)
                    for (int64_t j = 0; j < x; ++j) ((O *)out)[i * x + j] = O(((const I *)in)[(i * t + t - 1) * x + j]);
            });
        });
    });
}

// cpu/pool.cpp:88-137: the window position of highest rate (first in window
// row-major order, strict <), its value at every step.
int orc_rate_pool(const void *in, const void *rates, int type, int rtype, void *out, int64_t b, int64_t t, int64_t c,
                  int64_t h, int64_t w, int64_t oh, int64_t ow, const int64_t *kernel2, const int64_t *stride2)
{
    return guard([&] {
        dispatch(type, [&](auto zt) {
            dispatch(rtype, [&](auto zr) {
                using T = decltype(zt);
                using R = decltype(zr);
                for (int64_t i = 0; i < b; ++i)
                    for (int64_t k = 0; k < c; ++k)
                        for (int64_t oy = 0; oy < oh; ++oy)
                            for (int64_t ox = 0; ox < ow; ++ox)
                            {
                                const R *r = (const R *)rates + (i * c + k) * h * w;
                                R best = lowest<R>();
                                int64_t bi = 0;
                                for (int64_t a = 0; a < kernel2[0]; ++a)
                                    for (int64_t q = 0; q < kernel2[1]; ++q)
                                    {
                                        int64_t idx = (oy * stride2[0] + a) * w + ox * stride2[1] + q;
                                        if (best < r[idx]) best = r[idx], bi = idx;
                                    }
                                for (int64_t s = 0; s < t; ++s)
                                    ((T *)out)[(((i * t + s) * c + k) * oh + oy) * ow + ox] =
                                        ((const T *)in)[((i * t + s) * c + k) * h * w + bi];
                            }
            });
        });
    });
}
}  // extern "C"
