// Shared helpers for the sm_100a kernels and the C-ABI layer.
#pragma once

#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>
#include <stdexcept>
#include <string>

#include "../../include/spyker_b200.h"

namespace spk
{
// Host-side error carrying an spk_status; converted to a status code at the
// C boundary (no exception ever crosses it).
struct Error : std::runtime_error
{
    spk_status code;
    Error(spk_status c, const std::string &m) : std::runtime_error(m), code(c) {}
};

void set_error(const std::string &msg);

#define SPK_REQUIRE(cond, msg)                                                               \
    do                                                                                       \
    {                                                                                        \
        if (!(cond)) throw ::spk::Error(SPK_ERR_ARGUMENT, std::string(__func__) + ": " + msg); \
    } while (0)

#define SPK_CUDA(expr)                                                                                   \
    do                                                                                                   \
    {                                                                                                    \
        cudaError_t _e = (expr);                                                                         \
        if (_e != cudaSuccess)                                                                           \
            throw ::spk::Error(SPK_ERR_CUDA, std::string(#expr) + " failed: " + cudaGetErrorString(_e)); \
    } while (0)

// Every kernel launch site ends with SPK_LAUNCHED(): it checks the launch and
// counts it (spk_launch_count).
void count_launch();
#define SPK_LAUNCHED()                  \
    do                                  \
    {                                   \
        SPK_CUDA(cudaGetLastError());   \
        ::spk::count_launch();          \
    } while (0)

// Run `body` and translate exceptions into a status code.
template <typename F>
spk_status guarded(F &&body)
{
    try
    {
        body();
        return SPK_OK;
    }
    catch (const Error &e)
    {
        set_error(e.what());
        return e.code;
    }
    catch (const std::exception &e)
    {
        set_error(e.what());
        return SPK_ERR_ARGUMENT;
    }
}

inline cudaStream_t stream_of(spk_stream s) { return reinterpret_cast<cudaStream_t>(s); }

int sm_count();

// Grid for a grid-stride loop over `work` items with `threads` per block.
inline unsigned grid_for(int64_t work, int threads, int per_sm = 8)
{
    int64_t blocks = (work + threads - 1) / threads;
    int64_t cap = int64_t(sm_count()) * per_sm;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    return unsigned(blocks);
}

// Element types supported on the hot path (codes of the reference's Type enum).
template <typename F>
void dispatch(spk_dtype t, F &&f)
{
    switch (t)
    {
    case SPK_U8: f(uint8_t()); break;
    case SPK_I32: f(int32_t()); break;
    case SPK_I64: f(int64_t()); break;
    case SPK_F32: f(float()); break;
    case SPK_F64: f(double()); break;
    default: throw Error(SPK_ERR_UNSUPPORTED, "data type code " + std::to_string(int(t)) + " is not supported");
    }
}

template <typename F>
void dispatch_real(spk_dtype t, F &&f)
{
    switch (t)
    {
    case SPK_F32: f(float()); break;
    case SPK_F64: f(double()); break;
    default: throw Error(SPK_ERR_UNSUPPORTED, "only F32/F64 are supported here");
    }
}

template <typename T>
struct Lowest;
template <>
struct Lowest<uint8_t>
{
    static __host__ __device__ uint8_t v() { return 0; }
};
template <>
struct Lowest<int32_t>
{
    static __host__ __device__ int32_t v() { return INT32_MIN; }
};
template <>
struct Lowest<int64_t>
{
    static __host__ __device__ int64_t v() { return INT64_MIN; }
};
template <>
struct Lowest<float>
{
    static __host__ __device__ float v() { return -FLT_MAX; }
};
template <>
struct Lowest<double>
{
    static __host__ __device__ double v() { return -DBL_MAX; }
};

// Scalar parameters arrive as F64 and are converted to the data type with a
// C cast, as the reference's Scalar::to does.
template <typename T>
inline T scalar_to(double v)
{
    return T(v);
}

// float -> U16 with the x86-64 lowering the reference's CPU build uses
// (truncate to int32, keep the low 16 bits; NaN / out of range -> 0).
__device__ __forceinline__ uint16_t f2u16(float v)
{
    if (!(v > -2147483648.0f && v < 2147483648.0f)) return 0;
    return uint16_t(uint32_t(__float2int_rz(v)));
}

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Block-wide copy of the global byte range [src, src + n) into shared memory
// (dst 16-byte aligned).  Byte i lands at dst[(src & 15) + i], so the range's
// 16-byte-aligned interior moves with 16-byte loads and stores (four in
// flight per thread) and only the ragged ends go byte by byte.  Returns the
// offset (src & 15).  No barrier inside.
__device__ __forceinline__ int stage_bytes(unsigned char *dst, const unsigned char *src, int64_t n)
{
    const uintptr_t a = reinterpret_cast<uintptr_t>(src);
    const int shift = int(a & 15);
    unsigned char *d = dst + shift;
    const uintptr_t lo = (a + 15) & ~uintptr_t(15), hi = (a + uintptr_t(n)) & ~uintptr_t(15);
    if (lo >= hi)
    {
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) d[i] = src[i];
        return shift;
    }
    const int64_t head = int64_t(lo - a), tail = int64_t(hi - a);
    for (int64_t i = threadIdx.x; i < head; i += blockDim.x) d[i] = src[i];
    for (int64_t i = tail + threadIdx.x; i < n; i += blockDim.x) d[i] = src[i];
    const uint4 *s4 = reinterpret_cast<const uint4 *>(lo);
    uint4 *d4 = reinterpret_cast<uint4 *>(d + head);
    const int64_t n4 = int64_t(hi - lo) >> 4, step = blockDim.x;
    int64_t i = threadIdx.x;
    for (; i + 3 * step < n4; i += 4 * step)
    {
        const uint4 v0 = __ldg(s4 + i), v1 = __ldg(s4 + i + step), v2 = __ldg(s4 + i + 2 * step),
                    v3 = __ldg(s4 + i + 3 * step);
        d4[i] = v0, d4[i + step] = v1, d4[i + 2 * step] = v2, d4[i + 3 * step] = v3;
    }
    for (; i < n4; i += step) d4[i] = __ldg(s4 + i);
    return shift;
}

struct Pad4
{
    int64_t top, left, bottom, right;
};

inline Pad4 pad_of(const int64_t *p)
{
    SPK_REQUIRE(p != nullptr, "pad pointer is null");
    SPK_REQUIRE(p[0] >= 0 && p[1] >= 0 && p[2] >= 0 && p[3] >= 0, "pad items are incorrect");
    return {p[0], p[1], p[2], p[3]};
}

size_t dtype_size(spk_dtype t);
}  // namespace spk
