// Tensor-core (tcgen05) path of spk_conv: weights split into BF16 terms,
// FP32 accumulation in tensor memory.
#pragma once

#include "common.cuh"

namespace spk
{
size_t conv_tc_workspace(int64_t n, int64_t cin, int64_t h, int64_t w, int64_t cout, int64_t kh, int64_t kw,
                         int precision);
void conv_tc(const void *in, spk_dtype itype, const float *kernel, float *out, int64_t n, int64_t cin, int64_t h,
             int64_t w, int64_t cout, int64_t kh, int64_t kw, int64_t sy, int64_t sx, Pad4 p, int64_t oh, int64_t ow,
             int precision, void *ws, size_t ws_bytes, cudaStream_t s);
}  // namespace spk
