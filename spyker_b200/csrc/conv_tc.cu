// Tensor-core (tcgen05) convolution path.
#include "conv_tc.cuh"

namespace spk
{
size_t conv_tc_workspace(int64_t, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t, int) { return 0; }

void conv_tc(const void *, spk_dtype, const float *, float *, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t,
             int64_t, int64_t, int64_t, Pad4, int64_t, int64_t, int, void *, size_t, cudaStream_t)
{
    throw Error(SPK_ERR_UNSUPPORTED, "the tensor-core convolution path is not built yet");
}
}  // namespace spk
