// Conv STDP for callers that cannot allocate device memory.
//
// spk_rank_convstdp needs a scratch buffer for the first-spike times of every
// winner's receptive field, and expects the caller to provide it.  Some
// callers cannot call cudaMalloc at all: plug-in hosts whose allocator owns
// all device memory (a second allocator would fragment it or exceed its
// budget), or C callers without a device allocator of their own.  For
// them this file gives the same update with its scratch in a fixed static
// device array, so the call allocates nothing.
//
// The array is kNoAllocScratchBytes (32 MiB); every GPU that loads this part
// of the library holds it until the process exits.  A call whose scratch need
// (2 * B * count * Cin * KH * KW bytes for the receptive fields plus
// 2 * B * count for the winners, each rounded up to 256 bytes) exceeds it is
// rejected with SPK_ERR_ARGUMENT; split the batch into smaller calls.
#include "common.cuh"

namespace spk
{
void convstdp_into(const void *in, spk_dtype itype, int64_t b, int64_t t, int64_t cin, int64_t h, int64_t w,
                   float *kernel, int64_t cout, int64_t kh, int64_t kw, const void *out, int64_t oh, int64_t ow,
                   const double *configs, int64_t nconf, const int32_t *winners, const int32_t *counts, int64_t count,
                   int64_t sy, int64_t sx, const int64_t *pad4, void *scratch, cudaStream_t s);
size_t convstdp_prepost_bytes(int64_t b, int64_t count, int64_t cin, int64_t kh, int64_t kw);

namespace
{
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;

// Shared by every call on a device; it keeps the previous call's contents.
// Nothing in it needs to start at zero: the (pre, post) entries of every valid
// winner are written before they are read, and invalid slots are never read.
static __device__ __align__(256) unsigned char g_stdp_scratch[kNoAllocScratchBytes];

// Device address of the static array on the current device.  In host code
// `g_stdp_scratch` names a host-side stand-in, not device memory, so the
// address is looked up with that device current.  The lookup runs on every
// call (it is host-only and issues no stream work), so no address outlives a
// cudaDeviceReset.
void *scratch_address()
{
    void *p = nullptr;
    SPK_CUDA(cudaGetSymbolAddress(&p, g_stdp_scratch));
    SPK_REQUIRE(p != nullptr, "no device address for the static scratch");
    return p;
}
}  // namespace
}  // namespace spk

using namespace spk;

extern "C" {

spk_status spk_rank_convstdp_noalloc(const void *in, spk_dtype itype, int64_t b, int64_t t, int64_t cin, int64_t h,
                                     int64_t w, float *kernel, int64_t cout, int64_t kh, int64_t kw, const void *out,
                                     int64_t oh, int64_t ow, const double *configs_host, int64_t nconf,
                                     const int32_t *winners, const int32_t *counts, int64_t count, int64_t sy,
                                     int64_t sx, const int64_t *pad4_host, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(b >= 0 && count >= 1 && cin >= 1 && kh >= 1 && kw >= 1, "invalid dims");
        const size_t need = convstdp_prepost_bytes(b, count, cin, kh, kw);
        if (need > kNoAllocScratchBytes)
            throw Error(SPK_ERR_ARGUMENT, "spk_rank_convstdp_noalloc: this call needs " + std::to_string(need) +
                                              " bytes of scratch but the static scratch holds " +
                                              std::to_string(kNoAllocScratchBytes) +
                                              " bytes; process fewer samples per call");
        convstdp_into(in, itype, b, t, cin, h, w, kernel, cout, kh, kw, out, oh, ow, configs_host, nconf, winners,
                      counts, count, sy, sx, pad4_host, scratch_address(), stream_of(stream));
    });
}

}  // extern "C"
