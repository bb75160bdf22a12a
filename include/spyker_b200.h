/*
 * spyker_b200 — C ABI of the B200 (sm_100a) spiking-CNN hot path.
 *
 * Drop-in seam: each entry point replaces one `Core::cuda_<op>` /
 * `Core::cpu_<op>` backend function of Spyker (declared through the
 * `Declare(...)` table of src/spyker/impl.h:196-322 and the sparse table
 * impl.h:328-356), with the same argument meaning, but over plain device
 * pointers, sizes and a CUDA stream instead of Spyker's Dyn/Tensor types.
 *
 * Conventions
 *  - Every pointer named `in`/`out`/`data`/`kernel`/`winners`/`counts`/`ws` is a
 *    DEVICE pointer unless the comment says "host".
 *  - Layouts are the reference's: spikes and potentials [B, T, C, H, W]
 *    row-major; conv kernels [Cout, Cin, KH, KW]; pads are (top, left,
 *    bottom, right) as in src/spyker/shape.cpp:35-50.
 *  - Scalars (thresholds, fill values) are passed as double and converted to
 *    the data type with a C cast, as the reference's Scalar does
 *    (src/spyker/utils.cpp:290-295).
 *  - Work is enqueued on `stream` (a cudaStream_t; NULL = legacy default).
 *    Calls never synchronise the stream unless documented.
 *  - Winners travel as int32 records [B, count, 5] = (c, t, z, y, x)
 *    (src/spyker/utils.h:483-502) plus int32 per-sample counts [B].
 *  - Entry points that need scratch memory take a caller-provided workspace
 *    (`ws`, `ws_bytes`); the matching `_workspace` query returns the bytes
 *    needed.  The library never allocates device memory on these paths.
 *  - Return value: SPK_OK or an error code; spk_last_error() gives the
 *    message of the calling thread's last failure.  Errors never throw.
 */
#ifndef SPYKER_B200_H
#define SPYKER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum
{
    SPK_OK = 0,
    SPK_ERR_ARGUMENT = 1,    /* bad shape / size / pointer (reference: SpykerCompare throws) */
    SPK_ERR_CUDA = 2,        /* a CUDA runtime call or launch failed */
    SPK_ERR_UNSUPPORTED = 3, /* data type or option not supported by this build */
    SPK_ERR_DEVICE = 4       /* a kernel reported an error through its device status word */
} spk_status;

/* Codes of the reference's `enum class Type` (src/spyker/utils.h:96-120). */
typedef enum
{
    SPK_I8 = 0,
    SPK_I16 = 1,
    SPK_I32 = 2,
    SPK_I64 = 3,
    SPK_U8 = 4,
    SPK_U16 = 5,
    SPK_U32 = 6,
    SPK_U64 = 7,
    SPK_F16 = 8,
    SPK_F32 = 9,
    SPK_F64 = 10
} spk_dtype;

/* Arithmetic of the spike x weight contraction. */
typedef enum
{
    SPK_CONV_FP32 = 0,   /* plain FP32 SIMT direct convolution */
    SPK_CONV_BF16X2 = 1, /* tcgen05 tensor cores, weights split in BF16 hi+lo, FP32 accumulate */
    SPK_CONV_BF16X3 = 2  /* tcgen05 tensor cores, three BF16 terms (exact for weights in [2^-6, 1]) */
} spk_conv_precision;

typedef void *spk_stream;

/* ---- library ------------------------------------------------------------ */
const char *spk_last_error(void);
const char *spk_version(void);
/* Number of CUDA devices, or -1 when the runtime is unusable. */
int spk_device_count(void);
/* Number of kernels this library has launched in the process (all threads). */
uint64_t spk_launch_count(void);
/* Device status word of the tensor-core kernels: 0 = no error, 1 = a bounded
 * wait timed out.  Synchronous; reset != 0 clears it. */
int spk_device_status(int reset);
/* Number of (pixel, step) rows of the fused layer whose thresholded
 * channel decision was within the FP32 error bound and was recomputed with
 * FP64 sums, since the last reset.  Synchronous; reset != 0 clears it. */
unsigned long long spk_recheck_count(int reset);
/* Number of rows of the fused layer's first-crossing search that even the
 * exact term sums left open (a potential within its bound of a rounding
 * boundary that decides) and that were recomputed from the F32 weights in
 * the oracle's FP64 order, since the last reset.  Synchronous; reset != 0
 * clears it. */
unsigned long long spk_recompute_count(int reset);
/* Schedule of the tensor-core conv / fused-layer kernels for the calls that
 * follow (0 = automatic): pipeline stages (2..6, capped by shared memory),
 * tensor-memory accumulators (1 or 2, where 2 fit), resident CTAs per SM.
 * Results do not depend on it; an autotuner picks it per layer shape.
 * Process-wide (not thread-safe). */
spk_status spk_set_conv_schedule(int stages, int nacc, int ctas_per_sm);

/* ---- host-side kernel generation (src/spyker/cpu/init.cpp) -------------- */
/* Global generator: replaces Core::random_seed (src/spyker/impl.cpp:37-43). */
void spk_random_seed(uint64_t seed);
/* kernel ~ N(mean, std) from the global mt19937 (cpu/init.cpp:45-49). host. */
spk_status spk_normal_kernel(double *kernel_host, int64_t n, double mean, double std);
/* Normalised Gaussian (cpu/init.cpp:51-62). host, [size, size]. */
spk_status spk_gaussian_kernel(double *kernel_host, int64_t size, double std);
/* Normalised Gabor, theta in radians (cpu/init.cpp:64-77). host. */
spk_status spk_gabor_kernel(double *kernel_host, int64_t size, double sigma, double theta, double gamma,
                            double lambda, double psi);
/* LoG kernel (cpu/init.cpp:79-90). host. */
spk_status spk_log_kernel(double *kernel_host, int64_t size, double std);

/* ---- coding (replaces Core::rank_code, impl.h:248; cpu/code.cpp:122) ---- */
/* in [B, X], out [B, T, X] cumulative spikes.  sort!=0: rank order, ties in
 * index order (stable); sort==0: latency code.  Images of more than 16384
 * values take a device-wide sort that needs the workspace (16*B*X bytes plus
 * 2*B*X, rounded up); smaller images need none. */
size_t spk_rank_code_workspace(int64_t b, int64_t x, int sort);
spk_status spk_rank_code(const void *in, spk_dtype itype, void *out, spk_dtype otype, int64_t b, int64_t t, int64_t x,
                         int sort, void *ws, size_t ws_bytes, spk_stream stream);

/* ---- elementwise (impl.h:240-264; cpu/fire.cpp, cpu/time.cpp) ----------- */
/* Core::threshold: in place, x <= threshold -> value. */
spk_status spk_threshold(void *data, spk_dtype type, int64_t n, double threshold, double value, spk_stream stream);
/* Core::rank_infinite: data [B, T, X], steps 0..T-2 set to value. */
spk_status spk_rank_infinite(void *data, spk_dtype type, int64_t b, int64_t t, int64_t x, double value,
                             spk_stream stream);
/* Core::rank_fire: out = in > threshold. */
spk_status spk_rank_fire(const void *in, spk_dtype itype, void *out, spk_dtype otype, int64_t n, double threshold,
                         spk_stream stream);
/* Core::rank_gather: in [B, T, X] -> out [B, X] first t with in > threshold (T if none). */
spk_status spk_rank_gather(const void *in, spk_dtype itype, void *out, spk_dtype otype, int64_t b, int64_t t,
                           int64_t x, double threshold, spk_stream stream);
/* Core::rank_scatter: in [B, X] -> out [B, T, X] = (t >= in). */
spk_status spk_rank_scatter(const void *in, spk_dtype itype, void *out, spk_dtype otype, int64_t b, int64_t t,
                            int64_t x, spk_stream stream);
/* Core::pad: in [N, H, W] -> out [N, H+top+bottom, W+left+right] (cpu/pool.cpp:41-51). */
spk_status spk_pad(const void *in, void *out, spk_dtype type, int64_t n, int64_t h, int64_t w, const int64_t *pad4_host,
                   double value, spk_stream stream);

/* ---- pooling (Core::rank_pool, impl.h:268; cpu/pool.cpp:53-86) ---------- */
/* in [N, H, W] planes -> out [N, OH, OW]; max over window, zero pad. */
spk_status spk_rank_pool(const void *in, void *out, spk_dtype type, int64_t n, int64_t h, int64_t w, int64_t oh,
                         int64_t ow, int64_t ky, int64_t kx, int64_t sy, int64_t sx, const int64_t *pad4_host,
                         spk_stream stream);

/* ---- lateral inhibition (Core::rank_inhibit, impl.h:272; cpu/inhibit.cpp) */
/* data [B, T, C, X] in place. */
spk_status spk_rank_inhibit(void *data, spk_dtype type, int64_t b, int64_t t, int64_t c, int64_t x, double threshold,
                            spk_stream stream);

/* ---- winner-take-all (Core::rank_convwta/rank_fcwta, impl.h:276-282) ---- */
size_t spk_rank_convwta_workspace(int64_t b, int64_t t, int64_t c, int64_t h, int64_t w);
/* in [B, T, C, H, W] -> winners [B, count, 5], counts [B] (cpu/wta.cpp:123-152). */
spk_status spk_rank_convwta(const void *in, spk_dtype type, int64_t b, int64_t t, int64_t c, int64_t h, int64_t w,
                            int64_t ry, int64_t rx, int64_t count, double threshold, int32_t *winners, int32_t *counts,
                            void *ws, size_t ws_bytes, spk_stream stream);
size_t spk_rank_fcwta_workspace(int64_t b, int64_t t, int64_t n);
/* in [B, T, N] -> winners (x = neuron) (cpu/wta.cpp:72-96). */
spk_status spk_rank_fcwta(const void *in, spk_dtype type, int64_t b, int64_t t, int64_t n, int64_t radius,
                          int64_t count, double threshold, int32_t *winners, int32_t *counts, void *ws, size_t ws_bytes,
                          spk_stream stream);

/* ---- STDP (Core::rank_convstdp/rank_fcstdp, impl.h:284-296) -------------- */
/* configs_host: [nconf, 5] = (positive, negative, stabilize, lower, upper),
 * STDPConfig of src/spyker/utils.h:505-524 (nconf <= 16). */
size_t spk_rank_convstdp_workspace(int64_t b, int64_t count, int64_t cin, int64_t h, int64_t w, int64_t kh,
                                   int64_t kw);
/* in [B, T, Cin, H, W] spikes, kernel [Cout, Cin, KH, KW] F32 updated in place,
 * out [B, T, Cout, OH, OW] spikes; sequential in (sample, winner) order per
 * feature map (cpu/stdp.cpp:99-169). */
spk_status spk_rank_convstdp(const void *in, spk_dtype itype, int64_t b, int64_t t, int64_t cin, int64_t h, int64_t w,
                             float *kernel, int64_t cout, int64_t kh, int64_t kw, const void *out, int64_t oh,
                             int64_t ow, const double *configs_host, int64_t nconf, const int32_t *winners,
                             const int32_t *counts, int64_t count, int64_t sy, int64_t sx, const int64_t *pad4_host,
                             void *ws, size_t ws_bytes, spk_stream stream);
/* No counterpart in the reference.  The same update as spk_rank_convstdp for
 * callers that cannot allocate device memory (hosts whose allocator owns all
 * of the device's memory, or C callers without a device allocator): its
 * scratch lives in a static 32 MiB device array that
 * every GPU loading the library holds until exit, so the call allocates
 * nothing.  Calls needing more scratch than that (2*B*count*Cin*KH*KW bytes
 * plus 2*B*count, each rounded up to 256) fail with SPK_ERR_ARGUMENT; split
 * the batch.
 * Every call looks up the array's device address on the current device (a
 * host-side lookup, no stream work); the first call on a device may also
 * load the library's device code, so make it before any stream capture.
 * All calls share the array, so calls that overlap on the GPU (different
 * streams, or other threads) race. */
spk_status spk_rank_convstdp_noalloc(const void *in, spk_dtype itype, int64_t b, int64_t t, int64_t cin, int64_t h,
                                     int64_t w, float *kernel, int64_t cout, int64_t kh, int64_t kw, const void *out,
                                     int64_t oh, int64_t ow, const double *configs_host, int64_t nconf,
                                     const int32_t *winners, const int32_t *counts, int64_t count, int64_t sy,
                                     int64_t sx, const int64_t *pad4_host, spk_stream stream);
/* The two halves of spk_rank_convstdp (cpu/stdp.cpp:99-169), for STDP over
 * winners gathered from several GPUs: spk_rank_convstdp_prepost writes, for
 * every winner slot, the first-spike times of its receptive field
 * pre [B, count, Cin*KH*KW] u16 (T = silent or padding) and of the winner
 * post [B, count] u16; spk_stdp_scan applies the reference's ordered update
 * (sample after sample, slot after slot) to a kernel from such arrays.  The
 * map of a winner is record field `field` (2 = z for conv, 4 = x for fc);
 * pre of slot (s, j) starts at s * pre_sample_stride + j * pre_slot_stride.
 * f32_rule != 0 takes the event-list update of sparse/stdp.cpp:95-97. */
size_t spk_rank_convstdp_prepost_workspace(int64_t b, int64_t cin, int64_t h, int64_t w);
spk_status spk_rank_convstdp_prepost(const void *in, spk_dtype itype, int64_t b, int64_t t, int64_t cin, int64_t h,
                                     int64_t w, int64_t cout, int64_t kh, int64_t kw, const void *out, int64_t oh,
                                     int64_t ow, const int32_t *winners, const int32_t *counts, int64_t count,
                                     int64_t sy, int64_t sx, const int64_t *pad4_host, uint16_t *pre, uint16_t *post,
                                     void *ws, size_t ws_bytes, spk_stream stream);
spk_status spk_stdp_scan(float *kernel, int64_t nmaps, int64_t k, int64_t b, int64_t count, int64_t field,
                         const int32_t *winners, const int32_t *counts, const uint16_t *pre, int64_t pre_sample_stride,
                         int64_t pre_slot_stride, const uint16_t *post, const double *configs_host, int64_t nconf,
                         int f32_rule, spk_stream stream);
/* The scan of several networks in one launch (kernels [N, maps, k]): network
 * n walks the samples order[net_offsets[n] .. net_offsets[n+1]) (global sample
 * indexes into winners / counts / pre / post; null order = the range itself)
 * in that order with its configs net_configs[n][nconf][5] (positive, negative,
 * stabilize, lower, upper).  net_offsets, order and net_configs are device
 * arrays.  Each network's update equals spk_stdp_scan over its samples in
 * that order (the reference's per-sample sequential rule, cpu/stdp.cpp:99-169). */
spk_status spk_stdp_scan_nets(float *kernels, int64_t nnets, int64_t nmaps, int64_t k, int64_t b, int64_t count,
                              int64_t field, const int32_t *winners, const int32_t *counts, const uint16_t *pre,
                              int64_t pre_sample_stride, int64_t pre_slot_stride, const uint16_t *post,
                              const int64_t *net_offsets, const int32_t *order, const double *net_configs,
                              int64_t nconf, int f32_rule, spk_stream stream);
size_t spk_rank_fcstdp_workspace(int64_t b, int64_t t, int64_t ni);
/* in [B, T, I], kernel [O, I] F32 in place, out [B, T, O] (cpu/stdp.cpp:42-97). */
spk_status spk_rank_fcstdp(const void *in, spk_dtype itype, int64_t b, int64_t t, int64_t ni, float *kernel,
                           int64_t no, const void *out, const double *configs_host, int64_t nconf,
                           const int32_t *winners, const int32_t *counts, int64_t count, void *ws, size_t ws_bytes,
                           spk_stream stream);

/* ---- convolution (Core::conv, impl.h:224; cuda/conv.cu:257) ------------- */
/* in [N, Cin, H, W] (U8 spikes or F32), kernel [Cout, Cin, KH, KW] F32,
 * out [N, Cout, OH, OW] F32.  N folds batch and time. */
size_t spk_conv_workspace(int64_t n, int64_t cin, int64_t h, int64_t w, int64_t cout, int64_t kh, int64_t kw,
                          int precision);
spk_status spk_conv(const void *in, spk_dtype itype, const float *kernel, float *out, int64_t n, int64_t cin, int64_t h,
                    int64_t w, int64_t cout, int64_t kh, int64_t kw, int64_t sy, int64_t sx, const int64_t *pad4_host,
                    int precision, void *ws, size_t ws_bytes, spk_stream stream);

/* ---- fused layer: conv -> threshold -> inhibit -> fire + convwta -------- */
/* No single reference function: the composition of Core::conv, threshold,
 * rank_inhibit, rank_fire and rank_convwta (impl.h:224-282) that every STDP
 * training step of the reference's examples performs
 * (examples/kheradpisheh_mnist_dense.py:62-64), in one tcgen05 kernel whose
 * epilogue never writes the potentials.  in [B, T, Cin, H, W] U8 spikes,
 * kernel [Cout, Cin, KH, KW] F32; spikes out [B, T, Cout, OH, OW] U8 =
 * fire(out, fire_threshold) and winners = convwta(out, (ry, rx), count,
 * wta_threshold) with out = inhibit(threshold(conv(in), threshold, value),
 * inhibit_threshold).  Requires T <= 32, Cout >= 2, fire/WTA thresholds >= 0
 * and a tensor-core precision.  With pool_ky > 0 it also writes pooled =
 * pool(spikes, (pool_ky, pool_kx)) (stride = window, no padding; the
 * rank_pool of impl.h:268 on the spikes), [B, T, Cout, OH / pool_ky,
 * OW / pool_kx] U8; pooled may be null when pool_ky == 0.  count == 0
 * skips the winner selection (winners and counts may then be null).  The
 * workspace query returns 0 for layers whose accumulators (terms x Cout,
 * Cout rounded up to 16) exceed the 512 tensor-memory columns of a CTA even
 * with two terms (a three-term request above 170 channels keeps two: every
 * near-threshold decision is re-made exactly at either split).  With no
 * negative weight, cumulative 0/1 input and value <= the inhibit / fire / WTA
 * thresholds <= threshold, the layer runs as a first-crossing search on u8
 * weight digits (exact integer sums) instead of the dense kernel; results
 * are the same.  spk_recheck_count / spk_recompute_count count its rows
 * re-decided from exact sums and recomputed from the F32 weights. */
size_t spk_conv_fire_wta_workspace(int64_t b, int64_t t, int64_t cin, int64_t h, int64_t w, int64_t cout, int64_t kh,
                                   int64_t kw, int64_t sy, int64_t sx, const int64_t *pad4_host, int precision);
spk_status spk_conv_fire_wta(const void *in, spk_dtype itype, const float *kernel, int64_t b, int64_t t, int64_t cin,
                             int64_t h, int64_t w, int64_t cout, int64_t kh, int64_t kw, int64_t sy, int64_t sx,
                             const int64_t *pad4_host, double threshold, double value, double inhibit_threshold,
                             double fire_threshold, int64_t ry, int64_t rx, int64_t count, double wta_threshold,
                             uint8_t *spikes, int32_t *winners, int32_t *counts, int64_t pool_ky, int64_t pool_kx,
                             uint8_t *pooled, int precision, void *ws, size_t ws_bytes, spk_stream stream);
/* Several networks in one launch (a hyperparameter sweep): kernels
 * [N, Cout, Cin, KH, KW]; samples net_offsets_host[n] .. [n+1] belong to
 * network n (host array, checked: each network must start on a tile, i.e.
 * net_offsets[n] * OH * OW a multiple of 128 / pow2ceil(T), so pad batches);
 * sample_net [B] int32 and net_threshold [N] F32 are device arrays (the
 * threshold of Core::threshold per network; the other thresholds shared).
 * Per sample the results equal spk_conv_fire_wta with that network's kernel
 * and threshold. */
size_t spk_conv_fire_wta_nets_workspace(int64_t nnets, int64_t b, int64_t t, int64_t cin, int64_t h, int64_t w,
                                        int64_t cout, int64_t kh, int64_t kw, int64_t sy, int64_t sx,
                                        const int64_t *pad4_host, int precision);
spk_status spk_conv_fire_wta_nets(const void *in, spk_dtype itype, const float *kernels, int64_t nnets,
                                  const int64_t *net_offsets_host, const int32_t *sample_net,
                                  const float *net_threshold, int64_t b, int64_t t, int64_t cin, int64_t h, int64_t w,
                                  int64_t cout, int64_t kh, int64_t kw, int64_t sy, int64_t sx,
                                  const int64_t *pad4_host, double value, double inhibit_threshold,
                                  double fire_threshold, int64_t ry, int64_t rx, int64_t count, double wta_threshold,
                                  uint8_t *spikes, int32_t *winners, int32_t *counts, int64_t pool_ky, int64_t pool_kx,
                                  uint8_t *pooled, int precision, void *ws, size_t ws_bytes, spk_stream stream);

/* ---- fully connected (Core::fc / signfc, impl.h:228-236) ---------------- */
/* in [R, I] (U8 or F32), kernel [O, I] F32 -> out [R, O] F32. */
spk_status spk_fc(const void *in, spk_dtype itype, const float *kernel, float *out, int64_t r, int64_t ni, int64_t no,
                  int sign, spk_stream stream);

/* ---- filter banks (Core::dog/gabor/log, impl.h:200-212; cpu/dog.cpp) ---- */
/* which: 0 DoG, 1 Gabor, 2 LoG.  in [N, H, W] F32 planes; kernel F32
 * [2, F, KH, KW] (DoG, LoG) or [F, KH, KW] (Gabor); out [N, F or 2F, OH, OW]. */
spk_status spk_filter(int which, const float *in, const float *kernel, float *out, int64_t n, int64_t h, int64_t w,
                      int64_t f, int64_t kh, int64_t kw, int64_t oh, int64_t ow, const int64_t *pad4_host,
                      spk_stream stream);

/* ---- temporal backprop (Core::backward/labelize/fcbackward, impl.h:306-318) */
/* in/out [B, N] F32 first-spike times; target [B] int64 (cpu/backprop.cpp:40-62). */
spk_status spk_backward(const float *in, float *out, const int64_t *target, int64_t b, int64_t n, int64_t time,
                        double gamma, spk_stream stream);
/* in [B, T, N] -> out [B] int64 (cpu/backprop.cpp:68-99). */
spk_status spk_labelize(const void *in, spk_dtype type, int64_t *out, int64_t b, int64_t t, int64_t n,
                        double threshold, spk_stream stream);
/* kernel [O, I] F32 updated; in [B, I], out/grad [B, O], next [B, I] F32;
 * bp_host = (sfactor, lrate, lrf, lambda), sfactor updated on return
 * (synchronises the stream) (cpu/backprop.cpp:105-160). */
size_t spk_fcbackward_workspace(int64_t no, int64_t ni);
spk_status spk_fcbackward(float *kernel, int64_t no, int64_t ni, const float *in, const float *out, const float *grad,
                          float *next, int64_t b, float *bp_host, void *ws, size_t ws_bytes, spk_stream stream);

/* ---- first-spike layers trained through their spike times ----
 * The rule of the fc backward above (select = (t_in < t_out) * grad,
 * next = sum kernel * select; cpu/backprop.cpp:116-144) written for a conv
 * weight shared over output pixels (fc = the 1x1 case), as derivatives with
 * grad_out = dL/dt_out (= -grad of the target rule, cpu/backprop.cpp:40-52):
 *   grad_kernel[z,c,ky,kx] = -sum_{b,oy,ox} grad_out[b,z,oy,ox] * [t_in[b,c,iy,ix] < t_out[b,z,oy,ox]]
 *   grad_in[b,c,iy,ix]     =  sum_{z,ky,kx} kernel[z,c,ky,kx] * grad_out[b,z,oy,ox] * [same mask]
 * (iy, ix) = (oy*sy - top + ky, ox*sx - left + kx); padding never spikes.
 * Times are F32 [B, C, H, W] (T = never).  Replaces nothing in the reference
 * (its conv layers have no backward); the fc case equals Core::fcbackward's
 * select / next with lrate = lambda = 0 (impl.h:316-318). */
/* Earliest spike of each window (pool of cumulative spikes, cpu/pool.cpp:41-86);
 * padding = `time` (never).  stride2/pad4/kernel2 on the host. */
spk_status spk_fst_pool(const float *in, int64_t b, int64_t c, int64_t h, int64_t w, float *out, int64_t oh,
                        int64_t ow, const int64_t *kernel2_host, const int64_t *stride2_host, const int64_t *pad4_host,
                        double time, spk_stream stream);
/* Gradient of each window to its earliest in-range input (first in raster
 * order on ties); overlapping windows add up. */
spk_status spk_fst_pool_backward(const float *in, int64_t b, int64_t c, int64_t h, int64_t w, const float *grad_out,
                                 int64_t oh, int64_t ow, const int64_t *kernel2_host, const int64_t *stride2_host,
                                 const int64_t *pad4_host, float *grad_in, spk_stream stream);
/* grad_in [B, Cin, H, W] and / or grad_kernel [Cout, Cin, KH, KW] (either may be
 * null; grad_in needs H*W <= 1024).  grad_kernel is summed in FP64 in a fixed
 * order (deterministic); the workspace holds its per-group partial sums. */
size_t spk_fst_conv_backward_workspace(int64_t b, int64_t cin, int64_t cout, int64_t kh, int64_t kw);
spk_status spk_fst_conv_backward(const float *t_in, int64_t b, int64_t cin, int64_t h, int64_t w,
                                 const float *kernel, int64_t cout, int64_t kh, int64_t kw, const float *t_out,
                                 const float *grad_out, int64_t oh, int64_t ow, const int64_t *stride2_host,
                                 const int64_t *pad4_host, float *grad_in, float *grad_kernel, void *ws,
                                 size_t ws_bytes, spk_stream stream);
/* Forward of a first-spike conv layer on the tensor cores in one fused
 * kernel: t_out[b,z,oy,ox] = first t in 0..T-1 with potential(t) > threshold,
 * T when none, where potential(t) = conv of the cumulative spikes [t_in <= t]
 * (BF16x2/x3 split weights, the FP64 sum of the split terms rounded once to
 * F32, exactly as spk_conv's potentials followed by spk_rank_gather); the
 * potentials are never written.  t_in [B, Cin, H, W] F32 (values >= T =
 * never); T <= 126; all output channels in one CTA (workspace query 0
 * otherwise). */
size_t spk_fst_conv_times_workspace(int64_t b, int64_t cin, int64_t h, int64_t w, int64_t cout, int64_t kh,
                                    int64_t kw, int64_t time, int precision);
spk_status spk_fst_conv_times(const float *t_in, int64_t b, int64_t cin, int64_t h, int64_t w, const float *kernel,
                              int64_t cout, int64_t kh, int64_t kw, int64_t sy, int64_t sx, const int64_t *pad4_host,
                              int64_t time, double threshold, float *t_out, int precision, void *ws, size_t ws_bytes,
                              spk_stream stream);
/* The potential one step before each output spike, in FP64:
 * out[b,z,oy,ox] = sum kernel[z,c,ky,kx] * [t_in[b,c,iy,ix] < t_out[b,z,oy,ox]]
 * (the potential-level loss sum g * out has grad_kernel as its exact gradient). */
spk_status spk_fst_conv_prespike(const float *t_in, int64_t b, int64_t cin, int64_t h, int64_t w,
                                 const float *kernel, int64_t cout, int64_t kh, int64_t kw, const float *t_out,
                                 int64_t oh, int64_t ow, const int64_t *stride2_host, const int64_t *pad4_host,
                                 double *out, spk_stream stream);

/* ---- Canny edges (Core::canny, impl.h; cpu/canny.cpp:9-214) and
 * two-level quantize (Core::quantize; cpu/fire.cpp:116-131). ---- */
/* u8 images [n, h, w] -> u8 edges [n, h, w]; low / high converted to u8;
 * workspace spk_canny_workspace(n, h, w) bytes. */
int64_t spk_canny_workspace(int64_t n, int64_t h, int64_t w);
spk_status spk_canny(const uint8_t *in, uint8_t *out, int64_t n, int64_t h, int64_t w, double low, double high,
                     void *ws, int64_t ws_bytes, spk_stream stream);
/* in place: x < middle -> lower, else upper (values converted to the type). */
spk_status spk_quantize(void *data, spk_dtype type, int64_t n, double lower, double middle, double upper,
                        spk_stream stream);

/* ---- IDX (MNIST) files (Helper::mnistData / mnistLabel, helper/mnist.cpp:10-60)
 * read into caller memory (pinned host memory for an overlapped upload). ---- */
/* magic 2049 (labels: shape [N], ndim 1) or 2051 (images: [N, 1, rows, cols],
 * ndim 4); offset = the payload's byte offset.  Fails on a missing file, a
 * short header or another magic. */
spk_status spk_idx_shape(const char *path, int32_t magic, int64_t *shape, int64_t *ndim, int64_t *offset);
/* bytes of the payload at offset into dst, with up to `threads` positioned
 * reads; fails on a short file. */
spk_status spk_idx_read(const char *path, int64_t offset, void *dst, int64_t bytes, int threads);

/* ---- ZCA whitening (Core::zca_fit / zca_trans / zca_split, impl.h:212-222;
 * cpu/zca.cpp:67-155) with FP64 accumulation.  The eigendecomposition of the
 * covariance between the two steps is the caller's (FP64, on the GPU). ---- */
/* x [N, D] F32 -> mean [D] and covariance [D, D] (divisor N - 1), FP64.
 * work: spk_zca_stats_workspace(n, d) bytes (split-K partial sums; 0 = none). */
int64_t spk_zca_stats_workspace(int64_t n, int64_t d);
spk_status spk_zca_stats(const float *x, int64_t n, int64_t d, double *mean, double *cov, void *work,
                         int64_t work_bytes, spk_stream stream);
/* vectors [D, D] (eigenvectors in columns, row-major), values [D] ->
 * trans = U diag(1 / sqrt(max(values, 0) + epsilon)) U^T, FP64; work [D]. */
spk_status spk_zca_matrix(const double *vectors, const double *values, int64_t d, double epsilon, double *work,
                          double *trans, spk_stream stream);
/* out [N, D] F32 = (x - mean) trans (FP64 sums); out must not alias x. */
spk_status spk_zca_transform(const float *x, int64_t n, int64_t d, const double *mean, const double *trans, float *out,
                             spk_stream stream);
/* [N, D] -> [N, 2, D] = (max(x, 0), max(-x, 0)), F32 or F64. */
spk_status spk_zca_split(const void *in, spk_dtype type, void *out, int64_t n, int64_t d, spk_stream stream);

/* ---- rate (Poisson) coding (Core::rate_code / rate_fire / rate_gather /
 * rate_pool, impl.h:295-309) ----
 * Counts are cumulative: step t holds each neuron's spikes up to t. */
/* cpu/code.cpp:134-243: every position's rank (sort) or latency time picks a
 * row of the inter-spike interval table (cpu/init.cpp:120-149); a Poisson
 * process per position counts spikes.  Rows are the reference's multisets,
 * the draws come from a counter-based generator seeded from the library's
 * global generator (spk_random_seed), so results match the reference in
 * distribution, not draw for draw.  out [B, T, X]. */
size_t spk_rate_code_workspace(int64_t b, int64_t t, int64_t x, int sort);
spk_status spk_rate_code(const void *in, spk_dtype itype, void *out, spk_dtype otype, int64_t b, int64_t t, int64_t x,
                         int sort, void *ws, size_t ws_bytes, spk_stream stream);
/* The interval table [time][1024] U16 the rate code uses (host memory). */
void spk_rate_interval_table(int64_t time, uint16_t *out_host);
/* cpu/fire.cpp:84-113: in [B, T, X] -> running spike counts [B, T, X]. */
spk_status spk_rate_fire(const void *in, spk_dtype itype, void *out, spk_dtype otype, int64_t b, int64_t t, int64_t x,
                         double threshold, spk_stream stream);
/* cpu/time.cpp:87-92: the last step's counts, [B, T, X] -> [B, X]. */
spk_status spk_rate_gather(const void *in, spk_dtype itype, void *out, spk_dtype otype, int64_t b, int64_t t,
                           int64_t x, spk_stream stream);
/* cpu/pool.cpp:88-137: per window the position of highest rate (rates
 * [B, C, H, W]; first in row-major window order on ties), its values at
 * every step; in/out [B, T, C, H, W] / [B, T, C, OH, OW]; no padding. */
spk_status spk_rate_pool(const void *in, const void *rates, spk_dtype type, spk_dtype rtype, void *out, int64_t b,
                         int64_t t, int64_t c, int64_t h, int64_t w, int64_t oh, int64_t ow, const int64_t *kernel2_host,
                         const int64_t *stride2_host, const int64_t *pad4_host, spk_stream stream);

/* ---- event lists (the `sparse_*` table of impl.h:328-356; src/spyker/sparse) ----
 * A sparse spike tensor [U, T, C, H, W] (SparseTensor, utils.h:369-420; Sparse5,
 * base.h:493-528) is one CSR array on the device:
 *   offsets int64 [U*T + 1]: list i = u*T + t holds events offsets[i] .. offsets[i+1]-1;
 *   events  uint32: x | y << 8 | z << 16 (8-bit coordinates as Spridx).
 * Event order inside a list is the reference's.  Producers write into
 * caller buffers of at least the stated capacity (the worst case), so no call
 * waits for the host; offsets[U*T] is the number of events written.
 * C, H, W (and conv outputs) are limited to 256, T to 16384. */

/* Sparse::code, sparse/code.cpp:39-130: one event at the rank-order (sort) or
 * latency first-spike time of every position (none when it is >= T), lists in
 * (z, y, x) order.  cap >= U*C*H*W. */
size_t spk_sparse_code_workspace(int64_t u, int64_t t, int64_t c, int64_t h, int64_t w);
spk_status spk_sparse_code(const void *in, spk_dtype itype, int64_t u, int64_t c, int64_t h, int64_t w, int64_t t,
                           int sort, int64_t *offsets, uint32_t *events, int64_t cap, void *ws, size_t ws_bytes,
                           spk_stream stream);
/* SparseTensor(Tensor, threshold), sparse/opers.cpp:59-86: an event at the
 * first step whose value exceeds the threshold.  cap >= U*C*H*W. */
size_t spk_sparse_from_dense_workspace(int64_t u, int64_t t, int64_t c, int64_t h, int64_t w);
spk_status spk_sparse_from_dense(const void *in, spk_dtype itype, int64_t u, int64_t t, int64_t c, int64_t h,
                                 int64_t w, double threshold, int64_t *offsets, uint32_t *events, int64_t cap,
                                 void *ws, size_t ws_bytes, spk_stream stream);
/* SparseTensor::dense, sparse/opers.cpp:88-104: cumulative spikes [U, T, C, H, W];
 * Sparse::gather, sparse/opers.cpp:106-118: first event time [U, C, H, W] (T when none). */
size_t spk_sparse_dense_workspace(int64_t u, int64_t c, int64_t h, int64_t w);
spk_status spk_sparse_to_dense(const int64_t *offsets, const uint32_t *events, int64_t u, int64_t t, int64_t c,
                               int64_t h, int64_t w, void *out, spk_dtype otype, void *ws, size_t ws_bytes,
                               spk_stream stream);
spk_status spk_sparse_gather(const int64_t *offsets, const uint32_t *events, int64_t u, int64_t t, int64_t c,
                             int64_t h, int64_t w, void *out, spk_dtype otype, void *ws, size_t ws_bytes,
                             spk_stream stream);
/* Sparse::pad, sparse/pad.cpp:37-55: coordinates shifted by (top, left), 8-bit
 * wrap.  cap >= in_cap (the input's event capacity). */
spk_status spk_sparse_pad(const int64_t *offsets, const uint32_t *events, int64_t in_cap, int64_t u, int64_t t,
                          int64_t c, int64_t h, int64_t w, const int64_t *pad4_host, int64_t *out_offsets,
                          uint32_t *out_events, int64_t cap, spk_stream stream);
/* Sparse::pool, sparse/pool.cpp:37-64: the first event of every pooled cell;
 * stride must equal the kernel.  cap >= min(in_cap, U*C*OH*OW). */
size_t spk_sparse_pool_workspace(int64_t u, int64_t c, int64_t oh, int64_t ow, int64_t in_cap);
spk_status spk_sparse_pool(const int64_t *offsets, const uint32_t *events, int64_t in_cap, int64_t u, int64_t t,
                           int64_t c, int64_t h, int64_t w, const int64_t *kernel2_host, const int64_t *stride2_host,
                           const int64_t *pad4_host, int64_t oh, int64_t ow, int64_t *out_offsets,
                           uint32_t *out_events, int64_t cap, void *ws, size_t ws_bytes, spk_stream stream);
/* Sparse::inhibit, sparse/inhibit.cpp:37-65: per pixel only the channel of its
 * first event survives.  cap >= in_cap. */
size_t spk_sparse_inhibit_workspace(int64_t u, int64_t h, int64_t w, int64_t in_cap);
spk_status spk_sparse_inhibit(const int64_t *offsets, const uint32_t *events, int64_t in_cap, int64_t u, int64_t t,
                              int64_t c, int64_t h, int64_t w, int64_t *out_offsets, uint32_t *out_events, int64_t cap,
                              void *ws, size_t ws_bytes, spk_stream stream);
/* Sparse::conv, sparse/conv.cpp:42-160: incremental F32 potentials and fire
 * once above threshold; stride must be 1; kernel F32 [Cout, C, KH, KW].
 * cap >= U*Cout*OH*OW. */
size_t spk_sparse_conv_workspace(int64_t u, int64_t t, int64_t h, int64_t w, int64_t cout, int64_t kh, int64_t kw,
                                 const int64_t *pad4_host);
spk_status spk_sparse_conv(const int64_t *offsets, const uint32_t *events, int64_t u, int64_t t, int64_t c, int64_t h,
                           int64_t w, const float *kernel, int64_t cout, int64_t kh, int64_t kw, double threshold,
                           const int64_t *stride2_host, const int64_t *pad4_host, int64_t *out_offsets,
                           uint32_t *out_events, int64_t cap, void *ws, size_t ws_bytes, spk_stream stream);
/* Sparse::convwta, sparse/wta.cpp:44-95 -> winners [U, count, 5] = (0, t, z, y, x), counts [U]. */
spk_status spk_sparse_convwta(const int64_t *offsets, const uint32_t *events, int64_t u, int64_t t, int64_t c,
                              int64_t h, int64_t w, const int64_t *radius2_host, int64_t count, int32_t *winners,
                              int32_t *counts, spk_stream stream);
/* Conv::stdp(SparseTensor), sparse/stdp.cpp:41-133 (F32 update arithmetic). */
size_t spk_sparse_stdp_workspace(int64_t u, int64_t count, int64_t c, int64_t h, int64_t w, int64_t kh, int64_t kw,
                                 const int64_t *pad4_host);
spk_status spk_sparse_stdp(const int64_t *offsets, const uint32_t *events, int64_t u, int64_t t, int64_t c, int64_t h,
                           int64_t w, float *kernel, int64_t cout, int64_t kh, int64_t kw, const double *configs_host,
                           int64_t nconf, const int32_t *winners, const int32_t *counts, int64_t count,
                           const int64_t *pad4_host, void *ws, size_t ws_bytes, spk_stream stream);

#ifdef __cplusplus
}
#endif

#endif /* SPYKER_B200_H */
