// Tensor-core (tcgen05) spike x weight convolution with BF16-split weights.
//
// Implicit GEMM: D[m, n] = sum_k A[m, k] * W[n, k] with
//   m = (image, oy, ox) over N*OH*OW output positions (N folds batch, time),
//   k = (c, ky, kx) over Cin*KH*KW (the reference's kernel flattening),
//   A[m, k] = spike u8 of the receptive field (0/1, exact in BF16).
// Each F32 weight is split into BF16 terms w = h + m (+ l) (h = bf16(w),
// m = bf16(w - h), l = bf16(w - h - m)); every term gets its own FP32
// accumulator in tensor memory, so each partial sum stays exact for weights
// in [2^-6, 1] and the terms are added once in FP64 and rounded once to F32:
// BF16X3 reproduces the exactly rounded potential, BF16X2 (hi+lo) is within
// 2^-18 relative.
//
// CTA (persistent, 128 threads): per 128-row M tile and N tile, K is walked in
// 64-wide blocks through a two-stage shared-memory ring.  All threads gather
// the A block (u8 -> BF16) into the K-major no-swizzle canonical layout; the
// pre-split weight block is already stored in global memory in exactly that
// layout and is copied with 16-byte loads.  Thread 0 issues the tcgen05.mma
// instructions (M=128, N=n_tile, K=16) and commits them to the stage's
// mbarrier; the epilogue reads the accumulators with tcgen05.ld.  Every
// mbarrier wait is bounded: on timeout the kernel records an error in the
// device status word (spk_device_status) and leaves.
#include <algorithm>

#include "conv_tc.cuh"
#include "tc_ptx.cuh"

#include <cuda_bf16.h>

namespace spk
{
static __device__ int g_tc_status;

namespace
{
using namespace tc;

constexpr int BM = 128, BK = 64, kTcThreads = 128;
constexpr uint32_t kMaxProbes = 1u << 22;
constexpr int kMaxK = 4096;

struct TcParams
{
    const uint8_t *in;
    const uint4 *wimg;
    float *out;
    int64_t M, tiles, chw, ohw;
    int cin, h, w, cout, kh, kw, oh, ow, sy, sx, top, left;
    int K, kblocks, n_tile, n_tiles, nsplit;
    uint32_t tmem_cols, idesc;
};

__device__ __forceinline__ uint32_t bf16_bits(float v)
{
    return uint32_t(__bfloat16_as_ushort(__float2bfloat16_rn(v)));
}

// Weight images: [n_tiles][kblocks][nsplit][n_tile x 64] BF16 in the
// K-major no-swizzle layout (8-row groups of 1024 B, 8 K-chunks of 128 B,
// 16 B per row).  One thread per (n_tile block, k block, row, K chunk).
__global__ void split_weights_kernel(const float *__restrict__ kernel, uint4 *__restrict__ wimg, int cout, int K,
                                     int kblocks, int n_tile, int n_tiles, int nsplit)
{
    const int64_t total = int64_t(n_tiles) * kblocks * n_tile * 8;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x)
    {
        const int kc = int(i % 8);
        const int nl = int((i / 8) % n_tile);
        const int kb = int((i / (8 * n_tile)) % kblocks);
        const int nt = int(i / (int64_t(8) * n_tile * kblocks));
        const int n = nt * n_tile + nl;
        uint32_t parts[3][4];
#pragma unroll
        for (int e = 0; e < 8; e += 2)
        {
            uint32_t lo[3], hi[3];
#pragma unroll
            for (int q = 0; q < 2; ++q)
            {
                const int k = kb * BK + kc * 8 + e + q;
                const float wv = (n < cout && k < K) ? kernel[int64_t(n) * K + k] : 0.f;
                const __nv_bfloat16 h = __float2bfloat16_rn(wv);
                const float r1 = __fsub_rn(wv, __bfloat162float(h));
                const __nv_bfloat16 m = __float2bfloat16_rn(r1);
                const float r2 = __fsub_rn(r1, __bfloat162float(m));
                const __nv_bfloat16 l = __float2bfloat16_rn(r2);
                const uint32_t b0 = __bfloat16_as_ushort(h), b1 = __bfloat16_as_ushort(m), b2 = __bfloat16_as_ushort(l);
                if (q == 0)
                    lo[0] = b0, lo[1] = b1, lo[2] = b2;
                else
                    hi[0] = b0, hi[1] = b1, hi[2] = b2;
            }
#pragma unroll
            for (int p = 0; p < 3; ++p) parts[p][e / 2] = lo[p] | (hi[p] << 16);
        }
        const int64_t block = (int64_t(nt) * kblocks + kb) * nsplit;
        for (int p = 0; p < nsplit; ++p)
        {
            const int64_t idx = (block + p) * (int64_t(n_tile) * 8) + (nl / 8) * 64 + kc * 8 + (nl % 8);
            wimg[idx] = make_uint4(parts[p][0], parts[p][1], parts[p][2], parts[p][3]);
        }
    }
}

__device__ __forceinline__ bool wait_bounded(uint64_t *bar, uint32_t parity)
{
    for (uint32_t i = 0; i < kMaxProbes; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    atomicExch(&g_tc_status, 1);
    return false;
}

__global__ void __launch_bounds__(kTcThreads, 1) conv_tc_kernel(TcParams P)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmem_slot;

    const int tid = threadIdx.x, warp = tid >> 5;
    const int a_bytes = BM * BK * 2;                  // 16 KB
    const int b_bytes = P.nsplit * P.n_tile * BK * 2;  // nsplit x n_tile x 128 B
    unsigned char *sA[2] = {smem, smem + a_bytes};
    unsigned char *sB[2] = {smem + 2 * a_bytes, smem + 2 * a_bytes + b_bytes};
    int4 *tab = reinterpret_cast<int4 *>(smem + 2 * a_bytes + 2 * b_bytes);

    // k -> (offset within the image block, ky, kx, valid)
    for (int k = tid; k < P.kblocks * BK; k += blockDim.x)
    {
        const int khw = P.kh * P.kw;
        const int c = k / khw, r = k % khw, ky = r / P.kw, kx = r % P.kw;
        tab[k] = make_int4(c * P.h * P.w + ky * P.w + kx, ky, kx, k < P.K ? 1 : 0);
    }
    if (tid == 0)
    {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        fence_mbar_init();
    }
    if (warp == 0)
    {
        tmem_alloc(&tmem_slot, P.tmem_cols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    uint32_t uses[2] = {0, 0}, waited[2] = {0, 0};
    uint32_t it = 0;
    bool failed = false;

    for (int64_t tile = blockIdx.x; tile < P.tiles && !failed; tile += gridDim.x)
    {
        const int64_t mt = tile / P.n_tiles;
        const int nt = int(tile % P.n_tiles);
        const int64_t m = mt * BM + tid;
        const bool row_ok = m < P.M;
        int64_t img = 0, pix = 0;
        int iy0 = 0, ix0 = 0;
        if (row_ok)
        {
            img = m / P.ohw;
            pix = m % P.ohw;
            const int oy = int(pix / P.ow), ox = int(pix % P.ow);
            iy0 = oy * P.sy - P.top;
            ix0 = ox * P.sx - P.left;
        }
        const int64_t rowoff = img * P.chw + int64_t(iy0) * P.w + ix0;

        for (int kb = 0; kb < P.kblocks; ++kb, ++it)
        {
            const int st = it & 1;
            if (waited[st] < uses[st])
            {
                const bool ok = wait_bounded(&mbar[st], (uses[st] - 1) & 1);
                if (__syncthreads_or(!ok))
                {
                    failed = true;
                    break;
                }
                waited[st] = uses[st];
            }
            // A block: row tid, 8 chunks of 8 K values.
            unsigned char *a = sA[st] + (tid / 8) * 1024 + (tid % 8) * 16;
#pragma unroll 2
            for (int kc = 0; kc < 8; ++kc)
            {
                uint32_t pk[4];
#pragma unroll
                for (int e = 0; e < 8; e += 2)
                {
                    uint32_t v2[2];
#pragma unroll
                    for (int q = 0; q < 2; ++q)
                    {
                        const int4 t = tab[kb * BK + kc * 8 + e + q];
                        const int iy = iy0 + t.y, ix = ix0 + t.z;
                        uint32_t v = 0;
                        if (row_ok && t.w && iy >= 0 && iy < P.h && ix >= 0 && ix < P.w)
                            v = bf16_bits(float(P.in[rowoff + t.x]));
                        v2[q] = v;
                    }
                    pk[e / 2] = v2[0] | (v2[1] << 16);
                }
                *reinterpret_cast<uint4 *>(a + kc * 128) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
            }
            // B block: contiguous image of this (n tile, k block).
            const uint4 *src = P.wimg + (int64_t(nt) * P.kblocks + kb) * (b_bytes / 16);
            uint4 *dst = reinterpret_cast<uint4 *>(sB[st]);
            for (int i = tid; i < b_bytes / 16; i += blockDim.x) dst[i] = src[i];
            fence_proxy_async_smem();
            __syncthreads();
            if (tid == 0)
            {
                tc_fence_after();
                const uint32_t a_base = smem_u32(sA[st]), b_base = smem_u32(sB[st]);
                for (int p = 0; p < P.nsplit; ++p)
#pragma unroll
                    for (int s = 0; s < BK / 16; ++s)
                    {
                        const uint64_t ad = smem_desc(a_base + s * 256, 128, 1024);
                        const uint64_t bd = smem_desc(b_base + p * P.n_tile * 128 + s * 256, 128, 1024);
                        mma_bf16(tmem + uint32_t(p * P.n_tile), ad, bd, P.idesc, (kb > 0 || s > 0) ? 1u : 0u);
                    }
                mma_commit(&mbar[st]);
            }
            ++uses[st];
        }
        if (failed) break;

        // Epilogue: all MMAs of the tile are complete once the last commit is.
        const int last = (it - 1) & 1;
        {
            const bool ok = wait_bounded(&mbar[last], (uses[last] - 1) & 1);
            if (__syncthreads_or(!ok))
            {
                failed = true;
                break;
            }
            waited[0] = uses[0], waited[1] = uses[1];
        }
        tc_fence_after();
        const uint32_t lane_base = tmem + (uint32_t(warp * 32) << 16);
        for (int c0 = 0; c0 < P.n_tile; c0 += 16)
        {
            uint32_t r0[16], r1[16], r2[16];
            tmem_ld16(lane_base + uint32_t(c0), r0);
            tmem_ld16(lane_base + uint32_t(P.n_tile + c0), r1);
            if (P.nsplit == 3) tmem_ld16(lane_base + uint32_t(2 * P.n_tile + c0), r2);
            tmem_ld_wait();
            if (row_ok)
            {
#pragma unroll
                for (int j = 0; j < 16; ++j)
                {
                    const int n = nt * P.n_tile + c0 + j;
                    if (n < P.cout)
                    {
                        double acc = double(__uint_as_float(r0[j])) + double(__uint_as_float(r1[j]));
                        if (P.nsplit == 3) acc += double(__uint_as_float(r2[j]));
                        P.out[(img * P.cout + n) * P.ohw + pix] = float(acc);
                    }
                }
            }
        }
        tc_fence_before();
        __syncthreads();
    }

    // Teardown: make sure no MMA is still writing tensor memory, then free it.
    if (!failed)
        for (int st = 0; st < 2; ++st)
            if (waited[st] < uses[st]) wait_bounded(&mbar[st], (uses[st] - 1) & 1);
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
    {
        tc_fence_after();
        tmem_dealloc(tmem, P.tmem_cols);
    }
}

struct Plan
{
    int nsplit, n_tile, n_tiles, K, kblocks;
    uint32_t tmem_cols;
    size_t wimg_bytes, smem;
};

Plan make_plan(int64_t cin, int64_t cout, int64_t kh, int64_t kw, int precision)
{
    Plan pl{};
    pl.nsplit = precision == SPK_CONV_BF16X3 ? 3 : 2;
    const int64_t npad = ceil_div(cout, 16) * 16;
    const int64_t cap = pl.nsplit == 3 ? 128 : 256;
    pl.n_tiles = int(ceil_div(npad, cap));
    pl.n_tile = int(ceil_div(ceil_div(npad, pl.n_tiles), 16) * 16);
    pl.K = int(cin * kh * kw);
    pl.kblocks = int(ceil_div(pl.K, BK));
    uint32_t need = uint32_t(pl.nsplit * pl.n_tile), cols = 32;
    while (cols < need) cols <<= 1;
    pl.tmem_cols = cols;
    pl.wimg_bytes = size_t(pl.n_tiles) * pl.kblocks * pl.nsplit * pl.n_tile * BK * 2;
    size_t smem = 2 * size_t(BM * BK * 2) + 2 * size_t(pl.nsplit) * pl.n_tile * BK * 2 + size_t(pl.kblocks) * BK * 16;
    // At most 512 / tmem_cols CTAs may share an SM's tensor memory: size the
    // shared memory so that no more fit.
    const int per_sm = int(512 / cols);
    const size_t floor_smem = (228 * 1024) / size_t(per_sm + 1) + 1024;
    pl.smem = std::max(smem, floor_smem) + 1024;
    return pl;
}
}  // namespace

size_t conv_tc_workspace(int64_t, int64_t cin, int64_t, int64_t, int64_t cout, int64_t kh, int64_t kw, int precision)
{
    Plan pl = make_plan(cin, cout, kh, kw, precision);
    return pl.wimg_bytes + 256;
}

void conv_tc(const void *in, spk_dtype itype, const float *kernel, float *out, int64_t n, int64_t cin, int64_t h,
             int64_t w, int64_t cout, int64_t kh, int64_t kw, int64_t sy, int64_t sx, Pad4 p, int64_t oh, int64_t ow,
             int precision, void *ws, size_t ws_bytes, cudaStream_t s)
{
    if (itype != SPK_U8) throw Error(SPK_ERR_UNSUPPORTED, "the tensor-core path takes U8 spikes");
    Plan pl = make_plan(cin, cout, kh, kw, precision);
    SPK_REQUIRE(pl.K <= kMaxK, "Cin*KH*KW is limited to 4096 on the tensor-core path");
    SPK_REQUIRE(pl.smem <= 227 * 1024, "tile does not fit in shared memory");
    SPK_REQUIRE(ws != nullptr && ws_bytes >= pl.wimg_bytes, "workspace is too small");
    SPK_REQUIRE((reinterpret_cast<uintptr_t>(ws) & 15) == 0, "workspace must be 16-byte aligned");
    uint4 *wimg = reinterpret_cast<uint4 *>(ws);
    const int64_t wthreads = int64_t(pl.n_tiles) * pl.kblocks * pl.n_tile * 8;
    split_weights_kernel<<<grid_for(wthreads, 256), 256, 0, s>>>(kernel, wimg, int(cout), pl.K, pl.kblocks, pl.n_tile,
                                                                pl.n_tiles, pl.nsplit);
    SPK_LAUNCHED();

    TcParams P{};
    P.in = static_cast<const uint8_t *>(in);
    P.wimg = wimg;
    P.out = out;
    P.M = n * oh * ow;
    P.tiles = ceil_div(P.M, BM) * pl.n_tiles;
    P.chw = cin * h * w;
    P.ohw = oh * ow;
    P.cin = int(cin), P.h = int(h), P.w = int(w), P.cout = int(cout), P.kh = int(kh), P.kw = int(kw);
    P.oh = int(oh), P.ow = int(ow), P.sy = int(sy), P.sx = int(sx), P.top = int(p.top), P.left = int(p.left);
    P.K = pl.K, P.kblocks = pl.kblocks, P.n_tile = pl.n_tile, P.n_tiles = pl.n_tiles, P.nsplit = pl.nsplit;
    P.tmem_cols = pl.tmem_cols;
    P.idesc = idesc_bf16_f32(BM, pl.n_tile);
    SPK_CUDA(cudaFuncSetAttribute(conv_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(pl.smem)));
    const int64_t grid = std::min<int64_t>(P.tiles, int64_t(sm_count()));
    conv_tc_kernel<<<unsigned(grid), kTcThreads, pl.smem, s>>>(P);
    SPK_LAUNCHED();
}
}  // namespace spk

extern "C" int spk_device_status(int reset)
{
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, spk::g_tc_status, sizeof(int)) != cudaSuccess) return -1;
    if (reset)
    {
        int z = 0;
        if (cudaMemcpyToSymbol(spk::g_tc_status, &z, sizeof(int)) != cudaSuccess) return -1;
    }
    return v;
}
