// Device-wide exclusive prefix sum into int64 (three passes: per-block sums,
// a scan of the block sums (recursively), per-block rescans with offsets).
#pragma once

#include "common.cuh"

namespace spk
{
constexpr int kScanBlock = 512, kScanItems = 8, kScanTile = kScanBlock * kScanItems;

// Bytes of scratch scan_exclusive needs for n values.
inline size_t scan_workspace(int64_t n)
{
    size_t bytes = 0;
    while (n > kScanTile)
    {
        n = (n + kScanTile - 1) / kScanTile;
        bytes += ((size_t(n + 1) * 8 + 255) / 256) * 256;
    }
    return bytes;
}

namespace scan_detail
{
// Block-wide exclusive scan of one value per thread; returns the block total.
__device__ __forceinline__ int64_t block_exclusive(int64_t &v)
{
    __shared__ int64_t warp_sum[kScanBlock / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[warp] = x;
    __syncthreads();
    if (warp == 0)
    {
        int64_t s = lane < kScanBlock / 32 ? warp_sum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            const int64_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < kScanBlock / 32) warp_sum[lane] = s;
    }
    __syncthreads();
    const int64_t before = (warp > 0 ? warp_sum[warp - 1] : 0) + x - v;
    const int64_t total = warp_sum[kScanBlock / 32 - 1];
    __syncthreads();
    v = before;
    return total;
}

template <typename I>
__global__ void __launch_bounds__(kScanBlock) tile_sums(const I *__restrict__ in, int64_t n, int64_t *__restrict__ sums)
{
    const int64_t base = int64_t(blockIdx.x) * kScanTile + int64_t(threadIdx.x) * kScanItems;
    int64_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i)
        if (base + i < n) s += int64_t(in[base + i]);
    const int64_t total = block_exclusive(s);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// out[i] = offset[tile] + exclusive prefix within the tile; out[n] = total
// when this is the last tile.  `in` may alias `out`: a block reads its own
// tile before the barrier of the block scan and writes it after.
template <typename I>
__global__ void __launch_bounds__(kScanBlock) tile_scan(const I *in, int64_t n, const int64_t *offsets, int64_t *out)
{
    const int64_t base = int64_t(blockIdx.x) * kScanTile + int64_t(threadIdx.x) * kScanItems;
    int64_t v[kScanItems], s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i)
    {
        v[i] = (base + i < n) ? int64_t(in[base + i]) : 0;
        s += v[i];
    }
    const int64_t total = block_exclusive(s);
    int64_t run = s + (offsets ? offsets[blockIdx.x] : 0);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i)
    {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
    if (threadIdx.x == 0 && blockIdx.x == gridDim.x - 1) out[n] = (offsets ? offsets[blockIdx.x] : 0) + total;
}
}  // namespace scan_detail

// out[0..n] (n + 1 entries): out[i] = in[0] + ... + in[i-1].  `ws` holds
// scan_workspace(n) bytes (256-byte aligned).
template <typename I>
void scan_exclusive(const I *in, int64_t *out, int64_t n, void *ws, cudaStream_t s)
{
    if (n <= 0)
    {
        SPK_CUDA(cudaMemsetAsync(out, 0, sizeof(int64_t), s));
        return;
    }
    const int64_t tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles == 1)
    {
        scan_detail::tile_scan<I><<<1, kScanBlock, 0, s>>>(in, n, nullptr, out);
        SPK_LAUNCHED();
        return;
    }
    int64_t *sums = static_cast<int64_t *>(ws);
    int64_t *offs = sums;  // scanned in place into tiles + 1 entries
    void *rest = static_cast<char *>(ws) + ((size_t(tiles + 1) * 8 + 255) / 256) * 256;
    scan_detail::tile_sums<I><<<unsigned(tiles), kScanBlock, 0, s>>>(in, n, sums);
    SPK_LAUNCHED();
    // Scan the tile sums (in place is safe: each level reads its input fully
    // in the sums pass before the rescan pass writes).
    int64_t *tmp = sums;
    scan_exclusive<int64_t>(sums, tmp, tiles, rest, s);
    scan_detail::tile_scan<I><<<unsigned(tiles), kScanBlock, 0, s>>>(in, n, offs, out);
    SPK_LAUNCHED();
}
}  // namespace spk
