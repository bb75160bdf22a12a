// Event-list ("sparse") spiking path: src/spyker/sparse/*.cpp on the GPU.
//
// A sparse spike tensor [U, T, C, H, W] is a list of events per (sample u,
// step t); each event is a position (z, y, x) with u8 coordinates
// (src/spyker/base.h:493-528).  On the device the lists are one CSR array:
//   offsets int64 [U*T + 1], list i = u*T + t = events offsets[i] .. offsets[i+1]-1,
//   events  uint32, x | y << 8 | z << 16 (so ascending values are (z, y, x) order).
// The order of events inside a list is part of the semantics (inhibition,
// WTA and conv read them in order) and every kernel here reproduces the
// reference's order.  Outputs are written into caller buffers sized by the
// worst case, so nothing waits for the host.
//
// Building blocks: first-spike times -> lists (code, from-dense); per-cell
// "first event" filters through atomicMin over event indices plus a stable
// compaction (inhibit, pool); a warp per (sample, output map) for the
// incremental conv+fire; a warp per sample for the sequential WTA; STDP over
// the ordered per-map scan shared with the dense path.
#include "common.cuh"
#include "scan.cuh"

namespace spk
{
void rank_times(const void *in, spk_dtype itype, uint16_t *times, int64_t b, int64_t t, int64_t x, int sort, void *ws,
                cudaStream_t s);
size_t rank_times_ws(int64_t b, int64_t x, int sort);
void launch_stdp_scan(float *kernel, int64_t k, int64_t nmaps, int64_t b, int64_t count, int field,
                      const int32_t *winners, const int32_t *counts, const uint16_t *pre, int64_t ps, int64_t pw,
                      const uint16_t *post, const double *configs, int64_t nconf, bool f32_rule, cudaStream_t s);

namespace
{
constexpr int kListWarps = 8;          // warps per CTA of the warp-per-list kernels
constexpr int64_t kMaxSparseT = 16384; // steps per sample on this path
constexpr int kNone = 0x7f7f7f7f;      // "no event" of the atomicMin maps (memset 0x7f)

__device__ __forceinline__ uint32_t ev_pack(int z, int y, int x)
{
    return uint32_t(x & 255) | (uint32_t(y & 255) << 8) | (uint32_t(z & 255) << 16);
}
__device__ __forceinline__ int ev_z(uint32_t e) { return int(e >> 16) & 255; }
__device__ __forceinline__ int ev_y(uint32_t e) { return int(e >> 8) & 255; }
__device__ __forceinline__ int ev_x(uint32_t e) { return int(e) & 255; }

inline size_t al(size_t v) { return (v + 255) & ~size_t(255); }

// Carves consecutive 256-byte aligned pieces out of a workspace.
struct Carve
{
    char *p;
    size_t used = 0;
    template <typename T>
    T *take(size_t count)
    {
        T *r = reinterpret_cast<T *>(p + used);
        used += al(count * sizeof(T));
        return r;
    }
};

unsigned list_grid(int64_t lists) { return unsigned(std::max<int64_t>(1, ceil_div(lists, kListWarps))); }

// ---------------------------------------------------------------------------
// first-spike times -> event lists (sparse/code.cpp:52-61, sparse/opers.cpp:59-69)
// ---------------------------------------------------------------------------

// counts[u*T + t] = number of positions of sample u with time t (< T).
__global__ void times_count_kernel(const uint16_t *__restrict__ tm, int64_t x, int t, int32_t *__restrict__ counts)
{
    extern __shared__ int32_t hist[];
    for (int i = threadIdx.x; i < t; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    const uint16_t *row = tm + int64_t(blockIdx.x) * x;
    for (int64_t j = threadIdx.x; j < x; j += blockDim.x)
    {
        const int v = row[j];
        if (v < t) atomicAdd(&hist[v], 1);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < t; i += blockDim.x) counts[int64_t(blockIdx.x) * t + i] = hist[i];
}

// Events in position order inside each (sample, time) list.  Warp w of the
// CTA owns a contiguous segment of positions; pass 1 counts its times, the
// per-time prefix over warps gives each warp its cursors, pass 2 places the
// events with __match_any_sync ranks (stable within a 32-chunk).
__global__ void times_scatter_kernel(const uint16_t *__restrict__ tm, int64_t x, int t, int h, int w,
                                     const int64_t *__restrict__ offsets, uint32_t *__restrict__ events)
{
    extern __shared__ int32_t cur[];  // [warps][t]
    const int warps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t u = blockIdx.x;
    const uint16_t *row = tm + u * x;
    const int64_t seg = ceil_div(ceil_div(x, warps), 32) * 32;
    const int64_t lo = std::min<int64_t>(x, warp * seg), hi = std::min<int64_t>(x, lo + seg);
    for (int i = threadIdx.x; i < warps * t; i += blockDim.x) cur[i] = 0;
    __syncthreads();
    for (int64_t j = lo + lane; j < hi; j += 32)
    {
        const int v = row[j];
        if (v < t) atomicAdd(&cur[warp * t + v], 1);
    }
    __syncthreads();
    for (int v = threadIdx.x; v < t; v += blockDim.x)
    {
        int64_t run = offsets[u * t + v];
        for (int q = 0; q < warps; ++q)
        {
            const int c = cur[q * t + v];
            cur[q * t + v] = int32_t(run - offsets[u * t + v]);  // cursor relative to the list start
            run += c;
        }
    }
    __syncthreads();
    const int hw = h * w;
    for (int64_t j0 = lo; j0 < hi; j0 += 32)
    {
        const int64_t j = j0 + lane;
        const int v = (j < hi) ? int(row[j]) : t;
        const unsigned peers = __match_any_sync(0xffffffffu, v);
        const int rank = __popc(peers & ((1u << lane) - 1u));
        int base = 0;
        if (v < t) base = cur[warp * t + v];
        __syncwarp();
        if (v < t)
        {
            const int z = int(j / hw), r = int(j - int64_t(z) * hw), y = r / w, xx = r - y * w;
            events[offsets[u * t + v] + base + rank] = ev_pack(z, y, xx);
            if (rank == 0) cur[warp * t + v] = base + __popc(peers);
        }
        __syncwarp();
    }
}

void times_to_lists(const uint16_t *tm, int64_t u, int64_t t, int64_t c, int64_t h, int64_t w, int64_t *offsets,
                    uint32_t *events, Carve &ws, cudaStream_t s)
{
    const int64_t x = c * h * w;
    int32_t *counts = ws.take<int32_t>(size_t(u * t));
    void *scan_ws = ws.take<char>(scan_workspace(u * t));
    const size_t hist = size_t(t) * 4;
    if (hist > 48 * 1024)
        SPK_CUDA(cudaFuncSetAttribute(times_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(hist)));
    times_count_kernel<<<unsigned(u), 256, hist, s>>>(tm, x, int(t), counts);
    SPK_LAUNCHED();
    scan_exclusive<int32_t>(counts, offsets, u * t, scan_ws, s);
    const int warps = int(std::max<int64_t>(1, std::min<int64_t>(8, 8192 / t)));
    const size_t cur = size_t(warps) * t * 4;
    if (cur > 48 * 1024)
        SPK_CUDA(cudaFuncSetAttribute(times_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(cur)));
    times_scatter_kernel<<<unsigned(u), warps * 32, cur, s>>>(tm, x, int(t), int(h), int(w), offsets, events);
    SPK_LAUNCHED();
}

size_t times_to_lists_ws(int64_t u, int64_t t) { return al(size_t(u * t) * 4) + al(scan_workspace(u * t)); }

// first t with in > threshold (T when none), sparse/opers.cpp:59-69
template <typename T>
__global__ void threshold_times_kernel(const T *__restrict__ in, uint16_t *__restrict__ tm, int64_t u, int t,
                                       int64_t x, T thr)
{
    const int64_t total = u * x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t s = k / x, j = k - s * x;
        const T *p = in + s * t * x + j;
        int v = t;
        for (int q = 0; q < t; ++q)
            if (p[int64_t(q) * x] > thr)
            {
                v = q;
                break;
            }
        tm[k] = uint16_t(v);
    }
}

// ---------------------------------------------------------------------------
// lists -> dense (sparse/opers.cpp:88-118)
// ---------------------------------------------------------------------------

// map[u, z, y, x] = min over events of t (kNone when silent); events outside
// the shape are skipped.
__global__ void min_time_map_kernel(const int64_t *__restrict__ offsets, const uint32_t *__restrict__ events,
                                    int64_t lists, int t, int c, int h, int w, int32_t *__restrict__ map)
{
    const int64_t list = int64_t(blockIdx.x) * kListWarps + (threadIdx.x >> 5);
    if (list >= lists) return;
    const int lane = threadIdx.x & 31;
    const int64_t u = list / t;
    const int step = int(list - u * t);
    for (int64_t k = offsets[list] + lane; k < offsets[list + 1]; k += 32)
    {
        const uint32_t e = events[k];
        const int z = ev_z(e), y = ev_y(e), x = ev_x(e);
        if (z < c && y < h && x < w) atomicMin(&map[((u * c + z) * h + y) * int64_t(w) + x], step);
    }
}

template <typename O>
__global__ void map_to_gather_kernel(const int32_t *__restrict__ map, O *__restrict__ out, int64_t n, int t)
{
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += int64_t(gridDim.x) * blockDim.x)
    {
        const int v = map[k];
        out[k] = O(v == kNone ? t : v);
    }
}

template <typename O>
__global__ void map_to_dense_kernel(const int32_t *__restrict__ map, O *__restrict__ out, int64_t u, int t, int64_t x)
{
    const int64_t total = u * t * x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < total; k += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t s = k / (int64_t(t) * x), r = k - s * t * x, q = r / x, j = r - q * x;
        out[k] = O(map[s * x + j] <= q ? 1 : 0);
    }
}

// ---------------------------------------------------------------------------
// stable filters (sparse/inhibit.cpp:37-65, sparse/pool.cpp:37-64)
// ---------------------------------------------------------------------------

// Cell of an event for the filter; -1 when the event is dropped outright.
struct InhibitCell
{
    int h, w;
    __device__ int64_t cell(uint32_t e) const
    {
        const int y = ev_y(e), x = ev_x(e);
        return (y < h && x < w) ? int64_t(y) * w + x : -1;
    }
    __device__ int64_t cells() const { return int64_t(h) * w; }
};

struct PoolCell
{
    int c, oh, ow, ky, kx, top, left;
    __device__ int oy(uint32_t e) const { return ((top + ev_y(e)) / ky) & 255; }  // uint8_t((p + y) / k)
    __device__ int ox(uint32_t e) const { return ((left + ev_x(e)) / kx) & 255; }
    __device__ int64_t cell(uint32_t e) const
    {
        const int y = oy(e), x = ox(e), z = ev_z(e);
        return (y < oh && x < ow && z < c) ? (int64_t(z) * oh + y) * ow + x : -1;
    }
    __device__ int64_t cells() const { return int64_t(c) * oh * ow; }
};

// Event loops stop at `cap`, the input's capacity, whatever its offsets say.
template <typename Cell>
__global__ void first_event_kernel(const int64_t *__restrict__ offsets, const uint32_t *__restrict__ events,
                                   int64_t lists, int64_t cap, int t, Cell cell, int32_t *__restrict__ first)
{
    const int64_t list = int64_t(blockIdx.x) * kListWarps + (threadIdx.x >> 5);
    if (list >= lists) return;
    const int lane = threadIdx.x & 31;
    const int64_t u = list / t;
    const int64_t end = min(offsets[list + 1], cap);
    for (int64_t k = offsets[list] + lane; k < end; k += 32)
    {
        const int64_t q = cell.cell(events[k]);
        if (q >= 0) atomicMin(&first[u * cell.cells() + q], int32_t(k));
    }
}

// keep[k]: inhibition keeps the events of the channel of the pixel's first
// event; pooling keeps the first event of each pooled cell.
template <bool POOL, typename Cell>
__global__ void keep_kernel(const int64_t *__restrict__ offsets, const uint32_t *__restrict__ events, int64_t lists,
                            int64_t cap, int t, Cell cell, const int32_t *__restrict__ first,
                            int32_t *__restrict__ keep)
{
    const int64_t list = int64_t(blockIdx.x) * kListWarps + (threadIdx.x >> 5);
    if (list >= lists) return;
    const int lane = threadIdx.x & 31;
    const int64_t u = list / t;
    const int64_t end = min(offsets[list + 1], cap);
    for (int64_t k = offsets[list] + lane; k < end; k += 32)
    {
        const uint32_t e = events[k];
        const int64_t q = cell.cell(e);
        int32_t kept = 0;
        if (q >= 0)
        {
            const int32_t f = first[u * cell.cells() + q];
            kept = POOL ? (f == int32_t(k)) : (ev_z(events[f]) == ev_z(e));
        }
        keep[k] = kept;
    }
}

template <bool POOL, typename Cell>
__global__ void compact_kernel(const int64_t *__restrict__ offsets, const uint32_t *__restrict__ events, int64_t lists,
                               int64_t cap, Cell cell, const int32_t *__restrict__ keep,
                               const int64_t *__restrict__ pos, uint32_t *__restrict__ out)
{
    const int64_t list = int64_t(blockIdx.x) * kListWarps + (threadIdx.x >> 5);
    if (list >= lists) return;
    const int lane = threadIdx.x & 31;
    const int64_t end = min(offsets[list + 1], cap);
    for (int64_t k = offsets[list] + lane; k < end; k += 32)
        if (keep[k])
        {
            const uint32_t e = events[k];
            if constexpr (POOL)
                out[pos[k]] = ev_pack(ev_z(e), cell.oy(e), cell.ox(e));
            else
                out[pos[k]] = e;
        }
}

__global__ void remap_offsets_kernel(const int64_t *__restrict__ offsets, int64_t lists, int64_t cap,
                                     const int64_t *__restrict__ pos, int64_t *__restrict__ out)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i <= lists; i += int64_t(gridDim.x) * blockDim.x)
        out[i] = pos[min(offsets[i], cap)];
}

template <bool POOL, typename Cell>
void filter_lists(const int64_t *offsets, const uint32_t *events, int64_t in_cap, int64_t u, int64_t t, Cell cell,
                  int64_t ncells, int64_t *out_offsets, uint32_t *out_events, Carve &ws, cudaStream_t s)
{
    const int64_t lists = u * t;
    int32_t *first = ws.take<int32_t>(size_t(u * ncells));
    int32_t *keep = ws.take<int32_t>(size_t(in_cap));
    int64_t *pos = ws.take<int64_t>(size_t(in_cap + 1));
    void *scan_ws = ws.take<char>(scan_workspace(in_cap));
    SPK_CUDA(cudaMemsetAsync(first, 0x7f, size_t(u * ncells) * 4, s));
    SPK_CUDA(cudaMemsetAsync(keep, 0, size_t(in_cap) * 4, s));
    first_event_kernel<Cell><<<list_grid(lists), kListWarps * 32, 0, s>>>(offsets, events, lists, in_cap, int(t), cell,
                                                                           first);
    SPK_LAUNCHED();
    keep_kernel<POOL, Cell><<<list_grid(lists), kListWarps * 32, 0, s>>>(offsets, events, lists, in_cap, int(t), cell,
                                                                        first, keep);
    SPK_LAUNCHED();
    scan_exclusive<int32_t>(keep, pos, in_cap, scan_ws, s);
    compact_kernel<POOL, Cell><<<list_grid(lists), kListWarps * 32, 0, s>>>(offsets, events, lists, in_cap, cell, keep,
                                                                           pos, out_events);
    SPK_LAUNCHED();
    remap_offsets_kernel<<<grid_for(lists + 1, 256), 256, 0, s>>>(offsets, lists, in_cap, pos, out_offsets);
    SPK_LAUNCHED();
}

size_t filter_ws(int64_t u, int64_t ncells, int64_t in_cap)
{
    return al(size_t(u * ncells) * 4) + al(size_t(in_cap) * 4) + al(size_t(in_cap + 1) * 8) +
           al(scan_workspace(in_cap));
}

// ---------------------------------------------------------------------------
// incremental conv + fire (sparse/conv.cpp:42-130)
// ---------------------------------------------------------------------------

// One warp per (sample, output map).  The map's F32 potential plane (shared
// memory, or global scratch when it is large) receives, event after event in
// list order, the kernel tap of every neuron the event reaches: lanes own
// taps, and the taps of one event reach distinct neurons, so every neuron
// sees its additions in the reference's order.  After each step whose input
// list is non-empty, neurons above threshold fire once (listed in (y, x)
// order) and are parked at -FLT_MAX.  Fired neurons go to the map's slot of
// `fired` in firing order, with per-(sample, step, map) counts.
template <bool SMEM>
__global__ void sparse_conv_kernel(const int64_t *__restrict__ offsets, const uint32_t *__restrict__ events, int64_t u,
                                   int t, int c, const float *__restrict__ kernel, int cout, int kh, int kw, int top,
                                   int left, int oh, int ow, float thr, uint16_t *__restrict__ fired,
                                   int32_t *__restrict__ counts, float *__restrict__ planes)
{
    extern __shared__ float splanes[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t gw = int64_t(blockIdx.x) * (blockDim.x >> 5) + warp;
    if (gw >= u * cout) return;
    const int64_t s = gw / cout;
    const int q = int(gw - s * cout);
    const int ohw = oh * ow, taps = kh * kw;
    float *pot = SMEM ? splanes + int64_t(warp) * ohw : planes + gw * ohw;
    for (int i = lane; i < ohw; i += 32) pot[i] = 0.f;
    __syncwarp();
    const float *kq = kernel + int64_t(q) * c * taps;
    uint16_t *slot = fired + gw * ohw;
    int done = 0;
    for (int step = 0; step < t; ++step)
    {
        const int64_t b = offsets[s * t + step], e = offsets[s * t + step + 1];
        for (int64_t k = b; k < e; ++k)
        {
            const uint32_t ev = events[k];
            const int z = ev_z(ev), yy = ev_y(ev) + top, xx = ev_x(ev) + left;
            if (z < c)
                for (int tap = lane; tap < taps; tap += 32)
                {
                    const int ky = tap / kw, kx = tap - ky * kw;
                    const int y = yy - ky, x = xx - kx;
                    if (y >= 0 && y < oh && x >= 0 && x < ow) pot[y * ow + x] += kq[z * taps + tap];
                }
            __syncwarp();
        }
        int nf = 0;
        if (e > b)
        {
            for (int i0 = 0; i0 < ohw; i0 += 32)
            {
                const int i = i0 + lane;
                const bool f = i < ohw && pot[i] > thr;
                const unsigned m = __ballot_sync(0xffffffffu, f);
                const int at = done + nf + __popc(m & ((1u << lane) - 1u));
                if (f)
                {
                    if (at < ohw) slot[at] = uint16_t(i);
                    pot[i] = -FLT_MAX;
                }
                nf += __popc(m);
            }
            // A parked neuron fires again only if additions of about FLT_MAX
            // lift it back over the threshold; the slot holds OH*OW neurons
            // and any such extra events are dropped.
            nf = min(nf, ohw - done);
            __syncwarp();
        }
        if (lane == 0) counts[(s * t + step) * cout + q] = nf;
        done += nf;
    }
}

// Output lists: per (sample, step) the fired neurons map after map.
__global__ void conv_lists_kernel(const uint16_t *__restrict__ fired, const int32_t *__restrict__ counts,
                                  const int64_t *__restrict__ starts, int64_t u, int t, int cout, int ow, int ohw,
                                  uint32_t *__restrict__ out)
{
    const int64_t gw = int64_t(blockIdx.x) * kListWarps + (threadIdx.x >> 5);
    if (gw >= u * cout) return;
    const int lane = threadIdx.x & 31;
    const int64_t s = gw / cout;
    const int q = int(gw - s * cout);
    const uint16_t *slot = fired + gw * ohw;
    int done = 0;
    for (int step = 0; step < t; ++step)
    {
        const int64_t i = (s * t + step) * cout + q;
        const int n = counts[i];
        const int64_t dst = starts[i];
        for (int j = lane; j < n; j += 32)
        {
            const int p = slot[done + j], y = p / ow, x = p - y * ow;
            out[dst + j] = ev_pack(q, y, x);
        }
        done += n;
    }
}

__global__ void conv_offsets_kernel(const int64_t *__restrict__ starts, int64_t lists, int cout,
                                    int64_t *__restrict__ out)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i <= lists; i += int64_t(gridDim.x) * blockDim.x)
        out[i] = starts[i * cout];
}

// ---------------------------------------------------------------------------
// WTA (sparse/wta.cpp:44-95)
// ---------------------------------------------------------------------------

// One warp per sample, events in (step, list) order, 32 at a time: lanes test
// their event against the accepted boxes, then candidates are accepted from
// the lowest lane up, each acceptance re-testing the lanes after it.
__global__ void sparse_wta_kernel(const int64_t *__restrict__ offsets, const uint32_t *__restrict__ events, int64_t u,
                                  int t, int h, int w, int ry, int rx, int count, int32_t *__restrict__ winners,
                                  int32_t *__restrict__ counts)
{
    extern __shared__ int32_t boxes[];  // per warp: count x (z, ys, ye, xs, xe)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t s = int64_t(blockIdx.x) * (blockDim.x >> 5) + warp;
    if (s >= u) return;
    int32_t *bx = boxes + int64_t(warp) * count * 5;
    int n = 0;
    for (int step = 0; step < t && n < count; ++step)
    {
        const int64_t b = offsets[s * t + step], e = offsets[s * t + step + 1];
        for (int64_t k0 = b; k0 < e && n < count; k0 += 32)
        {
            const int64_t k = k0 + lane;
            const bool valid = k < e;
            const uint32_t ev = valid ? events[k] : 0u;
            const int z = ev_z(ev), y = ev_y(ev), x = ev_x(ev);
            bool ok = valid;
            for (int j = 0; j < n && ok; ++j)
            {
                const int32_t *q = bx + j * 5;
                if (z == q[0] || (y >= q[1] && y <= q[2] && x >= q[3] && x <= q[4])) ok = false;
            }
            unsigned cand = __ballot_sync(0xffffffffu, ok);
            while (cand && n < count)
            {
                const int l = __ffs(cand) - 1;
                const int zl = __shfl_sync(0xffffffffu, z, l), yl = __shfl_sync(0xffffffffu, y, l),
                          xl = __shfl_sync(0xffffffffu, x, l);
                if (lane == 0)
                {
                    int32_t *o = winners + (s * count + n) * 5;
                    o[0] = 0, o[1] = step, o[2] = zl, o[3] = yl, o[4] = xl;
                    int32_t *q = bx + n * 5;
                    q[0] = zl, q[1] = max(0, yl - ry), q[2] = min(h - 1, yl + ry), q[3] = max(0, xl - rx),
                    q[4] = min(w - 1, xl + rx);
                }
                ++n;
                __syncwarp();
                const bool hit = ok && lane > l &&
                                 (z == zl || (y >= max(0, yl - ry) && y <= min(h - 1, yl + ry) &&
                                              x >= max(0, xl - rx) && x <= min(w - 1, xl + rx)));
                ok = ok && lane > l && !hit;
                cand = __ballot_sync(0xffffffffu, ok);
            }
        }
    }
    if (lane == 0) counts[s] = n;
}

// ---------------------------------------------------------------------------
// STDP (sparse/stdp.cpp:41-133)
// ---------------------------------------------------------------------------

// last[u, z, yp, xp] = 1 + latest step of an event at padded position
// (y + top, x + left) (0 when none): the reference marks a window element
// with the time of the last event written there in (step, list) order.
__global__ void last_time_map_kernel(const int64_t *__restrict__ offsets, const uint32_t *__restrict__ events,
                                     int64_t lists, int t, int c, int hp, int wp, int top, int left,
                                     int32_t *__restrict__ last)
{
    const int64_t list = int64_t(blockIdx.x) * kListWarps + (threadIdx.x >> 5);
    if (list >= lists) return;
    const int lane = threadIdx.x & 31;
    const int64_t u = list / t;
    const int step = int(list - u * t);
    for (int64_t k = offsets[list] + lane; k < offsets[list + 1]; k += 32)
    {
        const uint32_t e = events[k];
        const int z = ev_z(e), y = ev_y(e) + top, x = ev_x(e) + left;
        if (z < c && y < hp && x < wp) atomicMax(&last[((u * c + z) * hp + y) * int64_t(wp) + x], step + 1);
    }
}

// pre[s, j, (z, ky, kx)] = time at window position (T when none);
// post[s, j] = the winner's step.  One CTA per (sample, winner slot).
__global__ void sparse_prepost_kernel(const int32_t *__restrict__ last, int t, int c, int hp, int wp, int kh, int kw,
                                      const int32_t *__restrict__ winners, const int32_t *__restrict__ counts,
                                      int count, uint16_t *__restrict__ pre, uint16_t *__restrict__ post)
{
    const int64_t s = blockIdx.x / count;
    const int j = int(blockIdx.x % count);
    if (j >= counts[s]) return;
    const int32_t *e = winners + (s * count + j) * 5;
    const int wy = e[3], wx = e[4];
    const int k = c * kh * kw;
    uint16_t *p = pre + (s * count + j) * int64_t(k);
    for (int i = threadIdx.x; i < k; i += blockDim.x)
    {
        const int z = i / (kh * kw), r = i - z * kh * kw, ky = r / kw, kx = r - ky * kw;
        const int y = wy + ky, x = wx + kx;
        int v = 0;
        if (y >= 0 && y < hp && x >= 0 && x < wp) v = last[((s * c + z) * hp + y) * int64_t(wp) + x];
        p[i] = uint16_t(v == 0 ? t : v - 1);
    }
    if (threadIdx.x == 0) post[s * count + j] = uint16_t(e[1] < 0 ? 0 : (e[1] > 65535 ? 65535 : e[1]));
}

void check_shape(int64_t u, int64_t t, int64_t c, int64_t h, int64_t w)
{
    SPK_REQUIRE(u >= 0 && t >= 1 && c >= 1 && h >= 1 && w >= 1, "invalid dims");
    SPK_REQUIRE(t <= kMaxSparseT, "event lists support at most 16384 steps");
    SPK_REQUIRE(c <= 256 && h <= 256 && w <= 256, "event coordinates are 8-bit: C, H and W must be at most 256");
}
}  // namespace
}  // namespace spk

using namespace spk;

extern "C" {

size_t spk_sparse_code_workspace(int64_t u, int64_t t, int64_t c, int64_t h, int64_t w)
{
    return al(size_t(u * c * h * w) * 2) + times_to_lists_ws(u, t) + al(rank_times_ws(u, c * h * w, 1));
}

spk_status spk_sparse_code(const void *in, spk_dtype itype, int64_t u, int64_t c, int64_t h, int64_t w, int64_t t,
                           int sort, int64_t *offsets, uint32_t *events, int64_t cap, void *ws, size_t ws_bytes,
                           spk_stream stream)
{
    return guarded([&] {
        check_shape(u, t, c, h, w);
        SPK_REQUIRE(cap >= u * c * h * w, "event capacity must be at least U*C*H*W");
        SPK_REQUIRE(ws && ws_bytes >= spk_sparse_code_workspace(u, t, c, h, w), "workspace is too small");
        cudaStream_t s = stream_of(stream);
        if (u == 0)
        {
            SPK_CUDA(cudaMemsetAsync(offsets, 0, 8, s));
            return;
        }
        Carve cv{static_cast<char *>(ws)};
        uint16_t *tm = cv.take<uint16_t>(size_t(u * c * h * w));
        void *sort_ws = cv.take<char>(rank_times_ws(u, c * h * w, sort));
        rank_times(in, itype, tm, u, t, c * h * w, sort, sort_ws, s);
        times_to_lists(tm, u, t, c, h, w, offsets, events, cv, s);
    });
}

size_t spk_sparse_from_dense_workspace(int64_t u, int64_t t, int64_t c, int64_t h, int64_t w)
{
    return al(size_t(u * c * h * w) * 2) + times_to_lists_ws(u, t);
}

spk_status spk_sparse_from_dense(const void *in, spk_dtype itype, int64_t u, int64_t t, int64_t c, int64_t h,
                                 int64_t w, double threshold, int64_t *offsets, uint32_t *events, int64_t cap,
                                 void *ws, size_t ws_bytes, spk_stream stream)
{
    return guarded([&] {
        check_shape(u, t, c, h, w);
        SPK_REQUIRE(cap >= u * c * h * w, "event capacity must be at least U*C*H*W");
        SPK_REQUIRE(ws && ws_bytes >= spk_sparse_from_dense_workspace(u, t, c, h, w), "workspace is too small");
        cudaStream_t s = stream_of(stream);
        if (u == 0)
        {
            SPK_CUDA(cudaMemsetAsync(offsets, 0, 8, s));
            return;
        }
        Carve cv{static_cast<char *>(ws)};
        const int64_t x = c * h * w;
        uint16_t *tm = cv.take<uint16_t>(size_t(u * x));
        dispatch(itype, [&](auto z) {
            using T = decltype(z);
            threshold_times_kernel<T><<<grid_for(u * x, 256), 256, 0, s>>>((const T *)in, tm, u, int(t), x,
                                                                           scalar_to<T>(threshold));
            SPK_LAUNCHED();
        });
        times_to_lists(tm, u, t, c, h, w, offsets, events, cv, s);
    });
}

size_t spk_sparse_dense_workspace(int64_t u, int64_t c, int64_t h, int64_t w) { return al(size_t(u * c * h * w) * 4); }

static void min_map(const int64_t *offsets, const uint32_t *events, int64_t u, int64_t t, int64_t c, int64_t h,
                    int64_t w, int32_t *map, cudaStream_t s)
{
    SPK_CUDA(cudaMemsetAsync(map, 0x7f, size_t(u * c * h * w) * 4, s));
    min_time_map_kernel<<<list_grid(u * t), kListWarps * 32, 0, s>>>(offsets, events, u * t, int(t), int(c), int(h),
                                                                     int(w), map);
    SPK_LAUNCHED();
}

spk_status spk_sparse_to_dense(const int64_t *offsets, const uint32_t *events, int64_t u, int64_t t, int64_t c,
                               int64_t h, int64_t w, void *out, spk_dtype otype, void *ws, size_t ws_bytes,
                               spk_stream stream)
{
    return guarded([&] {
        check_shape(u, t, c, h, w);
        SPK_REQUIRE(ws && ws_bytes >= spk_sparse_dense_workspace(u, c, h, w), "workspace is too small");
        if (u == 0) return;
        cudaStream_t s = stream_of(stream);
        int32_t *map = static_cast<int32_t *>(ws);
        min_map(offsets, events, u, t, c, h, w, map, s);
        dispatch(otype, [&](auto z) {
            using O = decltype(z);
            map_to_dense_kernel<O><<<grid_for(u * t * c * h * w, 256), 256, 0, s>>>(map, (O *)out, u, int(t),
                                                                                    c * h * w);
            SPK_LAUNCHED();
        });
    });
}

spk_status spk_sparse_gather(const int64_t *offsets, const uint32_t *events, int64_t u, int64_t t, int64_t c,
                             int64_t h, int64_t w, void *out, spk_dtype otype, void *ws, size_t ws_bytes,
                             spk_stream stream)
{
    return guarded([&] {
        check_shape(u, t, c, h, w);
        SPK_REQUIRE(ws && ws_bytes >= spk_sparse_dense_workspace(u, c, h, w), "workspace is too small");
        if (u == 0) return;
        cudaStream_t s = stream_of(stream);
        int32_t *map = static_cast<int32_t *>(ws);
        min_map(offsets, events, u, t, c, h, w, map, s);
        dispatch(otype, [&](auto z) {
            using O = decltype(z);
            map_to_gather_kernel<O><<<grid_for(u * c * h * w, 256), 256, 0, s>>>(map, (O *)out, u * c * h * w, int(t));
            SPK_LAUNCHED();
        });
    });
}

__global__ void pad_events_kernel(const int64_t *__restrict__ offsets, const uint32_t *__restrict__ events,
                                  int64_t lists, int64_t cap, int top, int left, uint32_t *__restrict__ out)
{
    const int64_t n = min(offsets[lists], cap);
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += int64_t(gridDim.x) * blockDim.x)
    {
        const uint32_t e = events[k];
        out[k] = ev_pack(ev_z(e), ev_y(e) + top, ev_x(e) + left);
    }
}

spk_status spk_sparse_pad(const int64_t *offsets, const uint32_t *events, int64_t in_cap, int64_t u, int64_t t,
                          int64_t c, int64_t h, int64_t w, const int64_t *pad4_host, int64_t *out_offsets,
                          uint32_t *out_events, int64_t cap, spk_stream stream)
{
    return guarded([&] {
        check_shape(u, t, c, h, w);
        Pad4 p = pad_of(pad4_host);
        SPK_REQUIRE(cap >= in_cap, "output capacity must be at least the input capacity");
        cudaStream_t s = stream_of(stream);
        SPK_CUDA(cudaMemcpyAsync(out_offsets, offsets, size_t(u * t + 1) * 8, cudaMemcpyDeviceToDevice, s));
        if (in_cap > 0)
        {
            pad_events_kernel<<<grid_for(in_cap, 256), 256, 0, s>>>(offsets, events, u * t, in_cap, int(p.top),
                                                                    int(p.left), out_events);
            SPK_LAUNCHED();
        }
    });
}

size_t spk_sparse_pool_workspace(int64_t u, int64_t c, int64_t oh, int64_t ow, int64_t in_cap)
{
    return filter_ws(u, c * oh * ow, in_cap);
}

spk_status spk_sparse_pool(const int64_t *offsets, const uint32_t *events, int64_t in_cap, int64_t u, int64_t t,
                           int64_t c, int64_t h, int64_t w, const int64_t *kernel2_host, const int64_t *stride2_host,
                           const int64_t *pad4_host, int64_t oh, int64_t ow, int64_t *out_offsets,
                           uint32_t *out_events, int64_t cap, void *ws, size_t ws_bytes, spk_stream stream)
{
    return guarded([&] {
        check_shape(u, t, c, h, w);
        Pad4 p = pad_of(pad4_host);
        SPK_REQUIRE(kernel2_host && stride2_host, "null kernel / stride");
        const int64_t ky = kernel2_host[0], kx = kernel2_host[1];
        if (stride2_host[0] != ky || stride2_host[1] != kx)
            throw Error(SPK_ERR_ARGUMENT, "Stride must be equal to kernel in sparse pool.");
        SPK_REQUIRE(ky >= 1 && kx >= 1, "kernel must be at least 1");
        SPK_REQUIRE(oh == (h + p.top + p.bottom - ky) / ky + 1 && ow == (w + p.left + p.right - kx) / kx + 1 &&
                        oh >= 1 && ow >= 1,
                    "output shape is not compatible");
        SPK_REQUIRE(cap >= std::min(in_cap, u * c * oh * ow), "output capacity is too small");
        SPK_REQUIRE(in_cap < (int64_t(1) << 31), "event lists are limited to 2^31 - 1 events");
        SPK_REQUIRE(ws && ws_bytes >= spk_sparse_pool_workspace(u, c, oh, ow, in_cap), "workspace is too small");
        cudaStream_t s = stream_of(stream);
        Carve cv{static_cast<char *>(ws)};
        PoolCell cell{int(c), int(oh), int(ow), int(ky), int(kx), int(p.top), int(p.left)};
        filter_lists<true>(offsets, events, in_cap, u, t, cell, c * oh * ow, out_offsets, out_events, cv, s);
    });
}

size_t spk_sparse_inhibit_workspace(int64_t u, int64_t h, int64_t w, int64_t in_cap)
{
    return filter_ws(u, h * w, in_cap);
}

spk_status spk_sparse_inhibit(const int64_t *offsets, const uint32_t *events, int64_t in_cap, int64_t u, int64_t t,
                              int64_t c, int64_t h, int64_t w, int64_t *out_offsets, uint32_t *out_events, int64_t cap,
                              void *ws, size_t ws_bytes, spk_stream stream)
{
    return guarded([&] {
        check_shape(u, t, c, h, w);
        SPK_REQUIRE(cap >= in_cap, "output capacity must be at least the input capacity");
        SPK_REQUIRE(in_cap < (int64_t(1) << 31), "event lists are limited to 2^31 - 1 events");
        SPK_REQUIRE(ws && ws_bytes >= spk_sparse_inhibit_workspace(u, h, w, in_cap), "workspace is too small");
        cudaStream_t s = stream_of(stream);
        Carve cv{static_cast<char *>(ws)};
        InhibitCell cell{int(h), int(w)};
        filter_lists<false>(offsets, events, in_cap, u, t, cell, h * w, out_offsets, out_events, cv, s);
    });
}

static void conv_dims(int64_t h, int64_t w, int64_t kh, int64_t kw, const int64_t *stride2, const int64_t *pad4,
                      int64_t &oh, int64_t &ow)
{
    SPK_REQUIRE(stride2 != nullptr, "null stride");
    if (stride2[0] != 1 || stride2[1] != 1) throw Error(SPK_ERR_ARGUMENT, "Stride must be 1 in sparse conv.");
    Pad4 p = pad_of(pad4);
    oh = h + p.top + p.bottom - kh + 1;
    ow = w + p.left + p.right - kw + 1;
    SPK_REQUIRE(oh >= 1 && ow >= 1, "input and kernel shapes are not compatible");
    SPK_REQUIRE(oh <= 256 && ow <= 256, "event coordinates are 8-bit: the output must be at most 256 x 256");
}

size_t spk_sparse_conv_workspace(int64_t u, int64_t t, int64_t h, int64_t w, int64_t cout, int64_t kh, int64_t kw,
                                 const int64_t *pad4_host)
{
    const int64_t s2[2] = {1, 1};
    int64_t oh = 0, ow = 0;
    if (spk_status st = guarded([&] { conv_dims(h, w, kh, kw, s2, pad4_host, oh, ow); }); st != SPK_OK) return 0;
    const int64_t n = u * t * cout;
    return al(size_t(u * cout * oh * ow) * 2) + al(size_t(n) * 4) + al(size_t(n + 1) * 8) + al(scan_workspace(n)) +
           al(size_t(u * cout * oh * ow) * 4);
}

spk_status spk_sparse_conv(const int64_t *offsets, const uint32_t *events, int64_t u, int64_t t, int64_t c, int64_t h,
                           int64_t w, const float *kernel, int64_t cout, int64_t kh, int64_t kw, double threshold,
                           const int64_t *stride2_host, const int64_t *pad4_host, int64_t *out_offsets,
                           uint32_t *out_events, int64_t cap, void *ws, size_t ws_bytes, spk_stream stream)
{
    return guarded([&] {
        check_shape(u, t, c, h, w);
        SPK_REQUIRE(cout >= 1 && cout <= 256 && kh >= 1 && kw >= 1, "invalid kernel dims");
        int64_t oh = 0, ow = 0;
        conv_dims(h, w, kh, kw, stride2_host, pad4_host, oh, ow);
        Pad4 p = pad_of(pad4_host);
        SPK_REQUIRE(cap >= u * cout * oh * ow, "event capacity must be at least U*Cout*OH*OW");
        SPK_REQUIRE(ws && ws_bytes >= spk_sparse_conv_workspace(u, t, h, w, cout, kh, kw, pad4_host),
                    "workspace is too small");
        cudaStream_t s = stream_of(stream);
        if (u == 0)
        {
            SPK_CUDA(cudaMemsetAsync(out_offsets, 0, 8, s));
            return;
        }
        Carve cv{static_cast<char *>(ws)};
        const int64_t ohw = oh * ow, n = u * t * cout, maps = u * cout;
        uint16_t *fired = cv.take<uint16_t>(size_t(maps * ohw));
        int32_t *counts = cv.take<int32_t>(size_t(n));
        int64_t *starts = cv.take<int64_t>(size_t(n + 1));
        void *scan_ws = cv.take<char>(scan_workspace(n));
        float *planes = cv.take<float>(size_t(maps * ohw));
        const size_t plane_bytes = size_t(ohw) * 4;
        const float thr = float(threshold);
        if (plane_bytes <= 24 * 1024)
        {
            const int wpc = int(std::max<size_t>(1, std::min<size_t>(8, (48 * 1024) / plane_bytes)));
            sparse_conv_kernel<true><<<unsigned(ceil_div(maps, wpc)), wpc * 32, wpc * plane_bytes, s>>>(
                offsets, events, u, int(t), int(c), kernel, int(cout), int(kh), int(kw), int(p.top), int(p.left),
                int(oh), int(ow), thr, fired, counts, nullptr);
        }
        else
            sparse_conv_kernel<false><<<unsigned(ceil_div(maps, 4)), 128, 0, s>>>(
                offsets, events, u, int(t), int(c), kernel, int(cout), int(kh), int(kw), int(p.top), int(p.left),
                int(oh), int(ow), thr, fired, counts, planes);
        SPK_LAUNCHED();
        scan_exclusive<int32_t>(counts, starts, n, scan_ws, s);
        conv_lists_kernel<<<list_grid(maps), kListWarps * 32, 0, s>>>(fired, counts, starts, u, int(t), int(cout),
                                                                      int(ow), int(ohw), out_events);
        SPK_LAUNCHED();
        conv_offsets_kernel<<<grid_for(u * t + 1, 256), 256, 0, s>>>(starts, u * t, int(cout), out_offsets);
        SPK_LAUNCHED();
    });
}

spk_status spk_sparse_convwta(const int64_t *offsets, const uint32_t *events, int64_t u, int64_t t, int64_t c,
                              int64_t h, int64_t w, const int64_t *radius2_host, int64_t count, int32_t *winners,
                              int32_t *counts, spk_stream stream)
{
    return guarded([&] {
        check_shape(u, t, c, h, w);
        SPK_REQUIRE(radius2_host && radius2_host[0] >= 0 && radius2_host[1] >= 0, "Radius items are incorrect.");
        SPK_REQUIRE(count >= 1 && count <= 1024, "winner count must be in [1, 1024]");
        if (u == 0) return;
        cudaStream_t s = stream_of(stream);
        const int wpc = int(std::max<int64_t>(1, std::min<int64_t>(8, (32 * 1024) / (count * 20))));
        sparse_wta_kernel<<<unsigned(ceil_div(u, wpc)), wpc * 32, size_t(wpc) * count * 20, s>>>(
            offsets, events, u, int(t), int(h), int(w), int(radius2_host[0]), int(radius2_host[1]), int(count), winners,
            counts);
        SPK_LAUNCHED();
    });
}

size_t spk_sparse_stdp_workspace(int64_t u, int64_t count, int64_t c, int64_t h, int64_t w, int64_t kh, int64_t kw,
                                 const int64_t *pad4_host)
{
    int64_t hp = h, wp = w;
    if (pad4_host) hp += pad4_host[0] + pad4_host[2], wp += pad4_host[1] + pad4_host[3];
    return al(size_t(u * c * hp * wp) * 4) + al(size_t(u * count * c * kh * kw) * 2) + al(size_t(u * count) * 2);
}

spk_status spk_sparse_stdp(const int64_t *offsets, const uint32_t *events, int64_t u, int64_t t, int64_t c, int64_t h,
                           int64_t w, float *kernel, int64_t cout, int64_t kh, int64_t kw, const double *configs_host,
                           int64_t nconf, const int32_t *winners, const int32_t *counts, int64_t count,
                           const int64_t *pad4_host, void *ws, size_t ws_bytes, spk_stream stream)
{
    return guarded([&] {
        check_shape(u, t, c, h, w);
        SPK_REQUIRE(cout >= 1 && kh >= 1 && kw >= 1 && count >= 1, "invalid dims");
        Pad4 p = pad_of(pad4_host);
        SPK_REQUIRE(ws && ws_bytes >= spk_sparse_stdp_workspace(u, count, c, h, w, kh, kw, pad4_host),
                    "workspace is too small");
        if (u == 0) return;
        cudaStream_t s = stream_of(stream);
        const int64_t hp = h + p.top + p.bottom, wp = w + p.left + p.right, k = c * kh * kw;
        Carve cv{static_cast<char *>(ws)};
        int32_t *last = cv.take<int32_t>(size_t(u * c * hp * wp));
        uint16_t *pre = cv.take<uint16_t>(size_t(u * count * k));
        uint16_t *post = cv.take<uint16_t>(size_t(u * count));
        SPK_CUDA(cudaMemsetAsync(last, 0, size_t(u * c * hp * wp) * 4, s));
        last_time_map_kernel<<<list_grid(u * t), kListWarps * 32, 0, s>>>(offsets, events, u * t, int(t), int(c),
                                                                          int(hp), int(wp), int(p.top), int(p.left),
                                                                          last);
        SPK_LAUNCHED();
        sparse_prepost_kernel<<<unsigned(u * count), 128, 0, s>>>(last, int(t), int(c), int(hp), int(wp), int(kh),
                                                                  int(kw), winners, counts, int(count), pre, post);
        SPK_LAUNCHED();
        launch_stdp_scan(kernel, k, cout, u, count, 2, winners, counts, pre, count * k, k, post, configs_host, nconf,
                         true, s);
    });
}

}  // extern "C"
