// ZCA whitening (src/spyker/cpu/zca.cpp:67-155, opers.cpp:807-831) with
// FP64 accumulation on the GPU:
//   fit:       mean = column means of X [N, D]; sigma = (X - mean)^T (X - mean)
//              / (N - 1); sigma = U diag(lambda) U^T; transform = U diag(1 /
//              sqrt(max(lambda, 0) + epsilon)) U^T
//   transform: X <- (X - mean) transform
//   split:     [N, D] -> [N, 2, D] = (max(x, 0), max(-x, 0))
// The reference computes these with BLAS/LAPACK in the input's precision
// (its build here has neither); the symmetric eigensolve between the two
// FP64 products is the caller's (a library routine on the GPU).
#include "common.cuh"

namespace spk
{
namespace
{
// C[m][p] = scale * sum_k A(k, m) B(k, p), FP64, 64 x 64 tiles, 256 threads x
// 4 x 4 outputs, K staged 16 at a time.  MODE selects the operand loads:
//   0 covariance:  A = B = X[k][m] - mean[m]       (k: sample)
//   1 whitening:   A(k, m) = U[m][k] w[k], B(k, p) = U[p][k]   (k: eigenpair)
//   2 transform:   A(k, n) = X[n][k] - mean[k], B(k, p) = T[k][p]
constexpr int kT = 64, kK = 16;

template <int MODE>
__global__ void __launch_bounds__(256) zca_gemm_kernel(const float *__restrict__ x, const double *__restrict__ mean,
                                                       const double *__restrict__ u, const double *__restrict__ wv,
                                                       const double *__restrict__ tm, double *__restrict__ c,
                                                       float *__restrict__ cf, int64_t rows, int64_t d, int64_t kdim,
                                                       int64_t kchunk, double scale)
{
    __shared__ double sa[kK][kT + 1], sb[kK][kT + 1];
    const int64_t m0 = int64_t(blockIdx.y) * kT, p0 = int64_t(blockIdx.x) * kT;
    if (MODE == 0 && p0 < m0) return;  // symmetric: upper tiles, mirrored below
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int64_t mdim = MODE == 2 ? rows : d;
    // split K: slice z sums k in [z kchunk, (z + 1) kchunk) into its own
    // [mdim, d] block of c
    const int64_t kbeg = int64_t(blockIdx.z) * kchunk, kend = min(kdim, kbeg + kchunk);
    c += int64_t(blockIdx.z) * mdim * d;
    double acc[4][4] = {};
    for (int64_t k0 = kbeg; k0 < kend; k0 += kK)
    {
        // operands stored with k contiguous (U rows, X rows in the transform)
        // are read with consecutive threads along k, the others along m / p
        for (int i = threadIdx.x; i < kK * kT; i += 256)
        {
            const bool a_kfast = MODE != 0, b_kfast = MODE == 1;
            const int akk = a_kfast ? i % kK : i / kT, amm = a_kfast ? i / kK : i % kT;
            const int bkk = b_kfast ? i % kK : i / kT, bmm = b_kfast ? i / kK : i % kT;
            const int64_t ka = k0 + akk, kb = k0 + bkk, m = m0 + amm, p = p0 + bmm;
            double a = 0.0, b = 0.0;
            if (MODE == 0)
            {
                if (ka < kend && m < d) a = double(x[ka * d + m]) - mean[m];
                if (kb < kend && p < d) b = double(x[kb * d + p]) - mean[p];
            }
            else if (MODE == 1)
            {
                if (ka < kend && m < d) a = u[m * d + ka] * wv[ka];
                if (kb < kend && p < d) b = u[p * d + kb];
            }
            else
            {
                if (ka < kend && m < rows) a = double(x[m * d + ka]) - mean[ka];
                if (kb < kend && p < d) b = tm[kb * d + p];
            }
            sa[akk][amm] = a;
            sb[bkk][bmm] = b;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kK; ++kk)
        {
            double av[4], bv[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) av[i] = sa[kk][ty * 4 + i], bv[i] = sb[kk][tx + 16 * i];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int jj = 0; jj < 4; ++jj) acc[i][jj] = fma(av[i], bv[jj], acc[i][jj]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj)
        {
            const int64_t m = m0 + ty * 4 + i, p = p0 + tx + 16 * jj;
            if (m >= mdim || p >= d) continue;
            const double v = acc[i][jj] * scale;
            if (MODE == 2)
                cf[m * d + p] = float(v);
            else
            {
                c[m * d + p] = v;
                if (MODE == 0) c[p * d + m] = v;
            }
        }
}

// Column means: a CTA owns 32 columns (one per lane, coalesced rows), its 8
// warps take every 8th row, and the 8 partial sums meet in shared memory in
// a fixed order, so the result does not depend on scheduling.
__global__ void __launch_bounds__(256) zca_mean_kernel(const float *__restrict__ x, double *__restrict__ mean, int64_t n,
                                                       int64_t d)
{
    __shared__ double part[8][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t j = int64_t(blockIdx.x) * 32 + lane;
    double s = 0.0;
    if (j < d)
        for (int64_t i = warp; i < n; i += 8) s += double(x[i * d + j]);
    part[warp][lane] = s;
    __syncthreads();
    if (warp == 0 && j < d)
    {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < 8; ++w) t += part[w][lane];
        mean[j] = t / double(n);
    }
}

// cov = scale * sum of the split-K slices, in slice order
__global__ void zca_reduce_kernel(const double *__restrict__ part, double *__restrict__ cov, int64_t dd, int slices,
                                  double scale)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < dd; i += int64_t(gridDim.x) * blockDim.x)
    {
        double t = 0.0;
        for (int z = 0; z < slices; ++z) t += part[z * dd + i];
        cov[i] = t * scale;
    }
}

__global__ void zca_weights_kernel(const double *__restrict__ lambda, double *__restrict__ w, int64_t d, double eps)
{
    for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < d; j += int64_t(gridDim.x) * blockDim.x)
        w[j] = 1.0 / sqrt((lambda[j] > 0.0 ? lambda[j] : 0.0) + eps);
}

template <typename T>
__global__ void zca_split_kernel(const T *__restrict__ in, T *__restrict__ out, int64_t n, int64_t d)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n * d; i += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t r = i / d, j = i - r * d;
        const T v = in[i];
        out[(r * 2) * d + j] = v > T(0) ? v : T(0);
        out[(r * 2 + 1) * d + j] = -v > T(0) ? -v : T(0);
    }
}

dim3 tiles(int64_t m, int64_t p, int z = 1)
{
    SPK_REQUIRE(ceil_div(m, kT) <= 65535, "too many rows for one call");
    return dim3(unsigned(ceil_div(p, kT)), unsigned(ceil_div(m, kT)), unsigned(z));
}

// Split-K slices of the covariance: the upper-triangle tiles alone fill the
// GPU only for large D, so small D splits the samples into up to 3 CTAs
// (the residency of this kernel) per SM, at least 1024 samples a slice.
int stats_slices(int64_t n, int64_t d)
{
    const int64_t t = ceil_div(d, kT), upper = t * (t + 1) / 2;
    int64_t s = (3 * int64_t(sm_count())) / upper;
    s = std::min<int64_t>(s, ceil_div(n, 1024));
    return int(std::max<int64_t>(1, std::min<int64_t>(s, 64)));
}
}  // namespace
}  // namespace spk

using namespace spk;

extern "C" {

int64_t spk_zca_stats_workspace(int64_t n, int64_t d)
{
    if (n < 2 || d < 1) return 0;
    const int slices = stats_slices(n, d);
    return slices > 1 ? int64_t(slices) * d * d * int64_t(sizeof(double)) : 0;
}

spk_status spk_zca_stats(const float *x, int64_t n, int64_t d, double *mean, double *cov, void *work,
                         int64_t work_bytes, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(n >= 2 && d >= 1 && ceil_div(d, 32) <= INT32_MAX, "ZCA needs at least two samples");
        SPK_REQUIRE(x && mean && cov, "null pointer");
        const int slices = stats_slices(n, d);
        SPK_REQUIRE(slices == 1 || (work && work_bytes >= spk_zca_stats_workspace(n, d)), "workspace too small");
        cudaStream_t s = stream_of(stream);
        zca_mean_kernel<<<unsigned(ceil_div(d, 32)), 256, 0, s>>>(x, mean, n, d);
        SPK_LAUNCHED();
        const double scale = 1.0 / double(n - 1);
        const int64_t kchunk = ceil_div(ceil_div(n, int64_t(slices)), int64_t(kK)) * kK;
        double *part = slices > 1 ? static_cast<double *>(work) : cov;
        zca_gemm_kernel<0><<<tiles(d, d, slices), 256, 0, s>>>(x, mean, nullptr, nullptr, nullptr, part, nullptr, n, d, n,
                                                               kchunk, slices > 1 ? 1.0 : scale);
        SPK_LAUNCHED();
        if (slices > 1)
        {
            zca_reduce_kernel<<<grid_for(d * d, 256), 256, 0, s>>>(part, cov, d * d, slices, scale);
            SPK_LAUNCHED();
        }
    });
}

spk_status spk_zca_matrix(const double *vectors, const double *values, int64_t d, double epsilon, double *work,
                          double *trans, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(d >= 1 && vectors && values && work && trans, "invalid arguments");
        cudaStream_t s = stream_of(stream);
        zca_weights_kernel<<<grid_for(d, 256), 256, 0, s>>>(values, work, d, epsilon);
        SPK_LAUNCHED();
        zca_gemm_kernel<1><<<tiles(d, d), 256, 0, s>>>(nullptr, nullptr, vectors, work, nullptr, trans, nullptr, d, d,
                                                        d, d, 1.0);
        SPK_LAUNCHED();
    });
}

spk_status spk_zca_transform(const float *x, int64_t n, int64_t d, const double *mean, const double *trans, float *out,
                             spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(n >= 0 && d >= 1 && x && mean && trans && out, "invalid arguments");
        SPK_REQUIRE(static_cast<const void *>(x) != static_cast<const void *>(out), "the output must not alias the input");
        if (n == 0) return;
        zca_gemm_kernel<2><<<tiles(n, d), 256, 0, stream_of(stream)>>>(x, mean, nullptr, nullptr, trans, nullptr, out,
                                                                        n, d, d, d, 1.0);
        SPK_LAUNCHED();
    });
}

spk_status spk_zca_split(const void *in, spk_dtype type, void *out, int64_t n, int64_t d, spk_stream stream)
{
    return guarded([&] {
        SPK_REQUIRE(n >= 0 && d >= 1, "invalid dims");
        if (n == 0) return;
        dispatch_real(type, [&](auto z) {
            using T = decltype(z);
            zca_split_kernel<T><<<grid_for(n * d, 256), 256, 0, stream_of(stream)>>>(static_cast<const T *>(in),
                                                                                     static_cast<T *>(out), n, d);
        });
        SPK_LAUNCHED();
    });
}

}  // extern "C"
