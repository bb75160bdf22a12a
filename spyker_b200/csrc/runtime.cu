// Library runtime: error reporting, device queries and the host-side kernel
// generators of the reference's layer constructors (src/spyker/cpu/init.cpp).
#include <atomic>
#include <cmath>
#include <ctime>
#include <mutex>
#include <random>

#include "common.cuh"

namespace spk
{
static thread_local std::string g_last_error;
static std::atomic<uint64_t> g_launches{0};

void set_error(const std::string &msg) { g_last_error = msg; }
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int sm_count()
{
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (cached[dev] == 0)
    {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cached[dev] = n;
    }
    return cached[dev];
}

size_t dtype_size(spk_dtype t)
{
    switch (t)
    {
    case SPK_I8:
    case SPK_U8: return 1;
    case SPK_I16:
    case SPK_U16:
    case SPK_F16: return 2;
    case SPK_I32:
    case SPK_U32:
    case SPK_F32: return 4;
    case SPK_I64:
    case SPK_U64:
    case SPK_F64: return 8;
    }
    return 0;
}

// The reference keeps one global std::mt19937 (src/spyker/impl.cpp:37) that
// layer constructors draw from; it is reproduced here so that the same seed
// and the same sequence of constructors give the same initial weights.
static std::mt19937 g_generator(static_cast<std::mt19937::result_type>(time(nullptr)));
static std::mutex g_generator_mutex;

// A 64-bit seed drawn from the global generator (the rate code's random
// streams: reproducible after spk_random_seed, like the reference's
// Generator() draws, cpu/code.cpp:192).
uint64_t draw_seed()
{
    std::lock_guard<std::mutex> lock(g_generator_mutex);
    const uint64_t hi = g_generator(), lo = g_generator();
    return (hi << 32) | lo;
}
}  // namespace spk

using namespace spk;

extern "C" {

const char *spk_last_error(void) { return g_last_error.c_str(); }

const char *spk_version(void) { return "spyker_b200 0.1.0 (sm_100a)"; }

uint64_t spk_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int spk_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return -1;
    return n;
}

void spk_random_seed(uint64_t seed)
{
    std::lock_guard<std::mutex> lock(g_generator_mutex);
    g_generator.seed(static_cast<std::mt19937::result_type>(seed));
}

spk_status spk_normal_kernel(double *kernel, int64_t n, double mean, double std)
{
    return guarded([&] {
        SPK_REQUIRE(kernel != nullptr && n >= 0, "invalid kernel buffer");
        std::lock_guard<std::mutex> lock(g_generator_mutex);
        std::normal_distribution<double> dist(mean, std);
        for (int64_t i = 0; i < n; ++i) kernel[i] = dist(g_generator);
    });
}

spk_status spk_gaussian_kernel(double *kernel, int64_t size, double std)
{
    return guarded([&] {
        SPK_REQUIRE(kernel != nullptr && size > 0, "invalid kernel buffer");
        const int64_t s = size / 2;
        double sum = 0;
        for (int64_t i = -s; i <= s; ++i)
            for (int64_t j = -s; j <= s; ++j)
            {
                double dist = std::sqrt(double(i * i + j * j));
                kernel[(i + s) * size + (j + s)] = std::exp(-.5 * std::pow(dist / std, 2));
            }
        for (int64_t i = 0; i < size * size; ++i) sum += kernel[i];
        for (int64_t i = 0; i < size * size; ++i) kernel[i] /= sum;
    });
}

spk_status spk_gabor_kernel(double *kernel, int64_t size, double sigma, double theta, double gamma, double lambda,
                            double psi)
{
    return guarded([&] {
        SPK_REQUIRE(kernel != nullptr && size > 0, "invalid kernel buffer");
        const double pi = 3.14159265358979323846;
        const int64_t s = size / 2;
        double sum = 0;
        for (int64_t i = -s; i <= s; ++i)
            for (int64_t j = -s; j <= s; ++j)
            {
                double x = i * std::cos(theta) + j * std::sin(theta);
                double y = -i * std::sin(theta) + j * std::cos(theta);
                double a = std::exp(-(x * x + gamma * gamma * y * y) / (2 * sigma * sigma));
                double b = std::cos(2 * pi * x / lambda + psi);
                kernel[(i + s) * size + (j + s)] = a * b;
            }
        for (int64_t i = 0; i < size * size; ++i) sum += kernel[i];
        for (int64_t i = 0; i < size * size; ++i) kernel[i] /= sum;
    });
}

spk_status spk_log_kernel(double *kernel, int64_t size, double std)
{
    return guarded([&] {
        SPK_REQUIRE(kernel != nullptr && size > 0, "invalid kernel buffer");
        const double pi = 3.14159265358979323846;
        const int64_t s = size / 2;
        const double div = -pi * std::pow(std, 4);
        for (int64_t i = -s; i <= s; ++i)
            for (int64_t j = -s; j <= s; ++j)
            {
                double a = (i * i + j * j) / (-2 * std * std);
                kernel[(i + s) * size + (j + s)] = (1 + a) * std::exp(a) / div;
            }
    });
}

}  // extern "C"
