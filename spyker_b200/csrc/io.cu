// IDX (MNIST) files read straight into caller memory, normally pinned host
// memory that a side stream then copies to the GPU while the previous batch
// is processed (helper/mnist.cpp:10-60: a big-endian header of magic 2049
// with the label count, or 2051 with count, rows and columns, then the u8
// payload).  The payload is read with positioned reads on several threads.
#include "common.cuh"

#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <thread>
#include <vector>

namespace spk
{
namespace
{
struct File
{
    int fd = -1;
    explicit File(const char *path) : fd(::open(path, O_RDONLY | O_CLOEXEC)) {}
    ~File()
    {
        if (fd >= 0) ::close(fd);
    }
};

bool read_at(int fd, void *dst, int64_t bytes, int64_t offset)
{
    auto *p = static_cast<char *>(dst);
    while (bytes > 0)
    {
        const ssize_t got = ::pread(fd, p, size_t(std::min<int64_t>(bytes, int64_t(1) << 30)), off_t(offset));
        if (got <= 0) return false;
        p += got, bytes -= got, offset += got;
    }
    return true;
}

int64_t big_endian(const unsigned char *b) { return (int64_t(b[0]) << 24) | (b[1] << 16) | (b[2] << 8) | b[3]; }
}  // namespace
}  // namespace spk

using namespace spk;

extern "C" {

spk_status spk_idx_shape(const char *path, int32_t magic, int64_t *shape, int64_t *ndim, int64_t *offset)
{
    return guarded([&] {
        SPK_REQUIRE(path && shape && ndim && offset, "null pointer");
        SPK_REQUIRE(magic == 2049 || magic == 2051, "IDX magic must be 2049 (labels) or 2051 (images)");
        File f(path);
        SPK_REQUIRE(f.fd >= 0, std::string("cannot open ") + path);
        const int words = magic == 2049 ? 2 : 4;
        unsigned char head[16];
        SPK_REQUIRE(read_at(f.fd, head, 4 * words, 0), std::string("short IDX header in ") + path);
        SPK_REQUIRE(big_endian(head) == magic, std::string("wrong IDX magic in ") + path);
        if (magic == 2049)
        {
            shape[0] = big_endian(head + 4);
            *ndim = 1;
        }
        else
        {
            shape[0] = big_endian(head + 4), shape[1] = 1, shape[2] = big_endian(head + 8), shape[3] = big_endian(head + 12);
            *ndim = 4;
        }
        *offset = 4 * words;
    });
}

spk_status spk_idx_read(const char *path, int64_t offset, void *dst, int64_t bytes, int threads)
{
    return guarded([&] {
        SPK_REQUIRE(path && (dst || bytes == 0) && bytes >= 0 && offset >= 0, "invalid arguments");
        File f(path);
        SPK_REQUIRE(f.fd >= 0, std::string("cannot open ") + path);
        const int64_t chunk = int64_t(16) << 20;
        const int n = int(std::max<int64_t>(1, std::min<int64_t>(std::max(threads, 1), (bytes + chunk - 1) / chunk)));
        std::vector<char> ok(size_t(n), 1);
        auto part = [&](int i) {
            const int64_t a = bytes * i / n, b = bytes * (i + 1) / n;
            ok[size_t(i)] = read_at(f.fd, static_cast<char *>(dst) + a, b - a, offset + a);
        };
        if (n == 1)
            part(0);
        else
        {
            std::vector<std::thread> pool;
            for (int i = 0; i < n; ++i) pool.emplace_back(part, i);
            for (auto &t : pool) t.join();
        }
        SPK_REQUIRE(std::all_of(ok.begin(), ok.end(), [](char c) { return c != 0; }),
                    std::string("short IDX payload in ") + path);
    });
}

}  // extern "C"
