// One layer step through the C++ Spyker:: layer (include/spyker_b200.hpp):
// DoG -> code -> fused conv/fire/WTA/pool -> STDP, and the same layer op by
// op.  Writes every result as raw bytes to <out_dir>/<name>.bin for the
// Python test to compare with the Python API on the same inputs.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "spyker_b200.hpp"

static void dump(const std::string &dir, const char *name, const Spyker::Tensor &t)
{
    std::vector<unsigned char> v(t.bytes());
    if (!v.empty()) t.to_host(v.data());
    FILE *f = std::fopen((dir + "/" + name + ".bin").c_str(), "wb");
    if (!f) throw Spyker::Error("cannot write output");
    std::fwrite(v.data(), 1, v.size(), f);
    std::fclose(f);
}

static void dump_winners(const std::string &dir, const char *name, const Spyker::Winners &w)
{
    std::vector<int64_t> v;
    for (size_t i = 0; i < w.size(); ++i)
        for (const auto &x : w[i]) v.insert(v.end(), {int64_t(i), x.c, x.t, x.z, x.y, x.x});
    FILE *f = std::fopen((dir + "/" + name + ".bin").c_str(), "wb");
    if (!f) throw Spyker::Error("cannot write output");
    std::fwrite(v.data(), sizeof(int64_t), v.size(), f);
    std::fclose(f);
}

int main(int argc, char **argv)
{
    if (argc < 2) return 2;
    const std::string dir = argv[1];
    try
    {
        const Spyker::Size b = 6, h = 20, w = 18, t = 15;
        std::vector<float> img(static_cast<size_t>(b * h * w));
        for (Spyker::Size i = 0; i < b; ++i)
            for (Spyker::Size y = 0; y < h; ++y)
                for (Spyker::Size x = 0; x < w; ++x)
                {
                    const double r = std::sin(0.37 * double(x + 3 * i)) * std::cos(0.23 * double(y * (i + 1)));
                    img[size_t((i * h + y) * w + x)] = float(0.5 + 0.5 * r);
                }
        auto images = Spyker::Tensor::from_host(img.data(), Spyker::Type::F32, {b, 1, h, w});
        dump(dir, "images", images);
        Spyker::DoG dog(3, {Spyker::DoGFilter(1, 2), Spyker::DoGFilter(2, 1)}, 3);
        auto codes = Spyker::code(dog(images), t);
        Spyker::Conv conv(2, 12, 5, 1, 2, 0.8, 0.05);
        conv.stdpconfig = {Spyker::STDPConfig(0.004, -0.003)};
        dump(dir, "codes", codes);
        dump(dir, "kernel0", conv.kernel);

        // op by op on the plain FP32 path
        auto pot = conv(codes);
        auto out = Spyker::inhibit(Spyker::threshold(pot, 4.0));
        auto spk_ops = Spyker::fire(out);
        auto win_ops = Spyker::convwta(out, 2, 3);
        auto pool_ops = Spyker::pool(spk_ops, 2);
        dump(dir, "spikes_ops", spk_ops);
        dump(dir, "pooled_ops", pool_ops);
        dump_winners(dir, "winners_ops", win_ops);

        // the fused layer on the tensor cores, then STDP with its winners
        conv.precision = SPK_CONV_BF16X3;
        auto layer = Spyker::conv_fire_wta(codes, conv, 4.0, 2, 3, 2);
        dump(dir, "spikes_fused", layer.spikes);
        dump(dir, "pooled_fused", layer.pooled);
        dump_winners(dir, "winners_fused", layer.winners);
        conv.stdp(codes, layer.winners, layer.spikes);
        dump(dir, "kernel1", conv.kernel);
        Spyker::synchronize();
        std::printf("ok\n");
    }
    catch (const std::exception &e)
    {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
