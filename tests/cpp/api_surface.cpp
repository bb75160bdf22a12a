// Compile-and-link check of the C++ Spyker:: layer's full surface: every
// module and function of include/spyker_b200.hpp named after the reference's
// opers.h is called once with the reference's argument forms.  Built (not run)
// by tests/test_cpp_layer.py::test_full_surface_links; the layer's results are
// compared with the Python API's in tests/cpp/layer_check.cpp.
#include <spyker_b200.hpp>

#include <cstdio>

using namespace Spyker;

int main()
{
    Tensor img(Type::F32, {2, 1, 28, 28});
    DoG dog(3, {DoGFilter(1, 2), DoGFilter(2, 1)}, 3);
    Gabor gabor(2, {GaborFilter(2, 45, .5, 4, 0), GaborFilter(2, 135, .5, 4, 0)}, 2);
    LoG log(2, std::vector<F64>{1.0, 2.0}, 2);
    Tensor d = dog(img), g = gabor(img), l = log(img);
    Tensor codes = code(d, 15, true), lat = code(d, 15, false, Type::U8);
    Conv conv(2, 8, 5, 1, 2, .8, .05);
    conv.stdpconfig = {STDPConfig(.004, -.003)};
    Tensor pot = threshold(conv(codes), 15);
    pot = inhibit(pot);
    Winners w = convwta(pot, 3, 5);
    Tensor spk = fire(pot);
    conv.stdp(codes, w, spk);
    Tensor pooled = pool(spk, 2), padded = pad(spk, 1), last = gather(spk), back = scatter(last, 15);
    Tensor inf = infinite(pot);
    Tensor flat = pooled.reshape({2, 15, 8 * 14 * 14});
    FC fc1(8 * 14 * 14, 10);
    fc1.stdpconfig = {STDPConfig(.004, -.003)};
    Tensor out = fc1(flat), sout = fc1(flat, true), plain = fc(flat, fc1.kernel);
    Winners fw = fcwta(out, 1, 2);
    fc1.stdp(flat, fw, fire(out));
    Tensor times(Type::F32, {2, 10}), target(Type::I64, {2});
    Tensor grad = backward(times, target, 15, 1.0);
    fc1.bpconfig = BPConfig(1, .01, .1, .001);
    Tensor in2(Type::F32, {2, 8 * 14 * 14});
    Tensor next = fc1.backward(in2, times, grad);
    Tensor labels = labelize(Tensor(Type::F32, {2, 15, 10}), 1.0);
    LayerOutput lo = conv_fire_wta(codes, conv, 15, 3, 5, 2);
    SparseTensor sc = Sparse::code(d, 15), sd(codes, 0.0);
    SparseTensor sp = Sparse::inhibit(conv(sc, 15.0));
    Winners sw = Sparse::convwta(sp, 3, 5);
    conv.stdp(sc, sw);
    SparseTensor sq = Sparse::pool(Sparse::pad(sp, 1), 2), sr = Sparse::conv(sd, conv.kernel, 15.0, 1, 2);
    Tensor first = Sparse::gather(sq), dense = sr.dense();
    std::printf("%lld %f %d %d\n", (long long)sq.numel(), sp.sparsity(), int(first.dims()), int(dense.dims()));
    synchronize();
    std::printf("%d %d %d %d %d %d %d %d %d\n", int(g.dims()), int(l.dims()), int(lat.dims()), int(padded.dims()),
                int(back.dims()), int(inf.dims()), int(sout.dims() + plain.dims()), int(next.dims() + labels.dims()),
                int(lo.spikes.dims()));
    return 0;
}
