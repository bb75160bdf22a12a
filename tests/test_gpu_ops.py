"""GPU parity: every op of the hot path through the public API (and hence the
C ABI) against the CPU oracle on seeded inputs.  Integer / index / spike /
winner outputs are compared bit-exactly; FP32 potentials against the FP64
oracle within a relative tolerance of 1e-5."""

import numpy as np
import pytest
import torch

import spyker_b200 as spyker
from spyker_b200 import synth
from tests.golden import make_golden

pytestmark = pytest.mark.gpu
DEV = "cuda"
CFG = [(0.004, -0.003, 1.0, 0.0, 1.0)]


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def host(t):
    return t.cpu().numpy()


def winners_np(w: spyker.Winners):
    rec = host(w.records).astype(np.int64)
    cnt = host(w.counts).astype(np.int64)
    for i in range(rec.shape[0]):
        rec[i, cnt[i]:] = 0
    return rec, cnt


def oracle_winners(win, cnt):
    win = win.copy()
    for i in range(win.shape[0]):
        win[i, cnt[i]:] = 0
    return win, cnt


@pytest.fixture(scope="module")
def dog(port):
    img = synth.strokes(32, seed=11).astype(np.float32) / 255
    return port.filter("dog", img[:, None], make_golden.dog_kernel(port), (3, 3, 3, 3))


@pytest.fixture(scope="module")
def layer(port, dog):
    codes = port.rank_code(dog, 15)
    w = synth.conv_weights(30, 2, 5, seed=2)
    pot = port.conv(codes, w, (1, 1), (2, 2, 2, 2))
    th = port.threshold(pot, 15.0)
    inh = port.inhibit(th)
    return dict(codes=codes, w=w, pot=pot, th=th, inh=inh, spk=port.fire(inh))


def test_filters_exact(port):
    img = synth.strokes(8, seed=5).astype(np.float32)[:, None] / 255
    dog = spyker.DoG(3, [spyker.DoGFilter(1, 2), spyker.DoGFilter(2, 1)], pad=3)
    assert np.array_equal(host(dog.kernel), make_golden.dog_kernel(port))
    assert np.array_equal(host(dog(cuda(img))), port.filter("dog", img, make_golden.dog_kernel(port), (3, 3, 3, 3)))
    log = spyker.LoG(3, [1.0, 2.0], pad=(1, 2))
    assert np.array_equal(host(log(cuda(img))), port.filter("log", img, host(log.kernel), (1, 2, 1, 2)))
    gab = spyker.Gabor(5, [spyker.GaborFilter(2.0, th, 0.5, 5.0, 0.0) for th in (0, 45, 90, 135)], pad=5)
    assert np.array_equal(host(gab(cuda(img))), port.filter("gabor", img, host(gab.kernel), (5, 5, 5, 5)))


def test_filters_exact_large_planes(port):
    """Planes taller than one CTA's staged rows (256 x 256, 11 x 11 Gabor
    bank; DoG on 64 x 96) against the FP64 oracle, bit for bit."""
    img = synth.textures(2, seed=3, size=256)[:, None]
    gab = spyker.Gabor(5, [spyker.GaborFilter(2.5, th, 0.5, lam, 0.0) for th in (0, 45, 90, 135) for lam in (5.0, 10.0)],
                       pad=5)
    assert np.array_equal(host(gab(cuda(img))), port.filter("gabor", img, host(gab.kernel), (5, 5, 5, 5)))
    img2 = synth.textures(3, seed=4, size=96)[:, None, :64, :]
    dog = spyker.DoG(3, [spyker.DoGFilter(1, 2), spyker.DoGFilter(2, 1)], pad=(2, 3))
    assert np.array_equal(host(dog(cuda(np.ascontiguousarray(img2)))),
                          port.filter("dog", np.ascontiguousarray(img2), host(dog.kernel), (2, 3, 2, 3)))


def stable_code(x: np.ndarray, time: int) -> np.ndarray:
    """Rank code with ties in index order (the GPU's documented order):
    cpu/code.cpp:93-101 with a stable sort, U16 conversion as x86-64 GCC."""
    flat = x.reshape(x.shape[0], -1)
    out = np.zeros((flat.shape[0], time, flat.shape[1]), np.uint8)
    for i in range(flat.shape[0]):
        v = flat[i].astype(np.float32)
        v = np.where(v == 0, np.float32(0), v)
        order = np.lexsort((np.arange(v.size), -v))
        cnt = int((v > v.min()).sum())
        with np.errstate(divide="ignore", invalid="ignore"):
            scale = np.float32(np.float32(time) + np.float32(1e-5)) / np.float32(cnt)
            prod = np.arange(v.size, dtype=np.float32) * scale
        ok = (prod > -2.0 ** 31) & (prod < 2.0 ** 31)
        tm = np.zeros(v.size, np.int64)
        tm[order] = np.where(ok, np.trunc(np.where(ok, prod, 0)).astype(np.int64) & 0xFFFF, 0)
        out[i] = tm[None, :] <= np.arange(time)[:, None]
    return out.reshape((x.shape[0], time) + x.shape[1:])


@pytest.mark.parametrize("sort", [True, False])
def test_code(port, dog, sort):
    got = host(spyker.code(cuda(dog), 15, sort=sort))
    want = port.rank_code(dog, 15, sort)
    if not sort:
        assert np.array_equal(got, want)
        return
    # Sorted: exact except for equal values split across a time bin, where the
    # reference's std::sort order is not stable; the GPU order is (value desc,
    # index asc), reproduced exactly by the stable restatement.
    match = (got == want).mean()
    assert match > 0.9999
    assert np.array_equal(got, stable_code(dog, 15))


def test_code_large_images(port):
    """Images above 16384 values (device-wide sort): the 8 x 256 x 256 Gabor
    geometry, a size that is not a multiple of the sort chunk, and u8 input
    full of ties."""
    rng = np.random.default_rng(21)
    big = rng.random((2, 8, 256, 256), dtype=np.float32)
    big[big < 0.3] = 0  # a large tied minimum
    got = host(spyker.code(cuda(big), 30))
    assert np.array_equal(got, stable_code(big, 30))
    odd = rng.random((3, 3, 100, 111), dtype=np.float32)
    got = host(spyker.code(cuda(odd), 15))
    assert np.array_equal(got, stable_code(odd, 15))
    assert np.array_equal(got, port.rank_code(odd, 15))  # no ties: the reference order too
    u8 = (rng.random((2, 40000)) * 7).astype(np.uint8)
    got = host(spyker.code(cuda(u8), 12, dtype="f32"))
    assert np.array_equal(got, stable_code(u8, 12).astype(np.float32))
    ev = spyker.sparse.code(cuda(odd), 15)
    want = port.sparse_from_dense(stable_code(odd, 15))
    off, zyx = ev.lists()
    assert np.array_equal(off, want[0]) and np.array_equal(zyx, want[1].reshape(-1, 3))


@pytest.mark.parametrize("x", [257, 300, 512, 513, 700, 1024, 1100, 1568, 2000, 2048])
def test_code_row_sizes(port, x):
    """Rows of 257..2048 values take the 256-thread register sort (2, 4 or 8
    keys per thread): F32 with a tied minimum and ties inside, u8 full of
    ties, F32 output, sizes off the 16-byte vector width, and the event-list
    times."""
    rng = np.random.default_rng(x)
    f = rng.random((5, x), dtype=np.float32)
    f[f < 0.4] = 0
    f[:, ::7] = f[:, 3:4]  # equal values across the row
    assert np.array_equal(host(spyker.code(cuda(f), 15)), stable_code(f, 15))
    u8 = (rng.random((3, x)) * 9).astype(np.uint8)
    assert np.array_equal(host(spyker.code(cuda(u8), 11)), stable_code(u8, 11))
    assert np.array_equal(host(spyker.code(cuda(f), 7, dtype="f32")), stable_code(f, 7).astype(np.float32))
    if x % 16:
        return  # event coordinates are 8-bit: lay the row out as [x / 16, 1, 16]
    img = f.reshape(5, x // 16, 1, 16)
    ev = spyker.sparse.code(cuda(img), 15)
    want = port.sparse_from_dense(stable_code(img, 15).reshape(5, 15, x // 16, 1, 16))
    off, zyx = ev.lists()
    assert np.array_equal(off, want[0]) and np.array_equal(zyx, want[1].reshape(-1, 3))


def test_code_u8_and_edges(port):
    img = synth.strokes(16, seed=3)
    assert np.array_equal(host(spyker.code(cuda(img), 10, sort=False)), port.rank_code(img, 10, False))
    assert np.array_equal(host(spyker.code(cuda(img), 10)), stable_code(img, 10))
    const = np.ones((3, 50), np.float32)
    assert np.array_equal(host(spyker.code(cuda(const), 15)), port.rank_code(const, 15))
    # one value above a large tied minimum: the time conversion wraps
    one = np.zeros((2, 9000), np.float32)
    one[:, 5] = 2.0
    assert np.array_equal(host(spyker.code(cuda(one), 15)), stable_code(one, 15))
    tiny = np.array([[3.0]], np.float32)
    assert np.array_equal(host(spyker.code(cuda(tiny), 4)), port.rank_code(tiny, 4))


def test_threshold_fire_infinite(port, layer):
    pot = layer["pot"]
    t = cuda(pot)
    spyker.threshold(t, 15.0)
    assert np.array_equal(host(t), port.threshold(pot, 15.0))
    t2 = spyker.threshold(cuda(pot), 10.0, 2.5, inplace=False)
    assert np.array_equal(host(t2), port.threshold(pot, 10.0, 2.5))
    assert np.array_equal(host(spyker.fire(cuda(layer["inh"]))), port.fire(layer["inh"]))
    assert np.array_equal(host(spyker.fire(cuda(pot), 20.0, "f32")), port.fire(pot, 20.0, np.float32))
    odd = cuda(pot).reshape(-1)[3:1000003]  # unaligned view, odd length
    assert np.array_equal(host(spyker.fire(odd.contiguous(), 18.0)), port.fire(host(odd), 18.0))
    assert np.array_equal(host(spyker.infinite(cuda(pot), 0.0)), port.infinite(pot, 0.0))
    # host arrays are processed on the GPU and written back in place
    h = pot.copy()
    spyker.threshold(h, 15.0)
    assert np.array_equal(h, port.threshold(pot, 15.0))


def test_gather_scatter_pad(port, layer):
    spk = layer["spk"]
    g = spyker.gather(cuda(spk))
    assert np.array_equal(host(g), port.gather(spk))
    assert np.array_equal(host(spyker.gather(cuda(layer["pot"]), 20.0, "f32")),
                          port.gather(layer["pot"], 20.0, np.float32))
    assert np.array_equal(host(spyker.scatter(g, 15)), port.scatter(host(g), 15))
    assert np.array_equal(host(spyker.pad(cuda(spk), (1, 2, 3, 4))), port.pad(spk, (1, 2, 3, 4), 0))


@pytest.mark.parametrize("args", [((2, 2), None, 0), ((3, 3), (2, 2), 1), ((2, 2), None, (1, 0, 1, 0)),
                                  ((28, 28), None, 0)])
def test_pool(port, layer, args):
    k, s, p = args
    p4 = spyker.expand4(p)
    for a in (layer["spk"], layer["inh"]):
        got = host(spyker.pool(cuda(a), k, s, p))
        assert np.array_equal(got, port.pool(a, spyker.expand2(k), spyker.expand2(s or k), p4))


def test_pool_staging_edges(port):
    """Planes staged from an unaligned view, tiles that end mid-range, and
    planes too large to stage (direct kernels)."""
    rng = np.random.default_rng(11)
    base = cuda(rng.random((7 * 3 * 5 * 13 * 11 + 3,), dtype=np.float32))
    view = base[3:].view(7, 3, 5, 13, 11)  # 12-byte offset from the allocation
    want = port.pool(host(view), (3, 2), (2, 3), (1, 0, 2, 1))
    assert np.array_equal(host(spyker.pool(view, (3, 2), (2, 3), (1, 0, 2, 1))), want)
    u8 = (rng.random((3, 4, 7, 9, 9)) < 0.3).astype(np.uint8)
    for k, s, p in (((2, 2), None, 0), ((9, 9), None, 0), ((4, 3), (1, 2), (3, 2, 1, 0))):
        got = host(spyker.pool(cuda(u8), k, s, p))
        assert np.array_equal(got, port.pool(u8, spyker.expand2(k), spyker.expand2(s or k), spyker.expand4(p)))
    big = rng.random((1, 2, 1, 180, 170), dtype=np.float32)  # 122 KB planes
    for k in (2, 10):
        got = host(spyker.pool(cuda(big), k))
        assert np.array_equal(got, port.pool(big, (k, k), (k, k), (0, 0, 0, 0)))


@pytest.mark.parametrize("values", ["spikes", "bytes"])
def test_pool_word_kernels(port, values):
    """u8 pooling from 32-bit words: 2-wide windows (rows of 2 and 3, output
    rows that end mid-word) and whole-plane windows, on 0/1 spikes and on any
    byte values; an unaligned view takes the per-output kernel."""
    rng = np.random.default_rng(17)
    hi = 2 if values == "spikes" else 256
    for shp, k in (((3, 5, 4, 12, 12), (2, 2)), ((2, 3, 5, 9, 20), (3, 2)), ((4, 2, 3, 6, 10), (6, 10)),
                   ((2, 15, 30, 14, 14), (14, 14)), ((2, 15, 30, 28, 28), (2, 2))):
        a = rng.integers(0, hi, size=shp).astype(np.uint8)
        got = host(spyker.pool(cuda(a), k))
        assert np.array_equal(got, port.pool(a, k, k, (0, 0, 0, 0)))
    base = cuda(rng.integers(0, hi, size=(2 * 3 * 12 * 12 + 1,)).astype(np.uint8))
    view = base[1:].view(2, 1, 3, 12, 12)
    assert np.array_equal(host(spyker.pool(view, 2)), port.pool(host(view), (2, 2), (2, 2), (0, 0, 0, 0)))


def test_inhibit(port, layer):
    for a, thr in ((layer["th"], 0.0), (layer["pot"], 25.0)):
        t = cuda(a)
        spyker.inhibit(t, thr)
        assert np.array_equal(host(t), port.inhibit(a, thr))
    u = layer["spk"].copy()
    t = cuda(u)
    spyker.inhibit(t)
    assert np.array_equal(host(t), port.inhibit(u))


@pytest.mark.parametrize("radius,count", [((3, 3), 5), ((1, 1), 8), ((0, 2), 40)])
def test_convwta(port, layer, radius, count):
    for a in (layer["inh"], layer["spk"]):
        got = winners_np(spyker.convwta(cuda(a), radius, count))
        want = oracle_winners(*port.convwta(a, radius, count))
        assert np.array_equal(got[1], want[1])
        assert np.array_equal(got[0], want[0])


def test_convwta_lists(port, layer):
    w = spyker.convwta(cuda(layer["inh"]), 3, 5)
    win, cnt = port.convwta(layer["inh"], (3, 3), 5)
    assert len(w) == win.shape[0]
    for i in range(len(w)):
        assert [(x.z, x.y, x.x) for x in w[i]] == [tuple(win[i, j, 2:]) for j in range(cnt[i])]


def test_fcwta_and_fc(port):
    rng = np.random.default_rng(9)
    x = (rng.random((16, 15, 120)) * 3).astype(np.float32)
    got = winners_np(spyker.fcwta(cuda(x), 2, 4, 1.0))
    want = oracle_winners(*port.fcwta(x, 2, 4, 1.0))
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    w = rng.random((10, 120)).astype(np.float32)
    out = host(spyker.fc(cuda(x), cuda(w)))
    ref = port.fc(x, w.astype(np.float64), out_dtype=np.float64)
    assert np.allclose(out, ref, rtol=1e-5, atol=1e-5)


def test_conv_fp32_within_tolerance(port, layer):
    got = host(spyker.conv(cuda(layer["codes"]), cuda(layer["w"]), 1, 2, precision="fp32"))
    ref = port.conv(layer["codes"], layer["w"].astype(np.float64), (1, 1), (2, 2, 2, 2), out_dtype=np.float64)
    rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-30)
    assert rel.max() <= 1e-5
    # strided, asymmetric pad, float input
    x = np.random.default_rng(1).random((4, 3, 3, 17, 19)).astype(np.float32)
    w = np.random.default_rng(2).random((7, 3, 3, 4)).astype(np.float32)
    got = host(spyker.conv(cuda(x), cuda(w), (2, 1), (1, 0, 2, 3), precision="fp32"))
    ref = port.conv(x, w.astype(np.float64), (2, 1), (1, 0, 2, 3), out_dtype=np.float64)
    assert np.allclose(got, ref, rtol=1e-5, atol=1e-6)


def test_conv_stdp(port, layer):
    codes, w, spk = layer["codes"], layer["w"], layer["spk"]
    win, cnt = port.convwta(spk, (3, 3), 5)
    conv = spyker.Conv(2, 30, 5, pad=2)
    conv.kernel.copy_(cuda(w))
    conv.stdpconfig = [spyker.STDPConfig(0.004, -0.003)]
    wdev = spyker.convwta(cuda(spk), 3, 5)
    conv.stdp(cuda(codes), wdev, cuda(spk))
    want = port.convstdp(codes, w, spk, CFG, win, cnt, (1, 1), (2, 2, 2, 2))
    assert np.array_equal(host(conv.kernel), want)
    # host winner lists, several configs, skipped negative config
    conv.kernel.copy_(cuda(w))
    conv.stdpconfig = [spyker.STDPConfig(0.004, -0.003), spyker.STDPConfig(0.01, -0.02, False, 0.2, 0.9)]
    lists = [[spyker.Winner((j % 3) - 1, 0, *win[i, j, 2:]) for j in range(cnt[i])] for i in range(len(cnt))]
    conv.stdp(cuda(codes), lists, cuda(spk))
    w2 = win.copy()
    w2[:, :, 0] = np.arange(win.shape[1])[None] % 3 - 1
    want = port.convstdp(codes, w, spk, CFG + [(0.01, -0.02, 0.0, 0.2, 0.9)], w2, cnt, (1, 1), (2, 2, 2, 2))
    assert np.array_equal(host(conv.kernel), want)


@pytest.mark.parametrize("kind", ["random01", "values"])
def test_conv_stdp_noncumulative_input(port, kind):
    """STDP inputs that are not cumulative 0/1 spikes (a word of four
    positions then takes the lane-by-lane first-spike scan) against the
    oracle; the other positions of the batch take the byte-sum path."""
    rng = np.random.default_rng(21 if kind == "random01" else 22)
    b, t, c, h, w = 6, 12, 3, 12, 12
    fst = rng.integers(0, t + 3, size=(b, c, h, w))
    x = (fst[:, None] <= np.arange(t)[None, :, None, None, None]).astype(np.uint8)
    flip = rng.random(x.shape) < 0.02
    x = np.where(flip, (1 - x) if kind == "random01" else 3 * x + 1, x).astype(np.uint8)
    wgt = rng.uniform(0.3, 0.9, size=(10, c, 3, 3)).astype(np.float32)
    o = (port.conv(x, wgt, (1, 1), (1, 1, 1, 1)) > 4.0).astype(np.uint8)
    win, cnt = port.convwta(o.astype(np.float32), (1, 1), 4)
    conv = spyker.Conv(c, 10, 3, pad=1)
    conv.kernel.copy_(cuda(wgt))
    conv.stdpconfig = [spyker.STDPConfig(0.004, -0.003)]
    conv.stdp(cuda(x), spyker.convwta(cuda(o.astype(np.float32)), 1, 4), cuda(o))
    want = port.convstdp(x, wgt, o, CFG, win, cnt, (1, 1), (1, 1, 1, 1))
    assert np.array_equal(host(conv.kernel), want)
    assert not np.array_equal(want, wgt)


def test_fc_stdp(port):
    rng = np.random.default_rng(3)
    x = (rng.random((12, 15, 64)) > 0.6).astype(np.uint8)
    w = rng.random((20, 64)).astype(np.float32)
    o = (port.fc(x, w, out_dtype=np.float32) > 12).astype(np.uint8)
    win, cnt = port.fcwta(o, 1, 3)
    fc = spyker.FC(64, 20)
    fc.kernel.copy_(cuda(w))
    fc.stdpconfig = [spyker.STDPConfig(0.004, -0.003)]
    fc.stdp(cuda(x), spyker.fcwta(cuda(o), 1, 3), cuda(o))
    assert np.array_equal(host(fc.kernel), port.fcstdp(x, w, o, CFG, win, cnt))


def test_backprop_helpers(port, golden):
    got = host(spyker.backward(cuda(golden["bw_in"]), cuda(golden["bw_target"]), 15, 2.0))
    assert np.array_equal(got, golden["bw_out"])
    assert np.array_equal(host(spyker.labelize(cuda(golden["fc_in"]), 2.5)), golden["labels"])
    x = golden["fc_in"]
    assert np.array_equal(host(spyker.labelize(cuda(x), 100.0)), port.labelize(x, 100.0))
    rng = np.random.default_rng(8)
    w = (rng.random((10, 40)) - 0.5).astype(np.float32)
    g = rng.standard_normal((16, 10)).astype(np.float32)
    xi = (rng.random((16, 40)) * 15).astype(np.float32)
    xo = (rng.random((16, 10)) * 15).astype(np.float32)
    fc = spyker.FC(40, 10)
    fc.kernel.copy_(cuda(w))
    fc.bpconfig = spyker.BPConfig(1.0, 0.01, 0.1, 0.001)
    nxt = fc.backward(cuda(xi), cuda(xo), cuda(g))
    k, n, sf = port.fcbackward(w, xi, xo, g, (1.0, 0.01, 0.1, 0.001))
    assert np.array_equal(host(fc.kernel), k)
    assert np.array_equal(host(nxt), n)
    assert abs(fc.bpconfig.sfactor - sf) <= 1e-6 * max(1.0, abs(sf))


def test_golden_pipeline_ops(golden):
    """Each GPU op on the reference's own intermediate results."""
    dog = spyker.DoG(3, [spyker.DoGFilter(1, 2), spyker.DoGFilter(2, 1)], pad=3)
    img = cuda(golden["images"][:, None].astype(np.float32) / np.float32(255))
    d = dog(img)
    assert np.array_equal(host(d), golden["dog"])
    c = spyker.code(d, 15, sort=False)
    assert np.array_equal(host(c), golden["codes_latency"])
    spk = cuda(golden["fire"])
    w = spyker.convwta(spk, 3, 5)
    assert spyker.pool(spk, 2).cpu().numpy().tobytes() == golden["pooled"].tobytes()
    assert np.array_equal(host(spyker.gather(spk)), golden["gather"])
    conv = spyker.Conv(2, 30, 5, pad=2)
    conv.kernel.copy_(cuda(golden["kernel"]))
    conv.stdpconfig = [spyker.STDPConfig(0.004, -0.003)]
    rec = [[spyker.Winner(*golden["winners"][i, j]) for j in range(golden["counts"][i])]
           for i in range(len(golden["counts"]))]
    conv.stdp(cuda(golden["codes"]), rec, spk)
    assert np.array_equal(host(conv.kernel), golden["stdp_kernel"])
    assert len(w) == 16


def test_end_to_end_layer(port, golden):
    """DoG -> code -> conv -> threshold -> inhibit -> WTA -> fire -> STDP on
    the GPU (FP32 conv) against the reference's results for the same images."""
    img = cuda(golden["images"][:, None].astype(np.float32) / np.float32(255))
    dog = spyker.DoG(3, [spyker.DoGFilter(1, 2), spyker.DoGFilter(2, 1)], pad=3)
    codes = spyker.code(dog(img), 15)
    code_match = (host(codes) == golden["codes"]).mean()
    assert code_match > 0.9999
    conv = spyker.Conv(2, 30, 5, pad=2)
    conv.kernel.copy_(cuda(golden["kernel"]))
    conv.stdpconfig = [spyker.STDPConfig(0.004, -0.003)]
    codes = cuda(golden["codes"])
    pot = conv(codes)
    out = spyker.inhibit(spyker.threshold(pot, 15.0))
    spk = spyker.fire(out)
    spike_match = (host(spk) == golden["fire"]).mean()
    assert spike_match > 0.999
    wins = spyker.convwta(out, 3, 5)
    conv.stdp(codes, wins, spk)
    if spike_match == 1.0:
        rec, cnt = winners_np(wins)
        assert np.array_equal(cnt, golden["counts"])


# ---------------------------------------------------------------------------
# tcgen05 BF16-split convolution
# ---------------------------------------------------------------------------

def _tc_case(port, seed, n, t, cin, h, w, cout, k, stride, pad, lo=0.5, hi=1.0):
    rng = np.random.default_rng(seed)
    fst = rng.integers(0, t + 3, size=(n, cin, h, w))
    spikes = (fst[:, None] <= np.arange(t)[None, :, None, None, None]).astype(np.uint8)
    wts = rng.uniform(lo, hi, size=(cout, cin, k, k)).astype(np.float32)
    exact = port.conv(spikes, wts, stride, pad, out_dtype=np.float32)
    ref64 = port.conv(spikes, wts.astype(np.float64), stride, pad, out_dtype=np.float64)
    return spikes, wts, exact, ref64


TC_SHAPES = [
    # n, t, cin, h, w, cout, k, stride, pad
    (4, 15, 2, 28, 28, 30, 5, (1, 1), (2, 2, 2, 2)),
    (3, 15, 30, 14, 14, 100, 5, (1, 1), (2, 2, 2, 2)),
    (2, 5, 7, 19, 23, 37, 3, (2, 1), (1, 0, 2, 3)),
    (1, 4, 16, 12, 12, 256, 5, (1, 1), (2, 2, 2, 2)),
]


@pytest.mark.parametrize("shape_", TC_SHAPES)
def test_conv_tc_bf16x3_exact(port, shape_):
    n, t, cin, h, w, cout, k, stride, pad = shape_
    spikes, wts, exact, _ = _tc_case(port, 17, n, t, cin, h, w, cout, k, stride, pad)
    spyker._lib.lib.spk_device_status(1)
    got = host(spyker.conv(cuda(spikes), cuda(wts), stride, pad, precision="bf16x3"))
    assert spyker._lib.lib.spk_device_status(1) == 0
    assert got.shape == exact.shape
    assert np.array_equal(got, exact), f"{int((got != exact).sum())} of {got.size} potentials differ"


@pytest.mark.parametrize("shape_", TC_SHAPES[:3])
def test_conv_tc_bf16x2_tolerance(port, shape_):
    n, t, cin, h, w, cout, k, stride, pad = shape_
    spikes, wts, _, ref64 = _tc_case(port, 23, n, t, cin, h, w, cout, k, stride, pad, lo=0.0, hi=1.0)
    got = host(spyker.conv(cuda(spikes), cuda(wts), stride, pad, precision="bf16x2"))
    rel = np.abs(got - ref64) / np.maximum(np.abs(ref64), 1e-30)
    assert rel.max() <= 1e-5
    assert spyker._lib.lib.spk_device_status(1) == 0


def test_conv_tc_small_weights_tolerance(port):
    # weights spanning eight decades: partial sums are no longer exact, but
    # the potentials stay within the 1e-5 relative bound of the FP64 oracle
    spikes, _, _, _ = _tc_case(port, 5, 2, 15, 30, 14, 14, 100, 5, (1, 1), (2, 2, 2, 2))
    rng = np.random.default_rng(6)
    wts = (10.0 ** rng.uniform(-8, 0, size=(100, 30, 5, 5))).astype(np.float32)
    ref64 = port.conv(spikes, wts.astype(np.float64), (1, 1), (2, 2, 2, 2), out_dtype=np.float64)
    got = host(spyker.conv(cuda(spikes), cuda(wts), 1, 2, precision="bf16x3"))
    rel = np.abs(got - ref64) / np.maximum(np.abs(ref64), 1e-30)
    assert rel.max() <= 1e-5


def test_end_to_end_layer_bf16x3(golden):
    """With the exact tensor-core conv the whole layer matches the reference."""
    codes = cuda(golden["codes"])
    conv = spyker.Conv(2, 30, 5, pad=2)
    conv.kernel.copy_(cuda(golden["kernel"]))
    conv.stdpconfig = [spyker.STDPConfig(0.004, -0.003)]
    conv.precision = "bf16x3"
    out = spyker.inhibit(spyker.threshold(conv(codes), 15.0))
    spk = spyker.fire(out)
    assert np.array_equal(host(spk), golden["fire"])
    wins = spyker.convwta(out, 3, 5)
    rec, cnt = winners_np(wins)
    assert np.array_equal(cnt, golden["counts"])
    assert np.array_equal(rec, oracle_winners(golden["winners"], golden["counts"])[0])
    conv.stdp(codes, wins, spk)
    assert np.array_equal(host(conv.kernel), golden["stdp_kernel"])
    assert np.array_equal(host(spyker.pool(spk, 2)), golden["pooled"])


# ---------------------------------------------------------------------------
# fused layer: conv -> threshold -> inhibit -> fire + convwta in one kernel
# ---------------------------------------------------------------------------

FUSED = [
    # b, t, cin, h, w, cout, k, pad, theta, radius, count
    (16, 15, 2, 28, 28, 30, 5, 2, 15.0, 3, 5),
    (12, 15, 30, 14, 14, 100, 5, 2, 10.0, 1, 8),
    (3, 30, 8, 21, 19, 64, 7, 3, 20.0, 2, 6),
    (7, 5, 3, 9, 11, 17, 3, 1, 2.5, 0, 40),
    (5, 32, 4, 10, 10, 20, 3, 1, 3.0, 1, 4),
    (6, 3, 9, 8, 9, 16, 3, 1, 4.0, 1, 3),
    (4, 2, 2, 12, 12, 8, 5, 2, 3.0, 2, 5),
    (4, 1, 5, 7, 6, 12, 3, 0, 2.0, 1, 2),
    (2, 6, 64, 32, 32, 32, 3, 1, 120.0, 1, 4),  # first-spike staging in two pixel runs
    (2, 30, 64, 12, 12, 256, 5, 2, 600.0, 1, 4),  # the large-image conv2 shape: channels in two parts
    (3, 15, 16, 10, 9, 200, 3, 1, 40.0, 2, 6),  # 200 channels: two parts with padding
]


@pytest.mark.parametrize("case", FUSED)
@pytest.mark.parametrize("prec", ["bf16x3", "bf16x2"])
def test_fused_layer_matches_ops(port, case, prec):
    b, t, cin, h, w, cout, k, pad, theta, radius, count = case
    rng = np.random.default_rng(b * 7 + t)
    fst = rng.integers(0, t + 4, size=(b, cin, h, w))
    x = cuda((fst[:, None] <= np.arange(t)[None, :, None, None, None]).astype(np.uint8))
    conv = spyker.Conv(cin, cout, k, pad=pad)
    conv.kernel.copy_(cuda(rng.uniform(0.3, 1.0, size=(cout, cin, k, k)).astype(np.float32)))
    conv.precision = prec
    spikes, wins = spyker.conv_fire_wta(x, conv, theta, radius, count)
    assert spyker._lib.lib.spk_device_status(1) == 0
    # against the oracle's FP64 pipeline (the layer's decisions are exact)
    inh = port.inhibit(port.threshold(port.conv(host(x), host(conv.kernel), (1, 1), (pad,) * 4), theta))
    assert np.array_equal(host(spikes), port.fire(inh))
    got = winners_np(wins)
    win, cnt = oracle_winners(*port.convwta(inh, (radius, radius), count))
    assert np.array_equal(got[1], cnt) and np.array_equal(got[0], win)
    assert int(got[1].sum()) > 0


@pytest.mark.parametrize("cout", [20, 256])
@pytest.mark.parametrize("kind", ["negative_weights", "value_above_threshold"])
def test_fused_layer_general_argmax(kind, cout):
    """Negative weights, or a threshold value above the threshold, take the
    epilogue's general argmax (the lean one needs neither); results equal
    the op-by-op pipeline.  At 256 channels the three-term accumulators do
    not fit the tensor memory and the dense kernel runs with two terms."""
    b, t, cin, h, w = 6, 15, 4, 12, 11
    rng = np.random.default_rng(11 if kind == "negative_weights" else 12)
    fst = rng.integers(0, t + 4, size=(b, cin, h, w))
    x = cuda((fst[:, None] <= np.arange(t)[None, :, None, None, None]).astype(np.uint8))
    lo = -0.5 if kind == "negative_weights" else 0.3
    conv = spyker.Conv(cin, cout, 3, pad=1)
    conv.kernel.copy_(cuda(rng.uniform(lo, 1.0, size=(cout, cin, 3, 3)).astype(np.float32)))
    conv.precision = "bf16x3"
    theta, value = (2.0, 0.0) if kind == "negative_weights" else (6.0, 7.5)
    spikes, wins = spyker.conv_fire_wta(x, conv, theta, 1, 4, value=value)
    out = spyker.inhibit(spyker.threshold(conv(x), theta, value))
    assert np.array_equal(host(spikes), host(spyker.fire(out)))
    got, want = winners_np(wins), winners_np(spyker.convwta(out, 1, 4))
    assert np.array_equal(got[1], want[1]) and np.array_equal(got[0], want[0])
    assert int(host(spikes).sum()) > 0
    assert spyker._lib.lib.spk_device_status(1) == 0


@pytest.mark.parametrize("case", [FUSED[0], FUSED[1], FUSED[4]])
def test_fused_layer_schedules_do_not_change_results(case):
    """Pipeline stages, accumulators and CTAs per SM change the speed only."""
    b, t, cin, h, w, cout, k, pad, theta, radius, count = case
    rng = np.random.default_rng(b * 3 + t)
    fst = rng.integers(0, t + 4, size=(b, cin, h, w))
    x = cuda((fst[:, None] <= np.arange(t)[None, :, None, None, None]).astype(np.uint8))
    conv = spyker.Conv(cin, cout, k, pad=pad)
    conv.kernel.copy_(cuda(rng.uniform(0.3, 1.0, size=(cout, cin, k, k)).astype(np.float32)))
    conv.precision = "bf16x3"
    base = spyker.conv_fire_wta(x, conv, theta, radius, count, pool=2)
    try:
        for st in [(3, 1, 0), (2, 0, 1), (6, 0, 0), (0, 1, 2)]:
            spyker._lib.call("spk_set_conv_schedule", *st)
            got = spyker.conv_fire_wta(x, conv, theta, radius, count, pool=2)
            assert torch.equal(got[0], base[0]) and torch.equal(got[2], base[2]), st
            assert np.array_equal(winners_np(got[1])[0], winners_np(base[1])[0]), st
            assert np.array_equal(winners_np(got[1])[1], winners_np(base[1])[1]), st
    finally:
        spyker._lib.call("spk_set_conv_schedule", 0, 0, 0)
    assert spyker._lib.lib.spk_device_status(1) == 0


@pytest.mark.parametrize("case", [((6, 15, 2, 28, 28, 30, 5, 2), (2, 2)), ((5, 15, 30, 14, 14, 100, 5, 2), (14, 14)),
                                  ((4, 9, 3, 13, 11, 12, 3, 1), (3, 2))])
def test_fused_layer_pooled(case):
    """The pooled spikes written by the fused kernel equal pool(spikes)."""
    (b, t, cin, h, w, cout, k, pad), p = case
    rng = np.random.default_rng(b + t)
    fst = rng.integers(0, t + 3, size=(b, cin, h, w))
    x = cuda((fst[:, None] <= np.arange(t)[None, :, None, None, None]).astype(np.uint8))
    conv = spyker.Conv(cin, cout, k, pad=pad)
    conv.kernel.copy_(cuda(rng.uniform(0.3, 1.0, size=(cout, cin, k, k)).astype(np.float32)))
    conv.precision = "bf16x3"
    theta = 0.4 * cin * k * k * 0.65
    spikes, wins, pooled = spyker.conv_fire_wta(x, conv, theta, 1, 3, pool=p)
    assert int(host(spikes).sum()) > 0
    assert np.array_equal(host(pooled), host(spyker.pool(spikes, p)))
    s2, w2 = spyker.conv_fire_wta(x, conv, theta, 1, 3)
    assert np.array_equal(host(s2), host(spikes))


def test_gabor_forward_pipeline(port):
    """The large-image forward pipeline at a reduced size: Gabor bank (4
    orientations x 2 wavelengths, 11x11) -> rank code T=30 -> conv1 64x7x7
    th20 fused with inhibition and pool 2 (no winner selection) -> conv2
    256x5x5 th12 (op by op: 3 x 256 accumulator columns exceed tensor
    memory) -> pool 2, against the oracle's FP64 pipeline on the same codes."""
    imgs = synth.textures(1, seed=5, size=32)
    filters = [spyker.GaborFilter(2.5, th, 0.5, lam, 0.0) for th in (0, 45, 90, 135) for lam in (5.0, 10.0)]
    gab = spyker.Gabor(5, filters, pad=5)
    g = gab(cuda(imgs[:, None]))
    assert np.array_equal(host(g), port.filter("gabor", imgs[:, None], host(gab.kernel), (5, 5, 5, 5)))
    codes = spyker.code(g, 30)
    assert np.array_equal(host(codes), stable_code(host(g), 30))
    w1 = synth.conv_weights(64, 8, 7, seed=11)
    w2 = synth.conv_weights(256, 64, 5, seed=12)
    c1, c2 = spyker.Conv(8, 64, 7, pad=3), spyker.Conv(64, 256, 5, pad=2)
    c1.kernel.copy_(cuda(w1)), c2.kernel.copy_(cuda(w2))
    c1.precision = c2.precision = "bf16x3"
    s1, none, p1 = spyker.conv_fire_wta(codes, c1, 20.0, 0, 0, pool=2)
    assert none is None
    s2, _, p2 = spyker.conv_fire_wta(p1, c2, 12.0, 0, 0, pool=2)
    hc = host(codes)
    r1 = port.fire(port.inhibit(port.threshold(port.conv(hc, w1, (1, 1), (3, 3, 3, 3)), 20.0)))
    assert np.array_equal(host(s1), r1)
    q1 = port.pool(r1, (2, 2))
    assert np.array_equal(host(p1), q1)
    r2 = port.fire(port.inhibit(port.threshold(port.conv(q1, w2, (1, 1), (2, 2, 2, 2)), 12.0)))
    assert np.array_equal(host(s2), r2)
    assert np.array_equal(host(p2), port.pool(r2, (2, 2)))
    assert int(r2.sum()) > 0


@pytest.mark.parametrize("kind", ["random", "values"])
def test_fused_layer_noncumulative(kind):
    """Inputs that are not cumulative 0/1 spikes take the producers' direct
    gather; results still equal the op-by-op pipeline."""
    rng = np.random.default_rng(5 if kind == "random" else 6)
    b, t, cin, h, w, cout = 6, 7, 10, 9, 8, 24
    x = (rng.random((b, t, cin, h, w)) < 0.3).astype(np.uint8)
    if kind == "values":
        x = np.cumsum(x, axis=1).clip(0, 3).astype(np.uint8)  # monotone but not 0/1
    x = cuda(x)
    conv = spyker.Conv(cin, cout, 3, pad=1)
    conv.kernel.copy_(cuda(rng.uniform(0.3, 1.0, size=(cout, cin, 3, 3)).astype(np.float32)))
    conv.precision = "bf16x3"
    spikes, wins = spyker.conv_fire_wta(x, conv, 3.0, 1, 4)
    out = spyker.inhibit(spyker.threshold(conv(x), 3.0))
    assert np.array_equal(host(spikes), host(spyker.fire(out)))
    got, want = winners_np(wins), winners_np(spyker.convwta(out, 1, 4))
    assert np.array_equal(got[1], want[1]) and np.array_equal(got[0], want[0])
    assert spyker._lib.lib.spk_device_status(1) == 0


def test_fused_layer_golden(golden):
    conv = spyker.Conv(2, 30, 5, pad=2)
    conv.kernel.copy_(cuda(golden["kernel"]))
    conv.precision = "bf16x3"
    spikes, wins = spyker.conv_fire_wta(cuda(golden["codes"]), conv, 15.0, 3, 5)
    assert np.array_equal(host(spikes), golden["fire"])
    rec, cnt = winners_np(wins)
    assert np.array_equal(cnt, golden["counts"])
    assert np.array_equal(rec, oracle_winners(golden["winners"], golden["counts"])[0])
