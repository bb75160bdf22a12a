"""The CPU restatement (oracle port) is pinned to the reference.

1. Against the committed golden fixtures, which are outputs of the
   reference's own CPU backend compiled here (tests/golden/make_golden.py).
2. Call for call against that reference build on fresh seeded inputs and
   edge cases (when oracle/_ref is present).
"""

import numpy as np
import pytest

from spyker_b200 import synth
from tests.golden import make_golden


def _eq(a, b):
    if isinstance(a, tuple):
        assert len(a) == len(b)
        for x, y in zip(a, b):
            _eq(x, y)
        return
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape and a.dtype == b.dtype
    assert np.array_equal(a, b), f"{int((a != b).sum())} mismatches"


def test_port_reproduces_golden(port, golden):
    d = make_golden.run(port)
    assert set(d) == set(golden)
    for k in golden:
        _eq(d[k], golden[k])


def test_golden_is_nontrivial(golden):
    assert golden["counts"].sum() > 0
    assert golden["codes"].any() and not golden["codes"].all()
    assert not np.array_equal(golden["stdp_kernel"], golden["kernel"])
    assert golden["sp_conv_off"][-1] > 0


CFG = [(0.004, -0.003, 1.0, 0.0, 1.0)]


@pytest.fixture(scope="module")
def data(port):
    img = synth.strokes(24, seed=7).astype(np.float32) / 255
    k = make_golden.dog_kernel(port)
    dog = port.filter("dog", img[:, None], k, (3, 3, 3, 3))
    return dog


def test_filters_and_kernels(port, ref):
    _eq(port.gaussian_kernel(7, 1.3), ref.gaussian_kernel(7, 1.3))
    _eq(port.gabor_kernel(11, 2.5, 0.7, 0.5, 5.0, 0.2), ref.gabor_kernel(11, 2.5, 0.7, 0.5, 5.0, 0.2))
    _eq(port.log_kernel(9, 1.5), ref.log_kernel(9, 1.5))
    img = synth.strokes(4, seed=3).astype(np.float32)[:, None] / 255
    k = make_golden.dog_kernel(port)
    for which, pad in (("dog", (3, 3, 3, 3)), ("log", (1, 2, 3, 0))):
        _eq(port.filter(which, img, k, pad), ref.filter(which, img, k, pad))
    g = np.stack([port.gabor_kernel(11, 2.0, t, 0.5, 5.0, 0.0) for t in (0, 0.8, 1.6)]).astype(np.float32)
    _eq(port.filter("gabor", img, g, (5, 5, 5, 5)), ref.filter("gabor", img, g, (5, 5, 5, 5)))


@pytest.mark.parametrize("sort", [True, False])
def test_code(port, ref, data, sort):
    _eq(port.rank_code(data, 15, sort), ref.rank_code(data, 15, sort))
    u8 = (data * 200).astype(np.uint8)
    _eq(port.rank_code(u8, 9, sort), ref.rank_code(u8, 9, sort))


def test_code_edge_cases(port, ref):
    const = np.ones((3, 50), np.float32)
    _eq(port.rank_code(const, 15), ref.rank_code(const, 15))
    sparse = np.zeros((2, 100000), np.float32)
    sparse[:, 0] = 1.0  # cnt = 1: the time conversion wraps in the reference
    _eq(port.rank_code(sparse, 15), ref.rank_code(sparse, 15))
    ties = np.repeat(np.arange(8, dtype=np.float32), 50)[None].repeat(2, 0)
    _eq(port.rank_code(ties, 4), ref.rank_code(ties, 4))
    _eq(port.rank_code(np.zeros((1, 1), np.float32), 3), ref.rank_code(np.zeros((1, 1), np.float32), 3))


def test_layer_ops(port, ref, data):
    codes = port.rank_code(data, 15)
    w = synth.conv_weights(30, 2, 5, seed=2)
    pot = port.conv(codes, w, (1, 1), (2, 2, 2, 2))
    _eq(pot, ref.conv(codes.reshape(-1, 2, 28, 28).astype(np.float32), w, (1, 1), (2, 2, 2, 2)).reshape(pot.shape))
    _eq(port.threshold(pot, 15.0), ref.threshold(pot, 15.0))
    _eq(port.threshold(pot, 10.0, 3.0), ref.threshold(pot, 10.0, 3.0))
    th = port.threshold(pot, 15.0)
    _eq(port.inhibit(th), ref.inhibit(th))
    _eq(port.inhibit(pot, 25.0), ref.inhibit(pot, 25.0))
    inh = port.inhibit(th)
    for r, k in (((3, 3), 5), ((0, 1), 40), ((2, 0), 1)):
        _eq(port.convwta(inh, r, k), ref.convwta(inh, r, k))
    spk = port.fire(inh)
    _eq(spk, ref.fire(inh))
    _eq(port.convwta(spk, (1, 1), 8), ref.convwta(spk, (1, 1), 8))
    _eq(port.fire(pot, 30.0, np.float32), ref.fire(pot, 30.0, np.float32))
    _eq(port.pool(spk, (2, 2)), ref.pool(spk, (2, 2)))
    _eq(port.pool(inh, (3, 3), (2, 2), (1, 1, 1, 1)), ref.pool(inh, (3, 3), (2, 2), (1, 1, 1, 1)))
    _eq(port.gather(spk), ref.gather(spk))
    _eq(port.gather(pot, 20.0, np.float32), ref.gather(pot, 20.0, np.float32))
    g = port.gather(spk)
    _eq(port.scatter(g, 15), ref.scatter(g, 15))
    _eq(port.infinite(pot, 0.0), ref.infinite(pot, 0.0))
    _eq(port.pad(spk, (1, 2, 3, 4), 0), ref.pad(spk, (1, 2, 3, 4), 0))


def test_stdp(port, ref, data):
    codes = port.rank_code(data, 15)
    w = synth.conv_weights(30, 2, 5, seed=3)
    spk = port.fire(port.inhibit(port.threshold(port.conv(codes, w, (1, 1), (2, 2, 2, 2)), 15.0)))
    win, cnt = port.convwta(spk, (3, 3), 5)
    _eq(port.convstdp(codes, w, spk, CFG, win, cnt, (1, 1), (2, 2, 2, 2)),
        ref.convstdp(codes, w, spk, CFG, win, cnt, (1, 1), (2, 2, 2, 2)))
    # several configs, negative config index (skipped) and no stabilisation
    cfgs = CFG + [(0.01, -0.02, 0.0, 0.2, 0.9)]
    win2 = win.copy()
    win2[:, :, 0] = np.arange(win.shape[1])[None] % 3 - 1  # -1, 0, 1
    _eq(port.convstdp(codes, w, spk, cfgs, win2, cnt, (1, 1), (2, 2, 2, 2)),
        ref.convstdp(codes, w, spk, cfgs, win2, cnt, (1, 1), (2, 2, 2, 2)))
    # stride 2, asymmetric pad
    out2 = port.fire(port.conv(codes, w, (2, 2), (1, 2, 0, 1)), 20.0)
    wn, cn = port.convwta(out2, (1, 1), 4)
    _eq(port.convstdp(codes, w, out2, CFG, wn, cn, (2, 2), (1, 2, 0, 1)),
        ref.convstdp(codes, w, out2, CFG, wn, cn, (2, 2), (1, 2, 0, 1)))


def test_fc_and_backprop(port, ref):
    rng = np.random.default_rng(11)
    x = (rng.random((8, 15, 40)) * 3).astype(np.float32)
    w = rng.random((10, 40)).astype(np.float32)
    _eq(port.fcwta(x, 2, 3, 1.0), ref.fcwta(x, 2, 3, 1.0))
    _eq(port.fc(x, w), ref.fc(x, w))
    _eq(port.fc(x, w - 0.5, True), ref.fc(x, w - 0.5, True))
    si = (x > 1.5).astype(np.uint8)
    so = (port.fc(si, w, out_dtype=np.float32) > 5).astype(np.uint8)
    wn, cn = port.fcwta(so.astype(np.float32), 1, 2, 0.5)
    _eq(port.fcstdp(si, w, so, CFG, wn, cn), ref.fcstdp(si, w, so, CFG, wn, cn))
    t = (rng.random((16, 10)) * 20).astype(np.float32)
    tg = rng.integers(0, 10, 16)
    _eq(port.backward(t, tg, 15, 2.0), ref.backward(t, tg, 15, 2.0))
    _eq(port.labelize(x, 2.5), ref.labelize(x, 2.5))
    _eq(port.labelize(x, 100.0), ref.labelize(x, 100.0))
    g = rng.standard_normal((16, 10)).astype(np.float32)
    xi = (rng.random((16, 40)) * 15).astype(np.float32)
    xo = (rng.random((16, 10)) * 15).astype(np.float32)
    a = port.fcbackward(w - 0.5, xi, xo, g, (1.0, 0.01, 0.1, 0.001))
    b = ref.fcbackward(w - 0.5, xi, xo, g, (1.0, 0.01, 0.1, 0.001))
    _eq(a[0], b[0])
    _eq(a[1], b[1])
    assert a[2] == b[2]


def test_sparse(port, ref, data):
    shp = (data.shape[0], 15, 2, 28, 28)
    ev = port.sparse_code(data, 15)
    _eq(ev, ref.sparse_code(data, 15))
    _eq(port.sparse_code(data, 15, False), ref.sparse_code(data, 15, False))
    codes = port.rank_code(data, 15)
    _eq(port.sparse_from_dense(codes), ref.sparse_from_dense(codes))
    _eq(port.sparse_to_dense(ev, shp), ref.sparse_to_dense(ev, shp))
    _eq(port.sparse_gather(ev, shp), ref.sparse_gather(ev, shp))
    w = synth.conv_weights(30, 2, 5, seed=5)
    (o1, s1) = port.sparse_conv(ev, shp, w, 15.0, (2, 2, 2, 2))
    _eq(o1, ref.sparse_conv(ev, shp, w, 15.0, (2, 2, 2, 2))[0])
    ih = port.sparse_inhibit(o1, s1)
    _eq(ih, ref.sparse_inhibit(o1, s1))
    sw = port.sparse_convwta(ih, s1, (3, 3), 5)
    _eq(sw, ref.sparse_convwta(ih, s1, (3, 3), 5))
    _eq(port.sparse_stdp(ev, shp, w, CFG, *sw, (2, 2, 2, 2)), ref.sparse_stdp(ev, shp, w, CFG, *sw, (2, 2, 2, 2)))
    _eq(port.sparse_pool(o1, s1, (2, 2), (1, 1, 1, 1))[0], ref.sparse_pool(o1, s1, (2, 2), (1, 1, 1, 1))[0])
    _eq(port.sparse_pad(o1, s1, (1, 2, 1, 2))[0], ref.sparse_pad(o1, s1, (1, 2, 1, 2))[0])


def test_oracle_reports_errors(port):
    with pytest.raises(RuntimeError, match="configuration index"):
        x = np.zeros((1, 2, 1, 5, 5), np.uint8)
        o = np.zeros((1, 2, 1, 5, 5), np.uint8)
        w = np.zeros((1, 1, 1, 1), np.float32)
        port.convstdp(x, w, o, CFG, np.array([[[3, 0, 0, 0, 0]]]), np.array([1]))


def test_ties_and_boundaries(port, ref):
    """The survey's parity hazards on crafted inputs: values exactly at the
    threshold (threshold zeroes <=, fire is strict >), channels with equal
    potentials (inhibit keeps the first, cpu/inhibit.cpp:59), WTA keys tied
    across channels and positions (first index, cpu/wta.cpp:53-62,133),
    one time step, odd map sizes for pooling; an empty batch on the
    restatement (the reference build stops with a division by zero on
    one)."""
    rng = np.random.default_rng(21)
    b, t, c, h, w = 3, 6, 4, 9, 7
    base = rng.integers(0, 4, size=(b, t, 1, h, w)).astype(np.float32) * 2.5  # 0, 2.5, 5, 7.5
    pot = np.repeat(base, c, axis=2)  # every channel tied
    pot[:, :, 2] += (rng.random((b, t, h, w)) < 0.2) * 2.5  # some channel-2 wins
    pot = np.cumsum(pot, axis=1).astype(np.float32)  # monotone in t, as potentials are
    for thr in (5.0, 7.5, 10.0):
        _eq(port.threshold(pot, thr), ref.threshold(pot, thr))
        _eq(port.fire(pot, thr), ref.fire(pot, thr))
    th = port.threshold(pot, 5.0)
    _eq(port.inhibit(th), ref.inhibit(th))
    _eq(port.inhibit(th, 10.0), ref.inhibit(th, 10.0))
    for r, k in (((1, 1), 3), ((0, 0), 50), ((2, 3), 2)):
        _eq(port.convwta(th, r, k), ref.convwta(th, r, k))
        _eq(port.convwta(port.inhibit(th), r, k), ref.convwta(port.inhibit(th), r, k))
    spk = port.fire(port.inhibit(th))
    _eq(port.pool(spk, (2, 2)), ref.pool(spk, (2, 2)))
    _eq(port.pool(spk, (3, 2), (2, 2), (0, 1, 1, 0)), ref.pool(spk, (3, 2), (2, 2), (0, 1, 1, 0)))
    x = rng.random((4, 30)).astype(np.float32)
    _eq(port.rank_code(x, 1), ref.rank_code(x, 1))
    _eq(port.rank_code(x, 1, False), ref.rank_code(x, 1, False))
    empty = np.zeros((0, t, c, h, w), np.float32)
    assert port.threshold(empty, 1.0).shape == empty.shape and port.fire(empty, 1.0).shape == empty.shape
