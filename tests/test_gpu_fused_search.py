"""The fused layer's first-crossing search (non-negative weights, cumulative
0/1 spikes) against the oracle's FP64 pipeline, in the regimes where its
decisions are hardest: weights at the bounds STDP drives them to, exact
ties of a potential with the threshold and between channels, weights far
below the largest of their channel, and weights reached by real STDP
training.  Spikes, pooled spikes, winner records and counts are compared
bit for bit; the oracle's potential is the F32 rounding of the FP64 sum of
the products in (channel, ky, kx) order."""

import numpy as np
import pytest
import torch

import spyker_b200 as spyker
from spyker_b200 import synth
from tests.golden import make_golden

pytestmark = pytest.mark.gpu


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def host(t):
    return t.cpu().numpy()


def winners_np(w):
    rec, cnt = host(w.records).astype(np.int64), host(w.counts).astype(np.int64)
    for i in range(rec.shape[0]):
        rec[i, cnt[i]:] = 0
    return rec, cnt


def cumulative(rng, b, t, c, h, w, never=4):
    fst = rng.integers(0, t + never, size=(b, c, h, w))
    return (fst[:, None] <= np.arange(t)[None, :, None, None, None]).astype(np.uint8)


def check(port, x, w, theta, radius, count, pad, pool=2, prec="bf16x3"):
    """Fused layer (spikes, winners, pooled) == the oracle's pipeline; returns
    the oracle's spike count and the rows re-decided exactly / recomputed."""
    cout, cin, k, _ = w.shape
    conv = spyker.Conv(cin, cout, k, pad=pad)
    conv.kernel.copy_(cuda(w))
    conv.precision = prec
    spyker._lib.lib.spk_recheck_count(1)
    spyker._lib.lib.spk_recompute_count(1)
    spk, wins, pooled = spyker.conv_fire_wta(cuda(x), conv, theta, radius, count, pool=pool)
    assert spyker._lib.lib.spk_device_status(1) == 0
    inh = port.inhibit(port.threshold(port.conv(x, w, (1, 1), (pad,) * 4), theta))
    ref = port.fire(inh)
    got = host(spk)
    assert np.array_equal(got, ref), f"{int((got != ref).sum())} spikes differ"
    assert np.array_equal(host(pooled), port.pool(ref, (pool, pool)))
    win, cnt = port.convwta(inh, (radius, radius), count)
    rec, gcnt = winners_np(wins)
    assert np.array_equal(gcnt, cnt)
    for i in range(win.shape[0]):
        win[i, cnt[i]:] = 0
    assert np.array_equal(rec, win)
    return int(ref.sum()), spyker._lib.lib.spk_recheck_count(1), spyker._lib.lib.spk_recompute_count(1)


LAYERS = [
    # b, t, cin, h, w, cout, k, pad, theta, radius, count
    (12, 15, 2, 28, 28, 30, 5, 2, 15.0, 3, 5),
    (10, 15, 30, 14, 14, 100, 5, 2, 10.0, 1, 8),
]


def weights(kind, rng, shape):
    if kind == "binary":  # STDP's end points: exactly 0 or 1
        return (rng.random(shape) < 0.5).astype(np.float32)
    if kind == "near_one":  # 1, 1 - 2^-20 and 0
        return rng.choice(np.array([0.0, 1.0 - 2.0 ** -20, 1.0], np.float32), size=shape)
    if kind == "tiny":  # 1 beside weights far below it, subnormals included
        vals = np.array([1.0, 1.0, 0.5, 1e-10, 2.0 ** -30, 1e-38, 3e-45, 0.0, 2.0 ** -24, 3.0e-8], np.float32)
        return rng.choice(vals, size=shape)
    if kind == "log_uniform":  # weights in transition, 2^-30 .. 1
        return np.exp2(rng.uniform(-30, 0, size=shape)).astype(np.float32)
    if kind == "halves":  # multiples of 1/2: potentials land on the threshold exactly
        return (rng.integers(0, 3, size=shape) * 0.5).astype(np.float32)
    raise ValueError(kind)


@pytest.mark.parametrize("layer", LAYERS)
@pytest.mark.parametrize("kind", ["binary", "near_one", "tiny", "log_uniform", "halves"])
def test_search_saturated_weights(port, layer, kind):
    b, t, cin, h, wd, cout, k, pad, theta, radius, count = layer
    rng = np.random.default_rng(sum(map(ord, kind)) + cin)
    x = cumulative(rng, b, t, cin, h, wd)
    w = weights(kind, rng, (cout, cin, k, k))
    # a threshold the potentials reach exactly (a half-integer near the median)
    th = float(np.round(np.median(port.conv(x[:, -1:], w, (1, 1), (pad,) * 4)) * 2) / 2)
    spikes, _, _ = check(port, x, w, max(th, 1.0), radius, count, pad)
    assert spikes > 0


@pytest.mark.parametrize("layer", LAYERS)
def test_search_channel_ties(port, layer):
    """Channels with identical weights tie exactly at every step: the first
    of them wins (cpu/inhibit.cpp's first max)."""
    b, t, cin, h, wd, cout, k, pad, theta, radius, count = layer
    rng = np.random.default_rng(3)
    x = cumulative(rng, b, t, cin, h, wd)
    w = rng.uniform(0.3, 1.0, size=(cout, cin, k, k)).astype(np.float32)
    w[1::2] = w[0::2][: w[1::2].shape[0]]
    w[cout - 3] = w[2]
    assert check(port, x, w, theta, radius, count, pad)[0] > 0


def test_search_potentials_at_threshold(port):
    """All weights 1 (a third of the maps see one channel only): every
    potential is an input count, so at integer thresholds many rows sit
    exactly on them and must not fire."""
    rng = np.random.default_rng(9)
    x = cumulative(rng, 8, 15, 2, 28, 28)
    w = np.ones((30, 2, 5, 5), np.float32)
    w[::3, 1] = 0.0
    for theta in (10.0, 15.0, 22.0):
        check(port, x, w, theta, 3, 5, 2)


@pytest.fixture(scope="module")
def trained(port):
    """Weights after 30 real STDP steps of the 2-layer network (96 stroke
    images a step, large learning rates) on the GPU: many at 1, many decayed
    towards 0, some in between."""
    img = synth.strokes(96, seed=41).astype(np.float32) / 255
    dog = spyker.DoG(3, [spyker.DoGFilter(1, 2), spyker.DoGFilter(2, 1)], pad=3)
    codes = spyker.code(dog(cuda(img[:, None])), 15)
    c1, c2 = spyker.Conv(2, 30, 5, pad=2), spyker.Conv(30, 100, 5, pad=2)
    c1.kernel.copy_(cuda(synth.conv_weights(30, 2, 5, seed=1)))
    c2.kernel.copy_(cuda(synth.conv_weights(100, 30, 5, seed=2)))
    for c in (c1, c2):
        c.stdpconfig = [spyker.STDPConfig(0.05, -0.04)]
        c.precision = "bf16x3"
    for _ in range(30):
        s1, w1, p1 = spyker.conv_fire_wta(codes, c1, 15.0, 3, 5, pool=2)
        c1.stdp(codes, w1, s1)
        s2, w2, _ = spyker.conv_fire_wta(p1, c2, 10.0, 1, 8, pool=2)
        c2.stdp(p1, w2, s2)
    return host(c1.kernel), host(c2.kernel), host(codes)


def test_search_trained_weights(port, trained):
    w1, w2, codes = trained
    assert (w1 > 0.999).mean() > 0.05 and (w1 < 1e-3).mean() > 0.05
    spk1 = port.fire(port.inhibit(port.threshold(port.conv(codes, w1, (1, 1), (2,) * 4), 15.0)))
    n1, _, _ = check(port, codes, w1, 15.0, 3, 5, 2)
    n2, _, _ = check(port, port.pool(spk1, (2, 2)), w2, 10.0, 1, 8, 2, pool=7)
    assert n1 > 0 and n2 > 0


def test_search_trained_weights_fresh_images(port, trained):
    w1, _, _ = trained
    img = synth.strokes(24, seed=77).astype(np.float32) / 255
    d = port.filter("dog", img[:, None], make_golden.dog_kernel(port), (3, 3, 3, 3))
    codes = port.rank_code(d, 15)
    assert check(port, codes, w1, 15.0, 3, 5, 2)[0] > 0


@pytest.mark.parametrize("kind", ["binary", "halves", "log_uniform"])
def test_search_channel_parts(port, kind):
    """256 output channels: the search runs the channels in two parts per
    tile and merges the parts' maxima; ties and saturated weights across the
    part boundary still resolve as the oracle does (first channel wins)."""
    rng = np.random.default_rng(sum(map(ord, kind)) + 256)
    b, t, cin, h, wd, cout, k, pad = 2, 15, 16, 10, 10, 256, 3, 1
    x = cumulative(rng, b, t, cin, h, wd)
    w = weights(kind, rng, (cout, cin, k, k))
    w[200:] = w[:56]  # channels 200.. tie exactly with channels 0..55 (other part)
    th = float(np.round(np.median(port.conv(x[:, -1:], w, (1, 1), (pad,) * 4)) * 2) / 2)
    assert check(port, x, w, max(th, 1.0), 1, 4, pad)[0] > 0


@pytest.mark.parametrize("side", [136, 132])
def test_search_large_maps(port, side):
    """Maps above 16384 output pixels (per-pixel codes in global memory, no
    WTA): 136 x 136 takes the multi-CTA writer (pooled width a multiple of
    4), 132 x 132 the per-sample one; spikes and pooled spikes equal the
    oracle's pipeline."""
    rng = np.random.default_rng(side)
    x = cumulative(rng, 2, 6, 2, side, side)
    w = rng.uniform(0.3, 1.0, size=(8, 2, 3, 3)).astype(np.float32)
    conv = spyker.Conv(2, 8, 3, pad=1)
    conv.kernel.copy_(cuda(w))
    conv.precision = "bf16x3"
    spk, wins, pooled = spyker.conv_fire_wta(cuda(x), conv, 4.0, 0, 0, pool=2)
    assert wins is None and spyker._lib.lib.spk_device_status(1) == 0
    ref = port.fire(port.inhibit(port.threshold(port.conv(x, w, (1, 1), (1, 1, 1, 1)), 4.0)))
    assert np.array_equal(host(spk), ref) and int(ref.sum()) > 0
    assert np.array_equal(host(pooled), port.pool(ref, (2, 2)))


def test_search_long_lists():
    """More than 2048 x 2048 output pixels in one call: the list compactions
    take the three-launch form (per-block counts, one-block scan, scatter);
    the result equals the two halves of the batch run separately (each on
    the one-launch form; samples are independent without WTA)."""
    rng = np.random.default_rng(5)
    b, side = 66, 256  # 66 * 256 * 256 = 4.33M output pixels
    x = cumulative(rng, b, 4, 2, side, side)
    w = rng.uniform(0.3, 1.0, size=(8, 2, 3, 3)).astype(np.float32)
    conv = spyker.Conv(2, 8, 3, pad=1)
    conv.kernel.copy_(cuda(w))
    conv.precision = "bf16x3"
    xd = cuda(x)
    spk, _, pooled = spyker.conv_fire_wta(xd, conv, 4.0, 0, 0, pool=2)
    assert spyker._lib.lib.spk_device_status(1) == 0
    for lo, hi in ((0, b // 2), (b // 2, b)):
        s_h, _, p_h = spyker.conv_fire_wta(xd[lo:hi].contiguous(), conv, 4.0, 0, 0, pool=2)
        assert torch.equal(spk[lo:hi], s_h) and torch.equal(pooled[lo:hi], p_h)
    assert int(spk[:, -1].sum()) > 0
