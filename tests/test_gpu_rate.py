"""Rate (Poisson) coding on the GPU against the reference's CPU backend
(oracle/_ref): fire, gather and pool bit for bit; the code in distribution
(its draws come from another generator) and in structure."""

import numpy as np
import pytest
import torch

import spyker_b200 as spyker
from spyker_b200 import synth
from tests.golden import make_golden

pytestmark = pytest.mark.gpu
DEV = "cuda"


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def host(t):
    return t.cpu().numpy()


@pytest.mark.parametrize("dtype", ["u8", "f32"])
def test_rate_fire_and_gather(ref, dtype):
    rng = np.random.default_rng(1)
    pot = np.cumsum(rng.random((4, 12, 3, 7, 6)).astype(np.float32), axis=1)
    npt = {"u8": np.uint8, "f32": np.float32}[dtype]
    got = spyker.fire(cuda(pot), 0.35, dtype=dtype, code="rate")
    want = ref.rate_fire(pot, 0.35, npt)
    assert np.array_equal(host(got), want)
    assert want.max() > 1
    g = spyker.gather(got, dtype=dtype, code="rate")
    assert np.array_equal(host(g), ref.rate_gather(want, npt))


@pytest.mark.parametrize("geo", [((2, 2), None), ((3, 3), (2, 2)), ((2, 3), (1, 2))])
def test_rate_pool(ref, geo):
    k, st = geo
    rng = np.random.default_rng(2)
    counts = np.cumsum(rng.integers(0, 2, size=(3, 8, 4, 9, 10)), axis=1).astype(np.uint8)
    rates = rng.integers(0, 3, size=(3, 4, 9, 10)).astype(np.float32)  # many ties
    got = spyker.pool(cuda(counts), k, st, rates=cuda(rates))
    assert np.array_equal(host(got), ref.rate_pool(counts, rates, k, st or k))


def test_rate_code_structure_and_seed():
    img = synth.strokes(16, seed=3).astype(np.float32)[:, None] / 255
    x = cuda(img)
    spyker.random_seed(7)
    a = host(spyker.code(x, 20, code="rate"))
    spyker.random_seed(7)
    b = host(spyker.code(x, 20, code="rate"))
    assert np.array_equal(a, b)  # reproducible after a seed
    c = host(spyker.code(x, 20, code="rate"))
    assert not np.array_equal(a, c)  # the next call draws new intervals
    d = np.diff(a.astype(np.int32), axis=1)
    assert d.min() >= 0 and d.max() <= 1  # running counts, at most one spike per step
    times = host(spyker.gather(spyker.code(x, 20), 0.0, dtype="u8"))  # rank times
    silent = times >= 20
    assert (a[:, -1][silent] == 0).all()  # positions without a rank spike never fire
    assert a[:, -1][~silent].mean() > 0.5


@pytest.mark.parametrize("sort", [False, True])
def test_rate_code_distribution_matches_reference(ref, port, sort):
    """Mean final count per rank / latency time against the reference's
    code over the same images (64 images x 1568 positions).  Positions whose
    time is T have no table row: the reference reads past its table there,
    the library never fires them; they are left out."""
    imgs = synth.strokes(64, seed=11).astype(np.float32)[:, None] / 255
    dog = port.filter("dog", imgs, make_golden.dog_kernel(port), (3, 3, 3, 3))
    t = 15
    got = host(spyker.code(cuda(dog), t, sort=sort, code="rate")).astype(np.float64)
    want = ref.rate_code(dog, t, sort=sort).astype(np.float64)
    times = port.gather(port.rank_code(dog, t, sort=sort), 0.0, np.uint8).reshape(64, -1)
    g, w = got[:, -1].reshape(64, -1), want[:, -1].reshape(64, -1)
    for r in range(t):
        m = times == r
        if m.sum() < 200:
            continue
        gm, wm = g[m].mean(), w[m].mean()
        se = np.sqrt(g[m].var() / m.sum() + w[m].var() / m.sum()) + 1e-9
        assert abs(gm - wm) <= 5 * se + 0.02, (r, gm, wm, se)
    live = times < t  # the reference reads past its table for silent positions
    assert abs(g[live].mean() - w[live].mean()) <= 0.02 * max(w[live].mean(), 1e-3) + 0.01
