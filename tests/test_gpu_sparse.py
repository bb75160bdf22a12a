"""Event-list path on the GPU against the oracle (sparse/*.cpp restated).

Every operation is compared exactly, event lists included in their order:
the inputs of each operation are the oracle's own lists, so an operation is
checked on its own, and the chain (code -> conv -> inhibit -> WTA -> STDP,
pool, pad) is checked end to end as well.
"""

import numpy as np
import pytest
import torch

import spyker_b200 as spyker
from spyker_b200 import synth
from tests.golden import make_golden
from tests.test_gpu_ops import stable_code

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)
CFG = [(0.004, -0.003, 1.0, 0.0, 1.0)]


def _eq_lists(got: spyker.SparseTensor, want):
    off, zyx = got.lists()
    woff, wzyx = want
    assert np.array_equal(off, np.asarray(woff, np.int64))
    assert np.array_equal(zyx, np.asarray(wzyx, np.uint8).reshape(-1, 3)), "event lists differ"


def _st(ev, shp):
    return spyker.SparseTensor.from_lists(ev[0], ev[1], shp, DEV)


@pytest.fixture(scope="module")
def dog(port):
    img = synth.strokes(24, seed=7).astype(np.float32) / 255
    return port.filter("dog", img[:, None], make_golden.dog_kernel(port), (3, 3, 3, 3))


@pytest.fixture(scope="module")
def chain(port, dog):
    shp = (dog.shape[0], 15, 2, 28, 28)
    ev = port.sparse_code(dog, 15)
    w = synth.conv_weights(30, 2, 5, seed=5)
    o1, s1 = port.sparse_conv(ev, shp, w, 15.0, (2, 2, 2, 2))
    ih = port.sparse_inhibit(o1, s1)
    return dict(shp=shp, ev=ev, w=w, o1=o1, s1=s1, ih=ih)


def test_code(port, dog):
    got = spyker.sparse.code(torch.from_numpy(dog).to(DEV), 15)
    assert got.shape == [dog.shape[0], 15, 2, 28, 28]
    # ties in index order, as the dense rank code of this library
    _eq_lists(got, port.sparse_from_dense(stable_code(dog, 15)))
    assert got.numel == port.sparse_code(dog, 15)[0][-1]
    lat = spyker.sparse.code(torch.from_numpy(dog).to(DEV), 15, sort=False)
    _eq_lists(lat, port.sparse_code(dog, 15, False))


def test_from_dense_dense_gather(port, dog, chain):
    codes = port.rank_code(dog, 15)
    st = spyker.SparseTensor(torch.from_numpy(codes).to(DEV))
    _eq_lists(st, port.sparse_from_dense(codes))
    pot = port.conv(codes, chain["w"], (1, 1), (2, 2, 2, 2))
    _eq_lists(spyker.SparseTensor(pot, 20.0), port.sparse_from_dense(pot, 20.0))
    shp = chain["shp"]
    ev = _st(chain["ev"], shp)
    assert np.array_equal(ev.dense().cpu().numpy(), port.sparse_to_dense(chain["ev"], shp))
    for dt, npt in (("u8", np.uint8), ("f32", np.float32), ("i32", np.int32)):
        got = spyker.sparse.gather(ev, dt).cpu().numpy()
        assert np.array_equal(got, port.sparse_gather(chain["ev"], shp, npt))
    assert abs(ev.sparsity() - chain["ev"][0][-1] / np.prod(shp)) < 1e-12
    assert np.array_equal(ev.copy().lists()[1], ev.lists()[1])


def test_conv_inhibit_wta_stdp(port, chain):
    shp, w = chain["shp"], chain["w"]
    ev = _st(chain["ev"], shp)
    o1 = spyker.sparse.conv(ev, torch.from_numpy(w).to(DEV), 15.0, 1, (2, 2, 2, 2))
    assert o1.shape == list(chain["s1"])
    _eq_lists(o1, chain["o1"])
    ih = spyker.sparse.inhibit(_st(chain["o1"], chain["s1"]))
    _eq_lists(ih, chain["ih"])
    win = spyker.sparse.convwta(_st(chain["ih"], chain["s1"]), 3, 5)
    want_w, want_c = port.sparse_convwta(chain["ih"], chain["s1"], (3, 3), 5)
    assert np.array_equal(win.counts.cpu().numpy(), want_c)
    assert np.array_equal(win.records.cpu().numpy().astype(np.int64), want_w)
    layer = spyker.Conv(2, 30, 5, pad=2)
    layer.kernel.copy_(torch.from_numpy(w))
    layer.stdpconfig = [spyker.STDPConfig(*CFG[0][:2])]
    layer.stdp(ev, win)
    want = port.sparse_stdp(chain["ev"], shp, w, CFG, want_w, want_c, (2, 2, 2, 2))
    assert not np.array_equal(want, w)
    assert np.array_equal(layer.kernel.cpu().numpy(), want)
    # the layer's sparse forward is Sparse::conv with its stride and pad
    _eq_lists(layer(ev, 15.0), port.sparse_conv(chain["ev"], shp, layer.kernel.cpu().numpy(), 15.0, (2, 2, 2, 2))[0])


def test_pool_pad(port, chain):
    o1 = _st(chain["o1"], chain["s1"])
    for k, p in (((2, 2), (1, 1, 1, 1)), ((3, 3), (0, 0, 0, 0)), ((2, 3), (0, 1, 2, 0))):
        got = spyker.sparse.pool(o1, k, None, p)
        _eq_lists(got, port.sparse_pool(chain["o1"], chain["s1"], k, p)[0])
    got = spyker.sparse.pad(o1, (1, 2, 1, 2))
    _eq_lists(got, port.sparse_pad(chain["o1"], chain["s1"], (1, 2, 1, 2))[0])
    assert got.shape == list(port.sparse_pad(chain["o1"], chain["s1"], (1, 2, 1, 2))[1])


def test_edges(port):
    # no events at all, long time axis, a single step
    zero = np.zeros((3, 40, 2, 9, 7), np.uint8)
    st = spyker.SparseTensor(zero)
    assert st.numel == 0
    w = synth.conv_weights(4, 2, 3, seed=1)
    out = spyker.sparse.conv(st, w, 0.5)
    assert out.numel == 0 and out.shape == [3, 40, 4, 7, 5]
    assert int(spyker.sparse.convwta(out, 1, 3).counts.sum()) == 0
    rng = np.random.default_rng(3)
    dense = (rng.random((2, 40, 3, 11, 13)) < 0.05).astype(np.uint8)
    ev = port.sparse_from_dense(dense)
    shp = dense.shape
    w3 = synth.conv_weights(5, 3, 3, seed=4) * 0.5
    _eq_lists(spyker.sparse.conv(_st(ev, shp), w3, 0.9, 1, 1), port.sparse_conv(ev, shp, w3, 0.9, (1, 1, 1, 1))[0])
    one = spyker.SparseTensor(dense[:, :1].copy())
    _eq_lists(one, port.sparse_from_dense(dense[:, :1].copy()))
    with pytest.raises(spyker.SpykerError, match="Stride must be 1"):
        spyker.sparse.conv(_st(ev, shp), w3, 0.9, 2)
    with pytest.raises(spyker.SpykerError, match="Stride must be equal to kernel"):
        spyker.sparse.pool(_st(ev, shp), 2, 1)
