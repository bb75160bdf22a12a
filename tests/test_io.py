"""Data IO on the host: the IDX (MNIST) reader against the reference's
Helper::mnistData / mnistLabel (helper/mnist.cpp, compiled in oracle/_ref) on
written files, truncated files, wrong magics and missing files; the CSV
reader against Helper::CSV (helper/csv.cpp) including its one-character
advance after a multi-character delimiter; the examples' `.npz` kernel
checkpoints and `to_tensor(...).to(kernel)` in-place load."""

import numpy as np
import pytest
import torch

import spyker_b200 as spyker
from spyker_b200 import io


def _idx_files(tmp_path, n=37, rows=28, cols=28):
    rng = np.random.default_rng(0)
    imgs = rng.integers(0, 256, size=(n, rows, cols), dtype=np.uint8)
    labels = rng.integers(0, 10, size=n, dtype=np.uint8)
    pi, pl = str(tmp_path / "images-idx3-ubyte"), str(tmp_path / "labels-idx1-ubyte")
    io.write_idx(pi, imgs)
    io.write_idx(pl, labels)
    return imgs, labels, pi, pl


def test_idx_matches_reference(ref, tmp_path):
    imgs, labels, pi, pl = _idx_files(tmp_path, n=37, rows=9, cols=13)
    trx, tr_y, tex, tey = spyker.read_mnist(pi, pl, pi, pl)
    want_x, want_y = ref.idx(pi, False), ref.idx(pl, True)
    assert want_x.shape == (37, 1, 9, 13) and want_y.shape == (37,)
    for got, want in ((trx, want_x), (tr_y, want_y), (tex, want_x), (tey, want_y)):
        assert got.dtype == torch.uint8 and tuple(got.shape) == want.shape
        assert np.array_equal(got.numpy(), want)
    assert np.array_equal(trx.numpy()[:, 0], imgs) and np.array_equal(tr_y.numpy(), labels)


def test_idx_failures_give_empty_like_reference(ref, tmp_path):
    _, _, pi, pl = _idx_files(tmp_path, n=5)
    short = str(tmp_path / "short")
    with open(pi, "rb") as f, open(short, "wb") as g:
        g.write(f.read()[:-7])
    missing = str(tmp_path / "missing")
    cases = [(pl, False), (pi, True), (short, False), (missing, False), (missing, True)]
    for path, labels in cases:
        assert ref.idx(path, labels) is None
        got = spyker.mnist_label(path) if labels else spyker.mnist_data(path)
        assert got.numel() == 0


def test_idx_multithreaded_payload(tmp_path):
    # a payload over the 16 MB chunk, read by several threads
    imgs = np.random.default_rng(1).integers(0, 256, size=(24000, 28, 28), dtype=np.uint8)
    path = str(tmp_path / "big-idx3-ubyte")
    io.write_idx(path, imgs)
    got = spyker.mnist_data(path)
    assert np.array_equal(got.numpy()[:, 0], imgs)


CSV_TEXT = "a, b, c\n\n1,2, 3\nx, , y, \nlast,  two\n"


@pytest.mark.parametrize("delim", [", ", ",", " "])
def test_csv_matches_reference(ref, tmp_path, delim):
    path = str(tmp_path / "t.csv")
    with open(path, "w") as f:
        f.write(CSV_TEXT)
    for skip in (0, 1, 3, 10):
        skipped, want = ref.csv_rows(path, delim, skip)
        c = spyker.CSV(path, delim)
        assert c.skip(skip) == skipped
        got = []
        while True:
            ok, row = c.readline()
            if not ok:
                break
            got.append(row)
        assert got == want
    ok, row = spyker.read_csv(path, delim)
    assert ok and row == ref.csv_rows(path, delim, 0, 1)[1][0]


def test_csv_missing_file():
    ok, row = spyker.read_csv("/nonexistent/file.csv")
    assert not ok and row == []


def test_npz_checkpoint_round_trip(tmp_path):
    k1 = torch.randn((30, 6, 5, 5))
    k2 = torch.randn((250, 30, 3, 3))
    path = str(tmp_path / "model.npz")
    # the examples' save: numpy.savez(path, conv1_kernel=to_numpy(kernel), ...)
    np.savez(path, conv1_kernel=spyker.to_numpy(k1), conv2_kernel=spyker.to_numpy(k2))
    a, b = torch.zeros_like(k1), torch.zeros_like(k2)
    data = np.load(path)
    # the examples' load: to_tensor(data[k]).to(kernel) copies in place
    assert spyker.to_tensor(data["conv1_kernel"], pinned=True).to(a) is None
    assert torch.equal(a, k1)
    c = torch.zeros_like(k2)
    io.load_kernels(path, conv2_kernel=c)
    assert torch.equal(c, k2)
    io.save_kernels(str(tmp_path / "m2.npz"), conv1_kernel=a, conv2_kernel=c)
    d = np.load(str(tmp_path / "m2.npz"))
    assert sorted(d.files) == ["conv1_kernel", "conv2_kernel"] and d["conv1_kernel"].dtype == np.float32
    with pytest.raises(ValueError):
        io.load_kernels(path, conv1_kernel=torch.zeros(3))
