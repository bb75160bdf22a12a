"""ZCA whitening on the GPU against the NumPy FP64 restatement of
cpu/zca.cpp:67-155 (oracle/zca.py): mean, whitening matrix and transformed
samples, in place and out of place, across NumPy / PyTorch inputs; the split
bit for bit; and at MNIST size (60000 x 784) the defining property, identity
covariance of the whitened samples."""

import numpy as np
import pytest
import torch

import spyker_b200 as spyker
from oracle import zca as oracle

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _samples(n, d, seed=0):
    rng = np.random.default_rng(seed)
    mix = rng.normal(size=(d, d)) / np.sqrt(d)
    return (rng.normal(size=(n, d)) @ mix + rng.normal(size=d)).astype(np.float32)


def _rel(got, want):
    return float(np.abs(np.asarray(got, np.float64) - want).max() / max(np.abs(want).max(), 1e-30))


@pytest.mark.parametrize("shape", [(3000, 200), (517, 3, 5, 7), (65, 64), (2, 1)])
def test_fit_matches_fp64_oracle(shape):
    x = _samples(shape[0], int(np.prod(shape[1:])), seed=len(shape)).reshape(shape)
    eps = 1e-2
    z = spyker.ZCA().fit(torch.from_numpy(x).to(DEV), eps)
    mean, trans = oracle.zca_fit(x, eps)
    assert z.mean.dtype == torch.float32 and z.transform.dtype == torch.float32
    assert _rel(z.mean.cpu().numpy(), mean) < 1e-6
    assert _rel(z.transform.cpu().numpy(), trans) < 1e-6
    want = oracle.zca_transform(x, mean, trans)
    got = z(torch.from_numpy(x).to(DEV), inplace=False)
    assert got.shape == x.shape
    assert _rel(got.cpu().numpy(), want) < 1e-5


def test_fit_transform_in_place_and_ecosystems():
    x = _samples(1200, 96, seed=5)
    keep = x.copy()
    eps = 1e-3
    mean, trans = oracle.zca_fit(keep, eps)
    want = oracle.zca_transform(keep, mean, trans)
    z = spyker.ZCA().fit(x, eps, transform=True)  # NumPy, in place
    assert _rel(x, want) < 1e-5
    keep0 = keep.copy()
    y = z(keep, inplace=False)
    assert isinstance(y, np.ndarray) and np.array_equal(keep, keep0)
    assert _rel(y, want) < 1e-5
    t = torch.from_numpy(keep.copy())
    a, b = z(t, t.clone())  # PyTorch CPU tensors, in place, two at once
    assert _rel(a.numpy(), want) < 1e-5 and torch.equal(a, b)


def test_mnist_size_whitening_is_identity_covariance():
    n, d = 60000, 784
    g = torch.Generator(device=DEV).manual_seed(11)
    # an orthogonal basis with scales 0.05..3: covariance eigenvalues 0.0025..9
    q = torch.linalg.qr(torch.randn((d, d), generator=g, device=DEV, dtype=torch.float64))[0]
    mix = q * torch.linspace(0.05, 3.0, d, device=DEV, dtype=torch.float64)
    x = (torch.randn((n, d), generator=g, device=DEV, dtype=torch.float64) @ mix.T).float().view(n, 1, 28, 28)
    z = spyker.ZCA().fit(x, 1e-9, transform=True)
    y = x.view(n, d).double()
    cov = (y - y.mean(0)).T @ (y - y.mean(0)) / (n - 1)
    assert float((cov - torch.eye(d, device=DEV, dtype=torch.float64)).abs().max()) < 2e-3
    assert float(y.mean(0).abs().max()) < 1e-3
    assert torch.allclose(z.transform, z.transform.T, atol=1e-6)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_split_bit_exact(dtype):
    x = torch.randn((7, 3, 9, 11), dtype=dtype).to(DEV)
    got = spyker.ZCA.split(x)
    want = oracle.zca_split(x.cpu().numpy())
    assert got.shape == (7, 2, 3, 9, 11) and got.dtype == dtype
    assert np.array_equal(got.cpu().numpy(), want)
    assert isinstance(spyker.ZCA.split(x.cpu().numpy()), np.ndarray)


def test_errors_and_save_load(tmp_path):
    with pytest.raises(TypeError):
        spyker.ZCA().fit(torch.zeros((4, 3), dtype=torch.float16, device=DEV), 0.1)
    with pytest.raises(ValueError):
        spyker.ZCA().fit(torch.zeros(4, device=DEV), 0.1)
    with pytest.raises(RuntimeError):
        spyker.ZCA()(torch.zeros((4, 3), device=DEV))
    x = _samples(300, 20, seed=2)
    z = spyker.ZCA().fit(x, 0.1)
    path = str(tmp_path / "zca.npz")
    z.save(path)
    w = spyker.ZCA()
    w.load(path)
    assert torch.equal(w.mean.cpu(), z.mean.cpu()) and torch.equal(w.transform.cpu(), z.transform.cpu())
    assert _rel(w(x, inplace=False), oracle.zca_transform(x, z.mean.cpu().double().numpy(),
                                                           z.transform.cpu().double().numpy())) < 1e-5


def test_cuda_tensor_in_place_and_split_after_transform():
    x = torch.from_numpy(_samples(800, 48, seed=8)).to(DEV).view(800, 3, 4, 4)
    keep = x.clone()
    z = spyker.ZCA().fit(x, 1e-2, transform=True)  # in place on the device tensor
    mean, trans = oracle.zca_fit(keep.cpu().numpy(), 1e-2)
    want = oracle.zca_transform(keep.cpu().numpy(), mean, trans)
    assert _rel(x.cpu().numpy(), want) < 1e-5
    s = spyker.ZCA.split(x)
    assert s.shape == (800, 2, 3, 4, 4)
    assert np.array_equal(s.cpu().numpy(), oracle.zca_split(x.cpu().numpy()))
