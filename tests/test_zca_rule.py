"""The NumPy FP64 ZCA restatement (oracle/zca.py) against the properties that
define ZCA whitening: with epsilon -> 0 the whitened samples have identity
covariance, the whitening matrix is symmetric and is the inverse square root
of the covariance, and the split keeps x = pos - neg with both parts >= 0;
and against the reference's own cpu/zca.cpp built with a Blasw stand-in."""

import numpy as np
import pytest

from oracle import zca


def _samples(n=2000, d=24, seed=0):
    rng = np.random.default_rng(seed)
    mix = rng.normal(size=(d, d))
    return (rng.normal(size=(n, d)) @ mix + rng.normal(size=d)).astype(np.float32)


def test_whitened_covariance_is_identity():
    x = _samples()
    mean, trans = zca.zca_fit(x, 1e-12)
    y = zca.zca_transform(x, mean, trans)
    cov = np.cov(y, rowvar=False)
    assert np.allclose(cov, np.eye(x.shape[1]), atol=1e-8)
    assert np.allclose(y.mean(axis=0), 0, atol=1e-8)


def test_transform_is_symmetric_inverse_root():
    x = _samples(d=16)
    mean, trans = zca.zca_fit(x, 0.0)
    sigma = np.cov(x.astype(np.float64), rowvar=False)
    assert np.allclose(trans, trans.T, atol=1e-12)
    assert np.allclose(trans @ sigma @ trans, np.eye(16), atol=1e-8)
    assert np.allclose(mean, x.astype(np.float64).mean(axis=0))


def test_epsilon_damps_small_directions():
    x = _samples(d=8)
    x[:, 7] = x[:, 6]  # a zero-variance direction
    _, trans = zca.zca_fit(x, 0.5)
    assert np.isfinite(trans).all()
    assert np.abs(trans).max() < 1 / np.sqrt(0.5) + 1e-9


def test_split_parts():
    x = np.random.default_rng(3).normal(size=(5, 3, 4)).astype(np.float32)
    s = zca.zca_split(x)
    assert s.shape == (5, 2, 3, 4) and s.dtype == np.float32
    assert (s >= 0).all() and np.array_equal(s[:, 0] - s[:, 1], x)


@pytest.mark.parametrize("n,d,dtype,eps,tol", [
    (2000, 24, np.float64, 1e-12, 1e-8),
    (517, 105, np.float64, 1e-12, 1e-8),
    (517, 105, np.float64, 0.1, 1e-12),
    (65, 64, np.float64, 1e-12, 1e-9),
    (800, 48, np.float32, 0.1, 2e-6),
    (3000, 200, np.float32, 0.1, 2e-6),
])
def test_restatement_matches_reference_build(ref, n, d, dtype, eps, tol):
    """oracle/zca.py against the reference's own cpu/zca.cpp, compiled with
    the Blasw stand-in (oracle/blasw_shim): mean, whitening matrix, the
    in-place transform of zca_fit and zca_trans agree to FP64 rounding of an
    eigenproblem (F32 inputs: the reference forms sigma in F32, so its
    whitening matrix carries F32 rounding)."""
    rng = np.random.default_rng(n + d)
    mix = rng.normal(size=(d, d)) / np.sqrt(d)
    x = (rng.normal(size=(n, d)) @ mix + rng.normal(size=d)).astype(dtype)
    mean, trans, whitened = ref.zca_fit(x, eps, transform=True)
    om, ot = zca.zca_fit(x, eps)
    want = zca.zca_transform(x, om, ot)

    def rel(a, b):
        return np.abs(a.astype(np.float64) - b).max() / np.abs(b).max()

    assert mean.dtype == dtype and trans.shape == (d, d)
    assert rel(mean, om) < tol and rel(trans, ot) < tol
    assert rel(whitened, want) < tol
    assert rel(ref.zca_trans(x, mean, trans), want) < tol
    assert np.array_equal(ref.zca_split(whitened), zca.zca_split(whitened))
