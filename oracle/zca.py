"""ZCA whitening restated in NumPy FP64: test infrastructure, the checker of
the library's GPU ZCA, never called by the library itself.

Follows src/spyker/cpu/zca.cpp:67-155 (zca_fit, zca_trans, zca_split):
  mean  = column means of X [N, D]                          (zca.cpp:74-77)
  sigma = (X - mean)^T (X - mean) / (N - 1)                 (zca.cpp:79-84)
  sigma = U diag(lambda) U^T, lambda ascending              (zca.cpp:86-87)
  trans = U diag(1 / sqrt(max(lambda, 0) + epsilon)) U^T    (zca.cpp:60-64, 89-97)
  transform: X <- (X - mean) trans                          (zca.cpp:99-118)
  split: [N, D] -> [N, 2, D] = (max(x, 0), max(-x, 0))      (zca.cpp:140-155)

Pinned to the reference's own cpu/zca.cpp: that file needs the Blasw
BLAS/LAPACK wrapper (github.com/Mathific/Blasw, an empty submodule in the
reference tree; zca.cpp:121-136 refuses without it), so oracle/Makefile
compiles it unmodified against oracle/blasw_shim (a stand-in giving gemv,
gemm/symm, syrk and a Jacobi eigensolver the semantics zca.cpp relies on),
and tests/test_zca_rule.py compares this restatement with that build as well
as with the defining properties of ZCA whitening.  The eigensolver inside the
pinned build is the stand-in's, not the reference's LAPACK.
"""

from __future__ import annotations

import numpy as np


def zca_fit(x: np.ndarray, epsilon: float):
    """(mean [D], trans [D, D]) in FP64 for samples x [N, ...]."""
    x = np.asarray(x, dtype=np.float64).reshape(x.shape[0], -1)
    mean = x.mean(axis=0)
    mid = x - mean
    sigma = mid.T @ mid / (x.shape[0] - 1)
    values, vectors = np.linalg.eigh(sigma)
    w = 1.0 / np.sqrt(np.maximum(values, 0.0) + epsilon)
    return mean, (vectors * w) @ vectors.T


def zca_transform(x: np.ndarray, mean: np.ndarray, trans: np.ndarray) -> np.ndarray:
    """(x - mean) trans in FP64, with x's shape."""
    flat = np.asarray(x, dtype=np.float64).reshape(x.shape[0], -1)
    return ((flat - mean) @ trans).reshape(x.shape)


def zca_split(x: np.ndarray) -> np.ndarray:
    """[N, ...] -> [N, 2, ...]: positive and negative parts."""
    return np.stack([np.maximum(x, 0), np.maximum(-x, 0)], axis=1).astype(x.dtype)
