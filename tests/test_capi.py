"""The C-ABI library loads, exports every declared entry point, and its
host-side logic (kernel generators, argument checks) is right — no GPU."""

import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from spyker_b200 import _lib
from spyker_b200.utils import expand2, expand4, least2, least3, shape, to5

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "spyker_b200.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(spk_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (spk_[a-z0-9_]+)", out))
    missing = [s for s in declared() if s not in exported]
    assert not missing, missing
    assert len(declared()) >= 30


def test_python_signatures_cover_header():
    assert set(declared()) <= set(_lib.SIGNATURES)


@pytest.mark.parametrize("size,std", [(7, 1.0), (7, 2.0), (5, 0.7), (13, 3.3)])
def test_gaussian_kernel_matches_reference(port, size, std):
    k = np.zeros((size, size))
    _lib.call("spk_gaussian_kernel", k.ctypes.data, size, std)
    assert np.array_equal(k, port.gaussian_kernel(size, std))


def test_gabor_and_log_kernels(port):
    k = np.zeros((11, 11))
    _lib.call("spk_gabor_kernel", k.ctypes.data, 11, 2.0, 0.6, 0.5, 5.0, 0.1)
    assert np.array_equal(k, port.gabor_kernel(11, 2.0, 0.6, 0.5, 5.0, 0.1))
    _lib.call("spk_log_kernel", k.ctypes.data, 11, 1.7)
    assert np.array_equal(k, port.log_kernel(11, 1.7))


def test_normal_kernel_is_seeded():
    a, b = np.zeros(50), np.zeros(50)
    _lib.lib.spk_random_seed(5)
    _lib.call("spk_normal_kernel", a.ctypes.data, 50, 0.8, 0.05)
    _lib.lib.spk_random_seed(5)
    _lib.call("spk_normal_kernel", b.ctypes.data, 50, 0.8, 0.05)
    assert np.array_equal(a, b) and abs(a.mean() - 0.8) < 0.05


def _status(name, *args):
    return getattr(_lib.lib, name)(*args)


def test_argument_errors_are_reported_without_a_gpu():
    pad = _lib.i64(0, 0, 0, 0)
    bad_pad = _lib.i64(0, -1, 0, 0)
    # shapes that do not fit the kernel
    st = _status("spk_conv", None, 4, None, None, 1, 1, 3, 3, 1, 5, 5, 1, 1, pad, 0, None, 0, None)
    assert st == 1 and b"not compatible" in _lib.lib.spk_last_error()
    st = _status("spk_conv", None, 4, None, None, 1, 1, 8, 8, 1, 5, 5, 1, 1, bad_pad, 0, None, 0, None)
    assert st == 1 and b"pad" in _lib.lib.spk_last_error()
    st = _status("spk_rank_code", None, 9, None, 4, 1, 0, 10, 1, None, 0, None)
    assert st == 1 and b"time" in _lib.lib.spk_last_error()
    st = _status("spk_rank_convwta", None, 9, 1, 1, 1, 1, 1, 0, 0, 0, 0.0, None, None, None, 0, None)
    assert st == 1 and b"count" in _lib.lib.spk_last_error()
    cfg = _lib.f64([0.1, -0.1, 1, 0, 1])
    st = _status("spk_rank_convstdp", None, 4, 1, 1, 1, 5, 5, None, 1, 1, 1, None, 5, 5, cfg, 0, None, None, 1, 1, 1,
                 pad, None, 0, None)
    assert st == 1 and b"STDP config" in _lib.lib.spk_last_error()
    # unsupported data type code
    st = _status("spk_threshold", C.c_void_p(16), 5, 10, 0.0, 0.0, None)
    assert st == 3
    # empty work is a no-op
    assert _status("spk_threshold", None, 9, 0, 0.0, 0.0, None) == 0


def test_shape_helpers():
    assert expand2(3) == (3, 3) and expand2([2, 5]) == (2, 5)
    assert expand4(2) == (2, 2, 2, 2) and expand4([1, 2]) == (1, 2, 1, 2) and expand4([1, 2, 3, 4]) == (1, 2, 3, 4)
    with pytest.raises(ValueError):
        expand4([1, 2, 3])
    assert least2([5]) == [1, 5] and least3([2, 3]) == [1, 2, 3] and to5([2, 3, 4, 5]) == [1, 2, 3, 4, 5]
    with pytest.raises(ValueError):
        to5([1, 2, 3])
    assert shape.conv([4, 15, 2, 28, 28], [30, 2, 5, 5], (1, 1), (2, 2, 2, 2)) == [4, 15, 30, 28, 28]
    assert shape.conv([4, 15, 2, 28, 28], [30, 2, 5, 5], (2, 2), (1, 2, 0, 1)) == [4, 15, 30, 13, 14]
    assert shape.pool([4, 15, 30, 28, 28], (2, 2), (2, 2), (1, 1, 1, 1)) == [4, 15, 30, 15, 15]
    with pytest.raises(ValueError):
        shape.conv([4, 15, 3, 28, 28], [30, 2, 5, 5], (1, 1), (0, 0, 0, 0))


def test_nvtx_ranges_wrap_calls(port, monkeypatch):
    """With the NVTX ranges on, every call is bracketed by one push and one
    pop named after the entry point, also when the call fails; results are
    unchanged."""
    import torch

    events = []
    monkeypatch.setattr(torch.cuda.nvtx, "range_push", lambda n: events.append(("push", n)))
    monkeypatch.setattr(torch.cuda.nvtx, "range_pop", lambda: events.append(("pop",)))
    _lib.set_nvtx(True)
    try:
        k = np.zeros((7, 7))
        _lib.call("spk_gaussian_kernel", k.ctypes.data, 7, 1.3)
        assert np.array_equal(k, port.gaussian_kernel(7, 1.3))
        with pytest.raises(_lib.SpykerError):
            _lib.call("spk_rank_code", None, 9, None, 4, 1, 0, 10, 1, None, 0, None)
    finally:
        _lib.set_nvtx(False)
    assert events == [("push", "spk_gaussian_kernel"), ("pop",), ("push", "spk_rank_code"), ("pop",)]
    _lib.call("spk_gaussian_kernel", k.ctypes.data, 7, 1.3)
    assert len(events) == 4


def test_pool_window_larger_than_plane_is_refused():
    """A window taller or wider than the padded plane has no output: refused
    before any launch (C division would give one output row)."""
    pad = _lib.i64(0, 0, 0, 0)
    # h = 1 under a 2x2 window: (1 - 2) / 2 + 1 == 1 in C
    st = _status("spk_rank_pool", C.c_void_p(16), C.c_void_p(16), 4, 1, 1, 8, 1, 4, 2, 2, 2, 2, pad, None)
    assert st == 1 and b"not compatible" in _lib.lib.spk_last_error()
    # the same plane padded to the window's height is fine up to the launch (n = 0: nothing runs)
    st = _status("spk_rank_pool", None, None, 4, 0, 1, 8, 1, 4, 2, 2, 2, 2, _lib.i64(1, 0, 0, 0), None)
    assert st == 0
