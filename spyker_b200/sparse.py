"""Sparse event-list path (src/python/spyker/sparse.py)."""

from __future__ import annotations


class SparseTensor:
    """Event lists per (sample, step) of (z, y, x) u8 coordinates."""

    def __init__(self, *args, **kwargs):
        raise NotImplementedError("the GPU sparse path is not built yet")


def _missing(*args, **kwargs):
    raise NotImplementedError("the GPU sparse path is not built yet")


code = conv = gather = pool = inhibit = convwta = stdp = _missing
