"""Event-list ("sparse") spiking path (src/python/spyker/sparse.py) on the GPU.

A :class:`SparseTensor` of shape [U, T, C, H, W] keeps, per (sample, step),
the list of spiking positions (z, y, x), as the reference's SparseTensor
(src/spyker/utils.h:369-420).  On the device the lists are one CSR array:
``offsets`` int64 [U*T + 1] and ``events`` int32 (x | y << 8 | z << 16);
``events`` is sized for the worst case, so building a tensor never waits for
the host.  Every function runs on the GPU through the ``spk_sparse_*`` C ABI.
"""

from __future__ import annotations

from typing import List, Sequence, Union

import numpy
import torch

from . import _lib
from ._lib import call, i64, ptr, stream
from .utils import Bound, default_device, expand2, expand4, shape, to4, to5, torch_dtype, type_code


def _ws(nbytes: int, dev: torch.device):
    if nbytes == 0:
        return None, 0
    return torch.empty(int(nbytes), dtype=torch.uint8, device=dev), int(nbytes)


class SparseTensor:
    """Sparse binary spikes [U, T, C, H, W] as per-(sample, step) event lists.

    ``SparseTensor(tensor, threshold=0.0)`` converts a dense [U, T, C, H, W]
    tensor: every position gets one event at the first step whose value is
    above ``threshold`` (src/spyker/sparse/opers.cpp:59-86).
    """

    def __init__(self, tensor=None, threshold: float = 0.0, *, _lists=None) -> None:
        if _lists is not None:
            self.offsets, self.events, self._shape = _lists
            return
        if tensor is None:
            raise ValueError("SparseTensor needs a dense tensor")
        a = Bound(tensor, default_device())
        x = a.dev.contiguous()
        s = to5(list(x.shape))
        u, t, c, h, w = s
        cap = u * c * h * w
        offsets = torch.empty(u * t + 1, dtype=torch.int64, device=x.device)
        events = torch.empty(max(cap, 1), dtype=torch.int32, device=x.device)
        ws, wsb = _ws(_lib.lib.spk_sparse_from_dense_workspace(u, t, c, h, w), x.device)
        call("spk_sparse_from_dense", ptr(x), type_code(x.dtype), u, t, c, h, w, float(threshold), ptr(offsets),
             ptr(events), cap, ptr(ws), wsb, stream())
        self.offsets, self.events, self._shape = offsets, events, tuple(s)

    # -- properties of the reference's SparseTensor (bind.cpp:241-250) --------
    @property
    def shape(self) -> List[int]:
        return list(self._shape)

    @property
    def dims(self) -> int:
        return len(self._shape)

    @property
    def numel(self) -> int:
        """Number of events."""
        return int(self.offsets[-1].item())

    @property
    def bytes(self) -> int:
        return int(self.offsets.numel() * 8 + self.numel * 4)

    @property
    def device(self) -> torch.device:
        return self.offsets.device

    @property
    def capacity(self) -> int:
        return int(self.events.numel())

    def __bool__(self) -> bool:
        return True

    def sparsity(self) -> float:
        return self.numel / float(numpy.prod(self._shape))

    def copy(self) -> "SparseTensor":
        return SparseTensor(_lists=(self.offsets.clone(), self.events.clone(), self._shape))

    def dense(self) -> torch.Tensor:
        """Cumulative u8 spikes [U, T, C, H, W] (src/spyker/sparse/opers.cpp:88-104)."""
        u, t, c, h, w = self._shape
        out = torch.empty(self._shape, dtype=torch.uint8, device=self.device)
        ws, wsb = _ws(_lib.lib.spk_sparse_dense_workspace(u, c, h, w), self.device)
        call("spk_sparse_to_dense", ptr(self.offsets), ptr(self.events), u, t, c, h, w, ptr(out),
             type_code(torch.uint8), ptr(ws), wsb, stream())
        return out

    def lists(self):
        """Host copy: (offsets int64 [U*T + 1], zyx u8 [E, 3])."""
        off = self.offsets.cpu().numpy()
        ev = self.events[: int(off[-1])].cpu().numpy().astype(numpy.uint32)
        zyx = numpy.stack([(ev >> 16) & 255, (ev >> 8) & 255, ev & 255], axis=1).astype(numpy.uint8)
        return off, zyx

    @staticmethod
    def from_lists(offsets, zyx, shape_, dev=None) -> "SparseTensor":
        dev = dev or default_device()
        zyx = numpy.asarray(zyx, dtype=numpy.uint32).reshape(-1, 3)
        packed = (zyx[:, 0] << 16) | (zyx[:, 1] << 8) | zyx[:, 2]
        u, t, c, h, w = shape_
        cap = max(len(packed), 1)
        ev = torch.zeros(cap, dtype=torch.int32, device=dev)
        if len(packed):
            ev[: len(packed)] = torch.from_numpy(packed.astype(numpy.int64).astype(numpy.int32)).to(dev)
        off = torch.from_numpy(numpy.asarray(offsets, dtype=numpy.int64)).to(dev)
        return SparseTensor(_lists=(off, ev, tuple(shape_)))

    def __repr__(self) -> str:
        return f"SparseTensor(shape={self.shape}, capacity={self.capacity})"


def _new(shape_, cap: int, dev: torch.device) -> SparseTensor:
    u, t = shape_[0], shape_[1]
    off = torch.empty(u * t + 1, dtype=torch.int64, device=dev)
    ev = torch.empty(max(int(cap), 1), dtype=torch.int32, device=dev)
    return SparseTensor(_lists=(off, ev, tuple(shape_)))


def _check(array) -> SparseTensor:
    if not isinstance(array, SparseTensor):
        raise TypeError("expected a SparseTensor")
    return array


def code(array, time: int, sort: bool = True) -> SparseTensor:
    """Rank-order (sort) or latency code into event lists (sparse/code.cpp:39-130)."""
    if time <= 0:
        raise ValueError("Input time can't be less than 1.")
    x = Bound(array, default_device()).dev.contiguous()
    s = to4(list(x.shape))
    u, c, h, w = s
    out = _new((u, time, c, h, w), u * c * h * w, x.device)
    ws, wsb = _ws(_lib.lib.spk_sparse_code_workspace(u, time, c, h, w), x.device)
    call("spk_sparse_code", ptr(x), type_code(x.dtype), u, c, h, w, time, int(bool(sort)), ptr(out.offsets),
         ptr(out.events), out.capacity, ptr(ws), wsb, stream())
    return out


def conv(array, kernel, threshold: float, stride=1, pad=0) -> SparseTensor:
    """Incremental convolution + fire on event lists (sparse/conv.cpp:42-160)."""
    a = _check(array)
    s2, p4 = expand2(stride), expand4(pad)
    k = Bound(kernel, a.device).dev
    if k.dtype != torch.float32:
        k = k.float()
    k = k.contiguous()
    u, t, c, h, w = a._shape
    cout, cin, kh, kw = k.shape
    if cin != c:
        raise ValueError("Input and kernel channels are not compatible.")
    oh = h + p4[0] + p4[2] - kh + 1
    ow = w + p4[1] + p4[3] - kw + 1
    out = _new((u, t, cout, oh, ow), u * cout * max(oh, 1) * max(ow, 1), a.device)
    ws, wsb = _ws(_lib.lib.spk_sparse_conv_workspace(u, t, h, w, cout, kh, kw, i64(*p4)), a.device)
    call("spk_sparse_conv", ptr(a.offsets), ptr(a.events), u, t, c, h, w, ptr(k), cout, kh, kw, float(threshold),
         i64(*s2), i64(*p4), ptr(out.offsets), ptr(out.events), out.capacity, ptr(ws), wsb, stream())
    return out


def pad(array, pad) -> SparseTensor:
    """Shift every event by (top, left) (sparse/pad.cpp:37-55)."""
    a = _check(array)
    p4 = expand4(pad)
    if min(p4) < 0:
        raise ValueError("Pad items are incorrect.")
    u, t, c, h, w = a._shape
    out = _new((u, t, c, h + p4[0] + p4[2], w + p4[1] + p4[3]), a.capacity, a.device)
    call("spk_sparse_pad", ptr(a.offsets), ptr(a.events), a.capacity, u, t, c, h, w, i64(*p4), ptr(out.offsets),
         ptr(out.events), out.capacity, stream())
    return out


def gather(array, dtype="u8") -> torch.Tensor:
    """First event time per position [U, C, H, W], T when silent (sparse/opers.cpp:106-118)."""
    a = _check(array)
    u, t, c, h, w = a._shape
    out = torch.empty((u, c, h, w), dtype=torch_dtype(dtype), device=a.device)
    ws, wsb = _ws(_lib.lib.spk_sparse_dense_workspace(u, c, h, w), a.device)
    call("spk_sparse_gather", ptr(a.offsets), ptr(a.events), u, t, c, h, w, ptr(out), type_code(out.dtype), ptr(ws),
         wsb, stream())
    return out


def pool(array, kernel, stride=None, pad=0) -> SparseTensor:
    """First event of every pooled cell; stride must equal the kernel (sparse/pool.cpp:37-64)."""
    a = _check(array)
    k2 = expand2(kernel)
    s2 = expand2(kernel if stride is None else stride)
    p4 = expand4(pad)
    if min(k2) < 1 or min(s2) < 1 or min(p4) < 0:
        raise ValueError("Kernel, stride or pad items are incorrect.")
    u, t, c, h, w = a._shape
    oshape = shape.pool([u, t, c, h, w], k2, s2, p4)
    oh, ow = oshape[3], oshape[4]
    cap = max(1, min(a.capacity, u * c * oh * ow))
    out = _new(oshape, cap, a.device)
    ws, wsb = _ws(_lib.lib.spk_sparse_pool_workspace(u, c, oh, ow, a.capacity), a.device)
    call("spk_sparse_pool", ptr(a.offsets), ptr(a.events), a.capacity, u, t, c, h, w, i64(*k2), i64(*s2), i64(*p4),
         oh, ow, ptr(out.offsets), ptr(out.events), out.capacity, ptr(ws), wsb, stream())
    return out


def inhibit(array) -> SparseTensor:
    """Per pixel keep the channel of its first event (sparse/inhibit.cpp:37-65)."""
    a = _check(array)
    u, t, c, h, w = a._shape
    out = _new(a._shape, a.capacity, a.device)
    ws, wsb = _ws(_lib.lib.spk_sparse_inhibit_workspace(u, h, w, a.capacity), a.device)
    call("spk_sparse_inhibit", ptr(a.offsets), ptr(a.events), a.capacity, u, t, c, h, w, ptr(out.offsets),
         ptr(out.events), out.capacity, ptr(ws), wsb, stream())
    return out


def convwta(array, radius, count: int):
    """Winners in (step, list) order outside every accepted box (sparse/wta.cpp:44-95)."""
    from .module import Winners

    a = _check(array)
    r2 = expand2(radius)
    if min(r2) < 0:
        raise ValueError("Radius items are incorrect.")
    if count <= 0:
        raise ValueError("Winners count can't be less than 1.")
    u, t, c, h, w = a._shape
    rec = torch.zeros((u, count, 5), dtype=torch.int32, device=a.device)
    cnt = torch.zeros((u,), dtype=torch.int32, device=a.device)
    call("spk_sparse_convwta", ptr(a.offsets), ptr(a.events), u, t, c, h, w, i64(*r2), count, ptr(rec), ptr(cnt),
         stream())
    return Winners(rec, cnt)


def stdp(layer, array, winners) -> None:
    """Conv::stdp(SparseTensor, winners): STDP from event lists (sparse/stdp.cpp:41-133)."""
    from .module import Winners, _check_winners, _configs

    a = _check(array)
    if len(layer.stdpconfig) == 0:
        raise ValueError("At least one STDP Config must be given.")
    if layer.kernel.dtype != torch.float32:
        raise TypeError("STDP needs an F32 kernel in spyker_b200")
    u, t, c, h, w = a._shape
    wn = Winners.from_lists(winners, a.device)
    _check_winners(wn, len(layer.stdpconfig), u)
    cout, cin, kh, kw = layer.kernel.shape
    if cin != c:
        raise ValueError("Input and kernel channels are not compatible.")
    p4 = layer._pad
    ws, wsb = _ws(_lib.lib.spk_sparse_stdp_workspace(u, wn.count, c, h, w, kh, kw, i64(*p4)), a.device)
    call("spk_sparse_stdp", ptr(a.offsets), ptr(a.events), u, t, c, h, w, ptr(layer.kernel), cout, kh, kw,
         _configs(layer.stdpconfig), len(layer.stdpconfig), ptr(wn.records), ptr(wn.counts), wn.count, i64(*p4),
         ptr(ws), wsb, stream())


def to_sparse(*arrays, threshold: float = 0.0):
    """Dense arrays to SparseTensors (src/python/spyker/utils.py:506-529)."""
    out = tuple(SparseTensor(a, threshold) for a in arrays)
    return out if len(out) > 1 else out[0]
