"""Spyker's Python API (src/python/spyker/module.py) over the sm_100a library.

Same names, arguments, defaults and error behaviour as the reference; every
operation runs on the GPU through the ``spk_*`` C ABI (``include/spyker_b200.h``)
on the current torch stream.  Outputs are allocated in the caller's
ecosystem: CUDA tensors in, CUDA tensors out (no copies); NumPy / CPU tensors
are staged through the device.
"""

from __future__ import annotations

import math
from typing import List, Sequence, Union

import numpy
import torch

from . import _lib
from ._lib import call, i64, ptr, stream
from .utils import (Bound, clone_array, default_device, expand2, expand4, least2, least3, shape, to3, to4, to5,
                    torch_dtype, type_code)

# Arithmetic of Conv layers: "bf16x3" (default, tcgen05), "bf16x2" (tcgen05,
# the hi+lo split), "fp32" (plain SIMT).
_PRECISION = {"fp32": 0, "bf16x2": 1, "bf16x3": 2}
_conv_precision = "fp32"


def set_conv_precision(name: str) -> None:
    """Select the arithmetic of the spike x weight contraction."""
    global _conv_precision
    if name not in _PRECISION:
        raise ValueError(f"precision must be one of {sorted(_PRECISION)}")
    _conv_precision = name


def conv_precision() -> str:
    return _conv_precision


def _workspace(nbytes: int, dev: torch.device):
    if nbytes == 0:
        return None, 0
    return torch.empty(int(nbytes), dtype=torch.uint8, device=dev), int(nbytes)


# ---------------------------------------------------------------------------
# configuration records (src/spyker/utils.h:483-547, opers.h:160-190)
# ---------------------------------------------------------------------------


class Winner:
    """Winner neuron (c: STDP config index, t: time, z: channel, y, x)."""

    __slots__ = ("c", "t", "z", "y", "x")

    def __init__(self, c: int = 0, t: int = 0, z: int = 0, y: int = 0, x: int = 0):
        self.c, self.t, self.z, self.y, self.x = int(c), int(t), int(z), int(y), int(x)

    def __repr__(self) -> str:
        return f"Winner(c={self.c}, t={self.t}, z={self.z}, y={self.y}, x={self.x})"

    def __eq__(self, o) -> bool:
        return isinstance(o, Winner) and (self.c, self.t, self.z, self.y, self.x) == (o.c, o.t, o.z, o.y, o.x)


class Winners(Sequence):
    """``List[List[Winner]]`` backed by device records [B, count, 5] + counts [B].

    Behaves like the reference's nested list (indexing, ``len``, iteration);
    the host copy is made on first access, and STDP consumes the device
    records directly without a host round trip.
    """

    def __init__(self, records: torch.Tensor, counts: torch.Tensor):
        self.records, self.counts = records, counts
        self._host: List[List[Winner]] | None = None

    @property
    def count(self) -> int:
        return int(self.records.shape[1])

    def lists(self) -> List[List[Winner]]:
        if self._host is None:
            rec = self.records.cpu().numpy()
            cnt = self.counts.cpu().numpy()
            self._host = [[Winner(*rec[i, j]) for j in range(int(cnt[i]))] for i in range(rec.shape[0])]
        return self._host

    def __getitem__(self, i):
        return self.lists()[i]

    def __len__(self) -> int:
        return int(self.records.shape[0])

    def __repr__(self) -> str:
        return repr(self.lists())

    @staticmethod
    def from_lists(winners, dev: torch.device) -> "Winners":
        if isinstance(winners, Winners):
            return winners
        count = max([len(w) for w in winners] + [1])
        rec = numpy.zeros((len(winners), count, 5), dtype=numpy.int32)
        cnt = numpy.zeros(len(winners), dtype=numpy.int32)
        for i, lst in enumerate(winners):
            cnt[i] = len(lst)
            for j, w in enumerate(lst):
                rec[i, j] = (w.c, w.t, w.z, w.y, w.x)
        return Winners(torch.from_numpy(rec).to(dev), torch.from_numpy(cnt).to(dev))


class STDPConfig:
    """STDP configuration (utils.h:505-524)."""

    def __init__(self, positive: float, negative: float, stabilize: bool = True, lower: float = 0.0,
                 upper: float = 1.0) -> None:
        self.positive, self.negative = float(positive), float(negative)
        self.stabilize, self.lower, self.upper = bool(stabilize), float(lower), float(upper)

    def _row(self):
        return (self.positive, self.negative, 1.0 if self.stabilize else 0.0, self.lower, self.upper)


class BPConfig:
    """Backpropagation configuration (utils.h:527-547)."""

    def __init__(self, sfactor: float = 1.0, lrate: float = 1.0, lrf: float = 1.0, lamda: float = 0.0) -> None:
        self.sfactor, self.lrate, self.lrf, self.lamda = float(sfactor), float(lrate), float(lrf), float(lamda)


class DoGFilter:
    def __init__(self, std1: float, std2: float) -> None:
        self.std1, self.std2 = float(std1), float(std2)


class GaborFilter:
    """Gabor parameters; ``theta`` in degrees (converted as opers.h:203-206)."""

    def __init__(self, sigma: float, theta: float, gamma: float, lambda_: float, psi: float) -> None:
        self.sigma, self.gamma, self.lambda_, self.psi = float(sigma), float(gamma), float(lambda_), float(psi)
        self.theta = float(theta) * 0.017453292519943295


def random_seed(seed: int) -> None:
    """Seed the global generator the layer constructors draw from."""
    _lib.lib.spk_random_seed(int(seed))


def _host_kernel(fn: str, size: int, *args) -> numpy.ndarray:
    k = numpy.zeros((size, size), dtype=numpy.float64)
    call(fn, k.ctypes.data, size, *[float(a) for a in args])
    return k


def _layer_device(dev) -> torch.device:
    if dev is None:
        return default_device()
    if isinstance(dev, torch.device) and dev.type == "cuda":
        return dev
    return default_device()


# ---------------------------------------------------------------------------
# filter banks (opers.cpp:245-315, 720-803)
# ---------------------------------------------------------------------------


def _filter(which: int, array, kernel: torch.Tensor, pad4, nk: int, fo: int):
    a = Bound(array, kernel.device)
    x = a.dev.to(torch.float32) if a.dev.dtype != torch.float32 else a.dev
    s = to4(list(x.shape))
    kh, kw = kernel.shape[-2:]
    oshape = shape.filt(s, kh, kw, pad4, fo)
    out = torch.empty(oshape, dtype=torch.float32, device=x.device)
    call("spk_filter", which, ptr(x.contiguous()), ptr(kernel), ptr(out), s[0] * s[1], s[2], s[3], nk, kh, kw,
         oshape[2], oshape[3], i64(*pad4), stream())
    return a.back(out)


class DoG:
    """Difference-of-Gaussians bank: out = max(g(std1) - g(std2), 0)."""

    def __init__(self, size: int, filters, pad=0, device=None, dtype="f32") -> None:
        if size <= 0:
            raise ValueError("Input size can't be less than 1.")
        flist = [filters] if isinstance(filters, DoGFilter) else list(filters)
        if not flist:
            raise ValueError("Input filters count can't be less then 1.")
        self._pad = expand4(pad)
        if min(self._pad) < 0:
            raise ValueError("Pad items are incorrect.")
        n = 2 * size + 1
        k = numpy.zeros((2, len(flist), n, n))
        for i, f in enumerate(flist):
            k[0, i] = _host_kernel("spk_gaussian_kernel", n, f.std1)
            k[1, i] = _host_kernel("spk_gaussian_kernel", n, f.std2)
        self.device = _layer_device(device)
        self.kernel = torch.from_numpy(k).to(torch_dtype(dtype)).to(self.device)

    def __call__(self, array):
        return _filter(0, array, self.kernel.float().contiguous(), self._pad, self.kernel.shape[1],
                       self.kernel.shape[1])


class Gabor:
    """Gabor bank (raw responses)."""

    def __init__(self, size: int, filters, pad=0, device=None, dtype="f32") -> None:
        if size <= 0:
            raise ValueError("Input size can't be less than 1.")
        flist = [filters] if isinstance(filters, GaborFilter) else list(filters)
        if not flist:
            raise ValueError("Input filters count can't be less then 1.")
        self._pad = expand4(pad)
        n = 2 * size + 1
        k = numpy.stack([_host_kernel("spk_gabor_kernel", n, f.sigma, f.theta, f.gamma, f.lambda_, f.psi)
                         for f in flist])
        self.device = _layer_device(device)
        self.kernel = torch.from_numpy(k).to(torch_dtype(dtype)).to(self.device)

    def __call__(self, array):
        return _filter(1, array, self.kernel.float().contiguous(), self._pad, self.kernel.shape[0],
                       self.kernel.shape[0])


class LoG:
    """Laplacian-of-Gaussian bank as DoG(std/sqrt2, std*sqrt2), split on/off."""

    def __init__(self, size: int, stds, pad=0, device=None, dtype="f32") -> None:
        if size <= 0:
            raise ValueError("Input size can't be less than 1.")
        slist = [stds] if isinstance(stds, (int, float)) else list(stds)
        if not slist:
            raise ValueError("Input stds count can't be less then 1.")
        self._pad = expand4(pad)
        n = 2 * size + 1
        k = numpy.zeros((2, len(slist), n, n))
        for i, s in enumerate(slist):
            k[0, i] = _host_kernel("spk_gaussian_kernel", n, s / math.sqrt(2))
            k[1, i] = _host_kernel("spk_gaussian_kernel", n, s * math.sqrt(2))
        self.device = _layer_device(device)
        self.kernel = torch.from_numpy(k).to(torch_dtype(dtype)).to(self.device)

    def __call__(self, array):
        f = self.kernel.shape[1]
        return _filter(2, array, self.kernel.float().contiguous(), self._pad, f, 2 * f)


class ZCA:
    """ZCA whitening (module.py ZCA, opers.cpp:807-831, cpu/zca.cpp:67-155).

    ``fit`` computes the feature means and the covariance of ``[N, D]`` (the
    input flattened per sample) with FP64 sums on the GPU, the symmetric
    eigendecomposition of the covariance in FP64 (``torch.linalg.eigh`` on
    the GPU), and the whitening matrix ``U diag(1 / sqrt(max(lambda, 0) +
    epsilon)) U^T`` in FP64.  ``mean`` and ``transform`` are F32 like the
    reference's; the FP64 copies are kept for applying the transform.
    """

    def __init__(self) -> None:
        self.mean = None
        self.transform = None
        self._mean64 = None
        self._trans64 = None

    def fit(self, array, epsilon: float, transform: bool = False) -> "ZCA":
        a = Bound(array)
        x = a.dev
        if x.dim() < 2:
            raise ValueError("Input dimensions must be at least 2D.")
        if x.dtype != torch.float32:
            raise TypeError("Input data type must be F32.")
        x2 = x.reshape(x.shape[0], -1)
        n, d = x2.shape
        mean = torch.empty(d, dtype=torch.float64, device=x.device)
        cov = torch.empty((d, d), dtype=torch.float64, device=x.device)
        wbytes = int(_lib.lib.spk_zca_stats_workspace(n, d))
        work = torch.empty(max(wbytes, 1), dtype=torch.uint8, device=x.device)
        call("spk_zca_stats", ptr(x2), n, d, ptr(mean), ptr(cov), ptr(work), wbytes, stream())
        lam, vec = torch.linalg.eigh(cov)
        vec = vec.contiguous()
        work = torch.empty(d, dtype=torch.float64, device=x.device)
        trans = torch.empty((d, d), dtype=torch.float64, device=x.device)
        call("spk_zca_matrix", ptr(vec), ptr(lam.contiguous()), d, float(epsilon), ptr(work), ptr(trans), stream())
        self._mean64, self._trans64 = mean, trans
        self.mean, self.transform = mean.float(), trans.float()
        if transform:
            self(array)
        return self

    def _apply(self, array):
        if self.mean is None or self.transform is None:
            raise RuntimeError("ZCA layer is not initialized.")
        a = Bound(array, writeable=True)
        x = a.dev
        if x.dim() < 2:
            raise ValueError("Input dimensions must be at least 2D.")
        if x.dtype != torch.float32:
            raise TypeError("Input data type must be F32.")
        x2 = x.reshape(x.shape[0], -1)
        n, d = x2.shape
        m64 = self._mean64 if self._mean64 is not None else self.mean.double()
        t64 = self._trans64 if self._trans64 is not None else self.transform.double()
        if m64.numel() != d or t64.shape != (d, d):
            raise ValueError("Input shape does not match the fitted ZCA.")
        m64, t64 = m64.to(x.device).contiguous(), t64.to(x.device).contiguous()
        out = torch.empty_like(x2)
        call("spk_zca_transform", ptr(x2), n, d, ptr(m64), ptr(t64), ptr(out), stream())
        x2.copy_(out)
        return a.write_back() if a.kind != "cuda" else array

    def __call__(self, *array, inplace: bool = True):
        if not inplace:
            array = [clone_array(x) for x in array]
        out = [self._apply(x) for x in array]
        return tuple(out) if len(out) > 1 else out[0]

    @staticmethod
    def split(array):
        """[N, ...] -> [N, 2, ...]: the positive and negative parts."""
        a = Bound(array)
        x = a.dev
        if x.dim() < 2:
            raise ValueError("Input dimensions must be more than 1.")
        if x.dtype not in (torch.float32, torch.float64):
            raise TypeError("ZCA split supports F32 and F64.")
        n = x.shape[0]
        d = x[0].numel() if x.dim() > 1 else 1
        out = torch.empty((n, 2) + tuple(x.shape[1:]), dtype=x.dtype, device=x.device)
        call("spk_zca_split", ptr(x), type_code(x.dtype), ptr(out), n, d, stream())
        return a.back(out)

    def save(self, path: str) -> None:
        numpy.savez(path, mean=self.mean.cpu().numpy(), transform=self.transform.cpu().numpy())

    def load(self, path: str) -> None:
        data = numpy.load(path)
        dev = default_device()
        self.mean = torch.from_numpy(data["mean"]).to(dev)
        self.transform = torch.from_numpy(data["transform"]).to(dev)
        self._mean64 = self._trans64 = None


# ---------------------------------------------------------------------------
# dense ops
# ---------------------------------------------------------------------------


def conv(array, kernel, stride=1, pad=0, precision: str | None = None):
    """Cross-correlation of spikes [B, T, C, H, W] with kernel [O, C, KH, KW]."""
    s2, p4 = expand2(stride), expand4(pad)
    if min(s2) < 1:
        raise ValueError("Stride items are incorrect.")
    if min(p4) < 0:
        raise ValueError("Pad items are incorrect.")
    kb = Bound(kernel)
    k = kb.dev.float().contiguous()
    a = Bound(array, k.device)
    x = a.dev
    s = to5(list(x.shape))
    oshape = shape.conv(s, list(k.shape), s2, p4)
    out = torch.empty(oshape, dtype=torch.float32, device=x.device)
    if x.dtype not in (torch.uint8, torch.float32):
        x = x.float()
    prec = _PRECISION[precision or _conv_precision]
    if x.dtype != torch.uint8:
        prec = _PRECISION["fp32"]  # the BF16-split tensor-core path is exact only for u8 spike inputs
    n = s[0] * s[1]
    nb = _lib.lib.spk_conv_workspace(n, s[2], s[3], s[4], k.shape[0], k.shape[2], k.shape[3], prec)
    ws, wsb = _workspace(nb, x.device)
    call("spk_conv", ptr(x), type_code(x.dtype), ptr(k), ptr(out), n, s[2], s[3], s[4], k.shape[0], k.shape[2],
         k.shape[3], s2[0], s2[1], i64(*p4), prec, ptr(ws), wsb, stream())
    return a.back(out)


def fc(array, kernel, sign: bool = False):
    k = Bound(kernel).dev.float().contiguous()
    a = Bound(array, k.device)
    x = a.dev if a.dev.dtype in (torch.uint8, torch.float32) else a.dev.float()
    s = to3(list(x.shape))
    oshape = shape.fc(s, list(k.shape))
    out = torch.empty(oshape, dtype=torch.float32, device=x.device)
    call("spk_fc", ptr(x), type_code(x.dtype), ptr(k), ptr(out), s[0] * s[1], s[2], k.shape[0], int(sign), stream())
    return a.back(out)


def pad(array, pad=0, value: float = 0.0):
    p4 = expand4(pad)
    if min(p4) < 0:
        raise ValueError("Pad items are incorrect.")
    a = Bound(array)
    x = a.dev
    s = to5(list(x.shape))
    oshape = shape.pad(s, p4)
    out = torch.empty(oshape, dtype=x.dtype, device=x.device)
    call("spk_pad", ptr(x), ptr(out), type_code(x.dtype), s[0] * s[1] * s[2], s[3], s[4], i64(*p4), float(value),
         stream())
    return a.back(out)


def threshold(array, threshold: float, value: float = 0.0, inplace: bool = True):
    """In place unless ``inplace=False``: ``x <= threshold -> value``."""
    if not inplace:
        array = clone_array(array)
    a = Bound(array, writeable=True)
    call("spk_threshold", ptr(a.dev), type_code(a.dev.dtype), a.dev.numel(), float(threshold), float(value), stream())
    return a.write_back() if a.kind != "cuda" else array


_threshold_op = threshold


def quantize(array, lower: float, middle: float, upper: float, inplace: bool = True):
    """In place unless ``inplace=False``: ``x < middle -> lower``, else
    ``upper`` (opers.cpp:480-486, cpu/fire.cpp:116-131); the three values
    are converted to the array's type first."""
    if not inplace:
        array = clone_array(array)
    a = Bound(array, writeable=True)
    call("spk_quantize", ptr(a.dev), type_code(a.dev.dtype), a.dev.numel(), float(lower), float(middle), float(upper),
         stream())
    return a.write_back() if a.kind != "cuda" else array


def code(array, time: int, sort: bool = True, dtype: str = "u8", code: str = "rank"):
    """Rank-order (``sort=True``) or latency coding into cumulative spikes;
    ``code="rate"``: Poisson spike counts driven by those times."""
    if code not in ("rank", "rate"):
        raise ValueError(f"Unknown code {code}.")
    if time <= 0:
        raise ValueError("Input time can't be less than 1.")
    a = Bound(array)
    x = a.dev
    s = least2(list(x.shape))
    if x.dtype not in (torch.float32, torch.uint8):
        x = x.float()
    x = x.reshape(s)
    out = torch.empty(shape.code(s, time), dtype=torch_dtype(dtype), device=x.device)
    x_elems = int(numpy.prod(s[1:]))
    if code == "rate":
        ws, wsb = _workspace(_lib.lib.spk_rate_code_workspace(s[0], time, x_elems, int(sort)), x.device)
        call("spk_rate_code", ptr(x), type_code(x.dtype), ptr(out), type_code(out.dtype), s[0], time, x_elems,
             int(sort), ptr(ws), wsb, stream())
        return a.back(out)
    ws, wsb = _workspace(_lib.lib.spk_rank_code_workspace(s[0], x_elems, int(sort)), x.device)
    call("spk_rank_code", ptr(x), type_code(x.dtype), ptr(out), type_code(out.dtype), s[0], time, x_elems, int(sort),
         ptr(ws), wsb, stream())
    return a.back(out)


def infinite(array, value: float = 0.0, inplace: bool = True):
    if not inplace:
        array = clone_array(array)
    a = Bound(array, writeable=True)
    s = least3(list(a.dev.shape))
    call("spk_rank_infinite", ptr(a.dev), type_code(a.dev.dtype), s[0], s[1], int(numpy.prod(s[2:])), float(value),
         stream())
    return a.write_back() if a.kind != "cuda" else array


def fire(array, threshold: float = 0.0, dtype: str = "u8", code: str = "rank"):
    if code not in ("rank", "rate"):
        raise ValueError(f"Unknown code {code}.")
    a = Bound(array)
    x = a.dev.contiguous()
    out = torch.empty(x.shape, dtype=torch_dtype(dtype), device=x.device)
    if code == "rate":
        s = least3(list(x.shape))
        call("spk_rate_fire", ptr(x), type_code(x.dtype), ptr(out), type_code(out.dtype), s[0], s[1],
             int(numpy.prod(s[2:])), float(threshold), stream())
        return a.back(out)
    call("spk_rank_fire", ptr(x), type_code(x.dtype), ptr(out), type_code(out.dtype), x.numel(), float(threshold),
         stream())
    return a.back(out)


def gather(array, threshold: float = 0.0, dtype: str = "u8", code: str = "rank"):
    if code not in ("rank", "rate"):
        raise ValueError(f"Unknown code {code}.")
    a = Bound(array)
    x = a.dev.contiguous()
    s = least3(list(x.shape))
    out = torch.empty(shape.gather(s), dtype=torch_dtype(dtype), device=x.device)
    if code == "rate":
        call("spk_rate_gather", ptr(x), type_code(x.dtype), ptr(out), type_code(out.dtype), s[0], s[1],
             int(numpy.prod(s[2:])), stream())
        return a.back(out)
    call("spk_rank_gather", ptr(x), type_code(x.dtype), ptr(out), type_code(out.dtype), s[0], s[1],
         int(numpy.prod(s[2:])), float(threshold), stream())
    return a.back(out)


def scatter(array, time: int, dtype: str = "u8"):
    if time <= 0:
        raise ValueError("Input time can't be less than 1.")
    a = Bound(array)
    x = a.dev
    s = least2(list(x.shape))
    out = torch.empty(shape.code(s, time), dtype=torch_dtype(dtype), device=x.device)
    call("spk_rank_scatter", ptr(x), type_code(x.dtype), ptr(out), type_code(out.dtype), s[0], time,
         int(numpy.prod(s[1:])), stream())
    return a.back(out)


def pool(array, kernel, stride=None, pad=0, rates=None):
    if rates is not None:
        return _rate_pool(array, kernel, stride, pad, rates)
    k2 = expand2(kernel)
    s2 = expand2(kernel if stride is None else stride)
    p4 = expand4(pad)
    if min(k2) < 1 or min(s2) < 1 or min(p4) < 0:
        raise ValueError("Kernel, stride or pad items are incorrect.")
    a = Bound(array)
    x = a.dev
    s = to5(list(x.shape))
    oshape = shape.pool(s, k2, s2, p4)
    out = torch.empty(oshape, dtype=x.dtype, device=x.device)
    call("spk_rank_pool", ptr(x), ptr(out), type_code(x.dtype), s[0] * s[1] * s[2], s[3], s[4], oshape[3], oshape[4],
         k2[0], k2[1], s2[0], s2[1], i64(*p4), stream())
    return a.back(out)


_pool_op = pool


def _rate_pool(array, kernel, stride, pad, rates):
    """Rate pooling (cpu/pool.cpp:88-137): per window the position of the
    highest rate, its values at every step."""
    k2 = expand2(kernel)
    s2 = expand2(kernel if stride is None else stride)
    p4 = expand4(pad)
    if min(k2) < 1 or min(s2) < 1 or min(p4) < 0:
        raise ValueError("Kernel, stride or pad items are incorrect.")
    a = Bound(array)
    x = a.dev.contiguous()
    s = to5(list(x.shape))
    r = Bound(rates, x.device).dev.contiguous()
    if list(r.shape) != [s[0], s[2], s[3], s[4]]:
        raise ValueError("Rates shape must be [B, C, H, W] of the input.")
    oshape = shape.pool(s, k2, s2, p4)
    out = torch.empty(oshape, dtype=x.dtype, device=x.device)
    call("spk_rate_pool", ptr(x), ptr(r), type_code(x.dtype), type_code(r.dtype), ptr(out), s[0], s[1], s[2], s[3],
         s[4], oshape[3], oshape[4], i64(*k2), i64(*s2), i64(*p4), stream())
    return a.back(out)


def inhibit(array, threshold: float = 0.0, inplace: bool = True):
    if not inplace:
        array = clone_array(array)
    a = Bound(array, writeable=True)
    s = to5(list(a.dev.shape))
    call("spk_rank_inhibit", ptr(a.dev), type_code(a.dev.dtype), s[0], s[1], s[2], s[3] * s[4], float(threshold),
         stream())
    return a.write_back() if a.kind != "cuda" else array


def convwta(array, radius, count: int, threshold: float = 0.0) -> Winners:
    r2 = expand2(radius)
    if min(r2) < 0:
        raise ValueError("Radius items are incorrect.")
    if count <= 0:
        raise ValueError("Winners count can't be less than 1.")
    x = Bound(array).dev
    s = to5(list(x.shape))
    rec = torch.zeros((s[0], count, 5), dtype=torch.int32, device=x.device) if count > 0 else None
    cnt = torch.zeros((s[0],), dtype=torch.int32, device=x.device) if count > 0 else None
    ws, wsb = _workspace(_lib.lib.spk_rank_convwta_workspace(*s), x.device)
    call("spk_rank_convwta", ptr(x), type_code(x.dtype), *s, r2[0], r2[1], count, float(threshold), ptr(rec), ptr(cnt),
         ptr(ws), wsb, stream())
    return Winners(rec, cnt)


def fcwta(array, radius: int, count: int, threshold: float = 0.0) -> Winners:
    if radius < 0:
        raise ValueError("Radius can't be less than 0.")
    if count <= 0:
        raise ValueError("Winners count can't be less than 1.")
    x = Bound(array).dev
    s = to3(list(x.shape))
    rec = torch.zeros((s[0], count, 5), dtype=torch.int32, device=x.device) if count > 0 else None
    cnt = torch.zeros((s[0],), dtype=torch.int32, device=x.device) if count > 0 else None
    ws, wsb = _workspace(_lib.lib.spk_rank_fcwta_workspace(*s), x.device)
    call("spk_rank_fcwta", ptr(x), type_code(x.dtype), *s, radius, count, float(threshold), ptr(rec), ptr(cnt), ptr(ws),
         wsb, stream())
    return Winners(rec, cnt)


def _configs(cfgs) -> "ctypes.Array":
    if len(cfgs) == 0:
        raise ValueError("At least one STDP Config must be given.")
    return _lib.f64([v for c in cfgs for v in c._row()])


def _check_winners(w: Winners, ncfg: int, batch: int) -> None:
    if len(w) == 0:
        raise ValueError("Winners can't be empty.")
    if len(w) != batch:
        raise ValueError("Winners and input batch sizes are not compatible.")
    if w._host is not None:
        for lst in w._host:
            for x in lst:
                if x.c >= ncfg:
                    raise ValueError("STDP configuration index is out of range.")


# ---------------------------------------------------------------------------
# layers
# ---------------------------------------------------------------------------


class Conv:
    """2D convolution layer with STDP (opers.cpp:804-889)."""

    def __init__(self, insize: int, outsize: int, kernel, stride=1, pad=0, mean: float = 0.5, std: float = 0.02,
                 device=None, dtype="f32") -> None:
        if insize <= 0 or outsize <= 0:
            raise ValueError("Input and output sizes can't be less than 1.")
        k2, self._stride, self._pad = expand2(kernel), expand2(stride), expand4(pad)
        if min(k2) < 1 or min(self._stride) < 1 or min(self._pad) < 0:
            raise ValueError("Kernel, stride or pad items are incorrect.")
        w = numpy.zeros(outsize * insize * k2[0] * k2[1], dtype=numpy.float64)
        call("spk_normal_kernel", w.ctypes.data, w.size, float(mean), float(std))
        self.device = _layer_device(device)
        self.kernel = torch.from_numpy(w.reshape(outsize, insize, *k2)).to(torch_dtype(dtype)).to(self.device)
        self.stdpconfig: List[STDPConfig] = []
        self.precision: str | None = None

    def __call__(self, array, threshold: float | None = None):
        if threshold is not None:
            from . import sparse

            return sparse.conv(array, self.kernel, threshold, self._stride, self._pad)
        return conv(array, self.kernel, self._stride, self._pad, self.precision)

    def stdp(self, array, winners, output=None) -> None:
        if output is None:
            from . import sparse

            return sparse.stdp(self, array, winners)
        if self.kernel.dtype != torch.float32:
            raise TypeError("STDP needs an F32 kernel in spyker_b200")
        if len(self.stdpconfig) == 0:
            raise ValueError("At least one STDP Config must be given.")
        x = Bound(array, self.device).dev
        o = Bound(output, self.device).dev
        s, so = to5(list(x.shape)), to5(list(o.shape))
        if x.dtype != o.dtype:
            raise TypeError("Input and output must have the same data type.")
        if so != shape.conv(s, list(self.kernel.shape), self._stride, self._pad):
            raise ValueError("Tensor shapes are not compatible.")
        w = Winners.from_lists(winners, x.device)
        _check_winners(w, len(self.stdpconfig), s[0])
        cout, cin, kh, kw = self.kernel.shape
        ws, wsb = _workspace(_lib.lib.spk_rank_convstdp_workspace(s[0], w.count, cin, s[3], s[4], kh, kw), x.device)
        call("spk_rank_convstdp", ptr(x), type_code(x.dtype), s[0], s[1], cin, s[3], s[4], ptr(self.kernel), cout, kh,
             kw, ptr(o), so[3], so[4], _configs(self.stdpconfig), len(self.stdpconfig), ptr(w.records), ptr(w.counts),
             w.count, self._stride[0], self._stride[1], i64(*self._pad), ptr(ws), wsb, stream())


class FC:
    """Fully connected layer with STDP and the sign-weight backward."""

    def __init__(self, insize: int, outsize: int, mean: float = 0.5, std: float = 0.02, device=None,
                 dtype="f32") -> None:
        if insize <= 0 or outsize <= 0:
            raise ValueError("Input and output sizes can't be less than 1.")
        w = numpy.zeros(outsize * insize, dtype=numpy.float64)
        call("spk_normal_kernel", w.ctypes.data, w.size, float(mean), float(std))
        self.device = _layer_device(device)
        self.kernel = torch.from_numpy(w.reshape(outsize, insize)).to(torch_dtype(dtype)).to(self.device)
        self.stdpconfig: List[STDPConfig] = []
        self.bpconfig = BPConfig()

    def __call__(self, array, sign: bool = False):
        return fc(array, self.kernel, sign)

    def stdp(self, array, winners, output) -> None:
        if len(self.stdpconfig) == 0:
            raise ValueError("At least one STDP Config must be given.")
        x = Bound(array, self.device).dev
        o = Bound(output, self.device).dev
        s, so = to3(list(x.shape)), to3(list(o.shape))
        if so != shape.fc(s, list(self.kernel.shape)):
            raise ValueError("Tensor shapes are not compatible.")
        w = Winners.from_lists(winners, x.device)
        _check_winners(w, len(self.stdpconfig), s[0])
        ws, wsb = _workspace(_lib.lib.spk_rank_fcstdp_workspace(s[0], s[1], s[2]), x.device)
        call("spk_rank_fcstdp", ptr(x), type_code(x.dtype), s[0], s[1], s[2], ptr(self.kernel), self.kernel.shape[0],
             ptr(o), _configs(self.stdpconfig), len(self.stdpconfig), ptr(w.records), ptr(w.counts), w.count, ptr(ws),
             wsb, stream())

    def backward(self, array, output, grad):
        x = Bound(array, self.device)
        o = Bound(output, self.device).dev.float().contiguous()
        g = Bound(grad, self.device).dev.float().contiguous()
        xi = x.dev.float().contiguous()
        b = xi.shape[0]
        nxt = torch.empty(xi.shape, dtype=torch.float32, device=xi.device)
        no, ni = self.kernel.shape
        bp = (numpy.array([self.bpconfig.sfactor, self.bpconfig.lrate, self.bpconfig.lrf, self.bpconfig.lamda],
                          dtype=numpy.float32))
        ws, wsb = _workspace(_lib.lib.spk_fcbackward_workspace(no, ni), xi.device)
        call("spk_fcbackward", ptr(self.kernel), no, ni, ptr(xi), ptr(o), ptr(g), ptr(nxt), b, bp.ctypes.data, ptr(ws),
             wsb, stream())
        self.bpconfig.sfactor = float(bp[0])
        return x.back(nxt)


def conv_fire_wta(array, conv: "Conv", threshold: float, radius, count: int, value: float = 0.0,
                  inhibit_threshold: float = 0.0, fire_threshold: float = 0.0, wta_threshold: float = 0.0,
                  precision: str | None = None, pool=None):
    """One fused layer step; returns ``(spikes, winners)`` equal to::

        out = inhibit(threshold(conv(array), threshold, value), inhibit_threshold)
        spikes, winners = fire(out, fire_threshold), convwta(out, radius, count, wta_threshold)

    With ``pool`` (a window, stride = window, no padding) it returns
    ``(spikes, winners, pool(spikes, pool))``, the pooled spikes written by the
    same kernel.  ``count=0`` skips the winner selection (forward passes);
    winners is then None.

    On the tensor-core precisions with u8 spikes, T <= 32, at least two output
    channels and non-negative fire/WTA thresholds, a single tcgen05 kernel does
    it without writing the potentials; otherwise the ops run one by one.
    """
    r2 = expand2(radius)
    prec = precision or conv.precision or _conv_precision
    x = Bound(array, conv.device).dev
    s = to5(list(x.shape))
    k = conv.kernel if conv.kernel.dtype == torch.float32 else conv.kernel.float()
    k = k.contiguous()
    cout, cin, kh, kw = k.shape
    if count < 0:
        raise ValueError("Winners count can't be less than 0.")
    fused = (prec != "fp32" and x.dtype == torch.uint8 and s[1] <= 32 and cout >= 2 and fire_threshold >= 0
             and wta_threshold >= 0 and min(r2) >= 0)
    if fused:
        oshape = shape.conv(s, list(k.shape), conv._stride, conv._pad)
        nb = _lib.lib.spk_conv_fire_wta_workspace(s[0], s[1], cin, s[3], s[4], cout, kh, kw, conv._stride[0],
                                                  conv._stride[1], i64(*conv._pad), _PRECISION[prec])
        fused = nb > 0 and s[1] * cout * (128 // (1 << (s[1] - 1).bit_length())) <= 32768
    p2 = expand2(pool) if pool is not None else None
    if p2 is not None and min(p2) < 1:
        raise ValueError("Kernel, stride or pad items are incorrect.")
    if not fused:
        out = inhibit(_threshold_op(conv_(x, conv, prec), threshold, value), inhibit_threshold)
        spk = fire(out, fire_threshold)
        wins = convwta(out, r2, count, wta_threshold) if count > 0 else None
        return (spk, wins) if p2 is None else (spk, wins, _pool_op(spk, p2))
    spikes = torch.empty(oshape, dtype=torch.uint8, device=x.device)
    pooled = None
    if p2 is not None:
        pooled = torch.empty(shape.pool(oshape, p2, p2, (0, 0, 0, 0)), dtype=torch.uint8, device=x.device)
    rec = torch.zeros((s[0], count, 5), dtype=torch.int32, device=x.device) if count > 0 else None
    cnt = torch.zeros((s[0],), dtype=torch.int32, device=x.device) if count > 0 else None
    ws, wsb = _workspace(nb, x.device)
    call("spk_conv_fire_wta", ptr(x), type_code(x.dtype), ptr(k), s[0], s[1], cin, s[3], s[4], cout, kh, kw,
         conv._stride[0], conv._stride[1], i64(*conv._pad), float(threshold), float(value), float(inhibit_threshold),
         float(fire_threshold), r2[0], r2[1], count, float(wta_threshold), ptr(spikes), ptr(rec), ptr(cnt),
         p2[0] if p2 else 0, p2[1] if p2 else 0, ptr(pooled), _PRECISION[prec], ptr(ws), wsb, stream())
    wins = Winners(rec, cnt) if count > 0 else None
    return (spikes, wins) if p2 is None else (spikes, wins, pooled)


def conv_(x, layer: "Conv", prec: str):
    return conv(x, layer.kernel, layer._stride, layer._pad, prec)


def stdp(conv: Conv, array, winners, output) -> None:
    """Low-level STDP helper (module.py:1325): same as ``conv.stdp``."""
    conv.stdp(array, winners, output)


def backward(array, target, time: int, gamma: float):
    if time <= 0:
        raise ValueError("Time steps must be higher than zero.")
    a = Bound(array)
    x = a.dev.float().contiguous()
    t = Bound(target, x.device).dev
    if t.dtype != torch.int64:
        raise TypeError("Target type must have I64 type.")
    if t.shape[0] != x.shape[0]:
        raise ValueError("Input and target shapes are not compatible.")
    out = torch.empty_like(x)
    call("spk_backward", ptr(x), ptr(out), ptr(t), x.shape[0], x[0].numel(), time, float(gamma), stream())
    return a.back(out)


def labelize(array, threshold: float):
    a = Bound(array)
    x = a.dev.float().contiguous() if a.dev.dtype != torch.float32 else a.dev
    out = torch.empty((x.shape[0],), dtype=torch.int64, device=x.device)
    call("spk_labelize", ptr(x), type_code(x.dtype), ptr(out), x.shape[0], x.shape[1], x[0, 0].numel(),
         float(threshold), stream())
    return a.back(out)


def canny(array, low: float, high: float):
    """Canny edges of u8 images (opers.cpp:223-243, cpu/canny.cpp:9-214):
    ``[N, C, H, W]`` (or 3-D) in, u8 of the same shape out.  As in the
    reference, the output is u8 and must have the input's type, so the
    input must be u8; ``low`` and ``high`` are converted to u8."""
    a = Bound(array)
    x = a.dev
    s4 = to4(list(x.shape))
    if x.dtype != torch.uint8:
        raise TypeError("Input and output must have the same type.")
    n, h, w = s4[0] * s4[1], s4[2], s4[3]
    out = torch.empty(x.shape, dtype=torch.uint8, device=x.device)
    ws, nb = _workspace(int(_lib.lib.spk_canny_workspace(n, h, w)), x.device)
    call("spk_canny", ptr(x), ptr(out), n, h, w, float(low), float(high), ptr(ws), nb, stream())
    return a.back(out)
