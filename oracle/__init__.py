"""ORACLE — test infrastructure only (the checker, never the product).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
legs may import this package.  It wraps two CPU libraries with one ABI:

* ``port``      — ``oracle/_build/liboracle_port.so``: this project's C++
  restatement of Spyker's CPU algorithms (``oracle/spyker_oracle.cpp``);
* ``reference`` — ``oracle/_ref/libspyker_ref.so``: Spyker's own CPU backend
  compiled from the reference sources (``oracle/Makefile``), with FP64
  direct loops standing in for the absent oneDNN/BLAS convolution.

All functions take and return NumPy arrays with the reference layouts
(spikes ``[B, T, C, H, W]`` etc.).
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_PATH = os.path.join(HERE, "_build", "liboracle_port.so")
REF_PATH = os.path.join(HERE, "_ref", "libspyker_ref.so")

# Type codes of the reference's `enum class Type` (utils.h:96-120).
_CODES = {
    np.dtype(np.int8): 0,
    np.dtype(np.int16): 1,
    np.dtype(np.int32): 2,
    np.dtype(np.int64): 3,
    np.dtype(np.uint8): 4,
    np.dtype(np.uint16): 5,
    np.dtype(np.uint32): 6,
    np.dtype(np.uint64): 7,
    np.dtype(np.float16): 8,
    np.dtype(np.float32): 9,
    np.dtype(np.float64): 10,
}

_P = C.c_void_p
_I = C.c_int64
_D = C.c_double


def build(force: bool = False) -> None:
    """Compile the checkers (``make -C oracle``)."""
    if force or not os.path.exists(PORT_PATH):
        subprocess.check_call(["make", "-C", HERE, "-j8", "all"])


def _i64(*v) -> np.ndarray:
    return np.ascontiguousarray(np.array(v, dtype=np.int64))


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class Oracle:
    """One of the two CPU checkers behind a NumPy interface."""

    def __init__(self, kind: str = "port"):
        path = PORT_PATH if kind == "port" else REF_PATH
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library {path} is not built (run `make -C oracle`)")
        self.kind = kind
        self.lib = C.CDLL(path)
        self.lib.orc_last_error.restype = C.c_char_p
        self.lib.orc_free.argtypes = [_P]

    # -- helpers ---------------------------------------------------------
    def _call(self, name: str, *args) -> None:
        fn = getattr(self.lib, name)
        conv = []
        for a in args:
            if isinstance(a, np.ndarray):
                conv.append(_P(_ptr(a)))
            elif isinstance(a, float):
                conv.append(_D(a))
            elif isinstance(a, (bool, int, np.integer)):
                conv.append(_I(int(a)))
            else:
                conv.append(a)
        fn.restype = C.c_int
        # The int-typed flags (itype/otype/sort/which) are passed as int64,
        # which is ABI-compatible with `int` on x86-64 SysV.
        if fn(*conv) != 0:
            raise RuntimeError(self.lib.orc_last_error().decode())

    @staticmethod
    def _c(a, dtype=None) -> np.ndarray:
        return np.ascontiguousarray(a if dtype is None else np.asarray(a, dtype=dtype))

    def _events_out(self, name: str, u: int, t: int, *args):
        off = C.POINTER(C.c_int64)()
        zyx = C.POINTER(C.c_uint8)()
        conv = list(args) + [C.byref(off), C.byref(zyx)]
        self._call(name, *conv)
        n = u * t
        offs = np.ctypeslib.as_array(off, shape=(n + 1,)).copy()
        total = int(offs[-1])
        data = np.ctypeslib.as_array(zyx, shape=(max(total, 1) * 3,))[: total * 3].copy().reshape(total, 3)
        self.lib.orc_free(C.cast(off, _P))
        self.lib.orc_free(C.cast(zyx, _P))
        return offs, data

    # -- dense ops -------------------------------------------------------
    def rank_code(self, x, time: int, sort: bool = True, dtype=np.uint8) -> np.ndarray:
        x = self._c(x)
        b = x.shape[0]
        flat = x.reshape(b, -1)
        out = np.zeros((b, time, flat.shape[1]), dtype=dtype)
        self._call("orc_rank_code", flat, _CODES[flat.dtype], out, _CODES[out.dtype], b, time, flat.shape[1], int(sort))
        return out.reshape((b, time) + x.shape[1:])

    def threshold(self, x, thr: float, value: float = 0.0) -> np.ndarray:
        x = self._c(x).copy()
        self._call("orc_threshold", x, _CODES[x.dtype], x.size, float(thr), float(value))
        return x

    def infinite(self, x, value: float = 0.0) -> np.ndarray:
        x = self._c(x).copy()
        self._call("orc_rank_infinite", x, _CODES[x.dtype], x.shape[0], x.shape[1], x[0, 0].size, float(value))
        return x

    def fire(self, x, thr: float = 0.0, dtype=np.uint8) -> np.ndarray:
        x = self._c(x)
        out = np.zeros(x.shape, dtype=dtype)
        self._call("orc_rank_fire", x, _CODES[x.dtype], out, _CODES[out.dtype], x.size, float(thr))
        return out

    def gather(self, x, thr: float = 0.0, dtype=np.uint8) -> np.ndarray:
        x = self._c(x)
        b, t = x.shape[:2]
        out = np.zeros((b,) + x.shape[2:], dtype=dtype)
        self._call("orc_rank_gather", x, _CODES[x.dtype], out, _CODES[out.dtype], b, t, x[0, 0].size, float(thr))
        return out

    def scatter(self, x, time: int, dtype=np.uint8) -> np.ndarray:
        x = self._c(x)
        b = x.shape[0]
        out = np.zeros((b, time) + x.shape[1:], dtype=dtype)
        self._call("orc_rank_scatter", x, _CODES[x.dtype], out, _CODES[out.dtype], b, time, x[0].size)
        return out

    def pad(self, x, pad4, value: float = 0.0) -> np.ndarray:
        x = self._c(x)
        h, w = x.shape[-2:]
        n = x.size // (h * w)
        out = np.zeros(x.shape[:-2] + (h + pad4[0] + pad4[2], w + pad4[1] + pad4[3]), dtype=x.dtype)
        self._call("orc_pad", x, out, _CODES[x.dtype], n, h, w, _i64(*pad4), float(value))
        return out

    def pool(self, x, kernel2, stride2=None, pad4=(0, 0, 0, 0)) -> np.ndarray:
        x = self._c(x)
        stride2 = kernel2 if stride2 is None else stride2
        h, w = x.shape[-2:]
        oh = (h + pad4[0] + pad4[2] - kernel2[0]) // stride2[0] + 1
        ow = (w + pad4[1] + pad4[3] - kernel2[1]) // stride2[1] + 1
        n = x.size // (h * w)
        out = np.zeros(x.shape[:-2] + (oh, ow), dtype=x.dtype)
        self._call("orc_rank_pool", x, out, _CODES[x.dtype], n, 1, h, w, oh, ow, _i64(*kernel2), _i64(*stride2),
                   _i64(*pad4))
        return out

    def inhibit(self, x, thr: float = 0.0) -> np.ndarray:
        x = self._c(x).copy()
        b, t, c = x.shape[:3]
        self._call("orc_rank_inhibit", x, _CODES[x.dtype], b, t, c, x[0, 0, 0].size, float(thr))
        return x

    def convwta(self, x, radius2, count: int, thr: float = 0.0):
        x = self._c(x)
        b, t, c, h, w = x.shape
        win = np.zeros((b, count, 5), dtype=np.int64)
        cnt = np.zeros(b, dtype=np.int64)
        self._call("orc_rank_convwta", x, _CODES[x.dtype], b, t, c, h, w, _i64(*radius2), count, float(thr), win, cnt)
        return win, cnt

    def fcwta(self, x, radius: int, count: int, thr: float = 0.0):
        x = self._c(x)
        b, t, n = x.shape
        win = np.zeros((b, count, 5), dtype=np.int64)
        cnt = np.zeros(b, dtype=np.int64)
        self._call("orc_rank_fcwta", x, _CODES[x.dtype], b, t, n, radius, count, float(thr), win, cnt)
        return win, cnt

    def convstdp(self, x, kernel, out, configs, winners, counts, stride2=(1, 1), pad4=(0, 0, 0, 0)) -> np.ndarray:
        """Returns the updated kernel (input kernel untouched)."""
        x, out = self._c(x), self._c(out)
        kernel = self._c(kernel).copy()
        b, t, cin, h, w = x.shape
        cout, _, kh, kw = kernel.shape
        oh, ow = out.shape[-2:]
        cfg = np.ascontiguousarray(np.array(configs, dtype=np.float64).reshape(-1, 5))
        winners = self._c(winners, np.int64)
        counts = self._c(counts, np.int64)
        self._call("orc_rank_convstdp", x, _CODES[x.dtype], b, t, cin, h, w, kernel, _CODES[kernel.dtype], cout, kh, kw,
                   out, oh, ow, cfg, cfg.shape[0], winners, counts, winners.shape[1], _i64(*stride2), _i64(*pad4))
        return kernel

    def fcstdp(self, x, kernel, out, configs, winners, counts) -> np.ndarray:
        x, out = self._c(x), self._c(out)
        kernel = self._c(kernel).copy()
        b, t, ni = x.shape
        no = kernel.shape[0]
        cfg = np.ascontiguousarray(np.array(configs, dtype=np.float64).reshape(-1, 5))
        winners = self._c(winners, np.int64)
        counts = self._c(counts, np.int64)
        self._call("orc_rank_fcstdp", x, _CODES[x.dtype], b, t, ni, kernel, _CODES[kernel.dtype], no, out, cfg,
                   cfg.shape[0], winners, counts, winners.shape[1])
        return kernel

    def conv(self, x, kernel, stride2=(1, 1), pad4=(0, 0, 0, 0), out_dtype=None) -> np.ndarray:
        """Dense conv of ``x`` ``[..., C, H, W]`` (leading dims folded)."""
        x, kernel = self._c(x), self._c(kernel)
        cin, h, w = x.shape[-3:]
        n = x.size // (cin * h * w)
        cout, _, kh, kw = kernel.shape
        oh = (h + pad4[0] + pad4[2] - kh) // stride2[0] + 1
        ow = (w + pad4[1] + pad4[3] - kw) // stride2[1] + 1
        out = np.zeros(x.shape[:-3] + (cout, oh, ow), dtype=out_dtype or kernel.dtype)
        self._call("orc_conv", x, _CODES[x.dtype], kernel, _CODES[kernel.dtype], out, _CODES[out.dtype], n, cin, h, w,
                   cout, kh, kw, oh, ow, _i64(*stride2), _i64(*pad4))
        return out

    def fc(self, x, kernel, sign: bool = False, out_dtype=None) -> np.ndarray:
        x, kernel = self._c(x), self._c(kernel)
        b, t, ni = x.shape
        no = kernel.shape[0]
        out = np.zeros((b, t, no), dtype=out_dtype or kernel.dtype)
        self._call("orc_fc", x, _CODES[x.dtype], kernel, _CODES[kernel.dtype], out, _CODES[out.dtype], b, t, ni, no,
                   int(sign))
        return out

    def filter(self, which: str, x, kernel, pad4=(0, 0, 0, 0)) -> np.ndarray:
        """DoG / Gabor / LoG of ``x`` ``[B, C, H, W]`` -> ``[B, C*F(*2), OH, OW]``."""
        code = {"dog": 0, "gabor": 1, "log": 2}[which]
        x, kernel = self._c(x, kernel.dtype), self._c(kernel)
        b, c, h, w = x.shape
        kh, kw = kernel.shape[-2:]
        f = kernel.shape[0] if which == "gabor" else kernel.shape[1]
        oh = h + pad4[0] + pad4[2] - kh + 1
        ow = w + pad4[1] + pad4[3] - kw + 1
        fo = 2 * f if which == "log" else f
        out = np.zeros((b, c * fo, oh, ow), dtype=kernel.dtype)
        self._call("orc_filter", code, x, kernel, out, _CODES[kernel.dtype], b * c, h, w, f, kh, kw, oh, ow,
                   _i64(*pad4))
        return out

    def gaussian_kernel(self, size: int, std: float) -> np.ndarray:
        k = np.zeros((size, size), dtype=np.float64)
        self._call("orc_gaussian_kernel", k, size, float(std))
        return k

    def gabor_kernel(self, size: int, sigma, theta, gamma, lambda_, psi) -> np.ndarray:
        k = np.zeros((size, size), dtype=np.float64)
        self._call("orc_gabor_kernel", k, size, float(sigma), float(theta), float(gamma), float(lambda_), float(psi))
        return k

    def log_kernel(self, size: int, std: float) -> np.ndarray:
        k = np.zeros((size, size), dtype=np.float64)
        self._call("orc_log_kernel", k, size, float(std))
        return k

    def backward(self, x, target, time: int, gamma: float) -> np.ndarray:
        x = self._c(x)
        target = self._c(target, np.int64)
        out = np.zeros_like(x)
        self._call("orc_backward", x, out, _CODES[x.dtype], target, x.shape[0], x.shape[1], time, float(gamma))
        return out

    def labelize(self, x, thr: float) -> np.ndarray:
        x = self._c(x)
        b, t = x.shape[:2]
        out = np.zeros(b, dtype=np.int64)
        self._call("orc_labelize", x, _CODES[x.dtype], out, b, t, x[0, 0].size, float(thr))
        return out

    def fcbackward(self, kernel, x, out, grad, bp):
        """Returns (updated kernel, next-gradient, updated sfactor)."""
        kernel = self._c(kernel, np.float32).copy()
        x, out, grad = self._c(x), self._c(out), self._c(grad)
        nxt = np.zeros_like(x)
        bpa = np.ascontiguousarray(np.array(bp, dtype=np.float32))
        no, ni = kernel.shape
        self._call("orc_fcbackward", kernel, no, ni, x, out, grad, nxt, _CODES[x.dtype], x.shape[0], bpa)
        return kernel, nxt, float(bpa[0])

    # -- rate coding -------------------------------------------------------
    def poisson_table(self, time: int, bins: int = 1024) -> np.ndarray:
        out = np.zeros((time, bins), dtype=np.uint16)
        self._call("orc_poisson_table", time, bins, out)
        return out

    def rate_code(self, x, time: int, sort: bool = True, dtype=np.uint8) -> np.ndarray:
        x = self._c(x)
        b = x.shape[0]
        out = np.zeros((b, time) + x.shape[1:], dtype=dtype)
        self._call("orc_rate_code", x, _CODES[x.dtype], out, _CODES[out.dtype], b, time, x[0].size, int(sort))
        return out

    def rate_fire(self, x, thr: float = 0.0, dtype=np.uint8) -> np.ndarray:
        x = self._c(x)
        b, t = x.shape[:2]
        out = np.zeros(x.shape, dtype=dtype)
        self._call("orc_rate_fire", x, _CODES[x.dtype], out, _CODES[out.dtype], b, t, x[0, 0].size, float(thr))
        return out

    def rate_gather(self, x, dtype=np.uint8) -> np.ndarray:
        x = self._c(x)
        b, t = x.shape[:2]
        out = np.zeros((b,) + x.shape[2:], dtype=dtype)
        self._call("orc_rate_gather", x, _CODES[x.dtype], out, _CODES[out.dtype], b, t, x[0, 0].size)
        return out

    def rate_pool(self, x, rates, kernel2, stride2=None) -> np.ndarray:
        x, rates = self._c(x), self._c(rates)
        stride2 = stride2 or kernel2
        b, t, c, h, w = x.shape
        oh = (h - kernel2[0]) // stride2[0] + 1
        ow = (w - kernel2[1]) // stride2[1] + 1
        out = np.zeros((b, t, c, oh, ow), dtype=x.dtype)
        self._call("orc_rate_pool", x, rates, _CODES[x.dtype], _CODES[rates.dtype], out, b, t, c, h, w, oh, ow,
                   _i64(*kernel2), _i64(*stride2))
        return out

    # -- data helpers (reference build only) -----------------------------
    def csv_rows(self, path: str, delim: str = ", ", skip: int = 0, max_rows: int = 1 << 20):
        """(skipped, rows) read by Helper::CSV (helper/csv.cpp:10-70)."""
        cap = max(os.path.getsize(path) * 2 + 64, 64) if os.path.exists(path) else 64
        out = C.create_string_buffer(cap)
        ln, sk = C.c_int64(), C.c_int64()
        fn = self.lib.orc_ref_csv
        fn.restype = C.c_int
        if fn(path.encode(), delim.encode(), _I(skip), _I(max_rows), out, _I(cap), C.byref(ln), C.byref(sk)) != 0:
            raise RuntimeError(self.lib.orc_last_error().decode())
        raw = out.raw[: ln.value].decode()
        return sk.value, [r.split("\x1f") for r in raw.split("\x1e")[:-1]]

    def idx(self, path: str, labels: bool):
        """Helper::mnistLabel / mnistData (helper/mnist.cpp:31-60): None for
        the empty tensor, else the u8 array."""
        cap = os.path.getsize(path) if os.path.exists(path) else 0
        out = np.zeros(max(cap, 1), dtype=np.uint8)
        shape, ndim = np.zeros(4, dtype=np.int64), C.c_int64()
        fn = self.lib.orc_ref_idx
        fn.restype = C.c_int
        if fn(path.encode(), _I(int(labels)), _P(_ptr(out)), _I(cap), _P(_ptr(shape)), C.byref(ndim)) != 0:
            raise RuntimeError(self.lib.orc_last_error().decode())
        if ndim.value == 0:
            return None
        dims = tuple(int(v) for v in shape[: ndim.value])
        return out[: int(np.prod(dims))].reshape(dims).copy()

    def canny(self, x, low: float, high: float) -> np.ndarray:
        """cpu/canny.cpp on u8 images [..., H, W] (reference build only)."""
        x = self._c(x, np.uint8)
        h, w = x.shape[-2:]
        n = int(np.prod(x.shape[:-2]))
        out = np.zeros_like(x)
        self._call("orc_ref_canny", x, out, n, h, w, float(low), float(high))
        return out

    def quantize(self, x, lower: float, middle: float, upper: float) -> np.ndarray:
        """cpu/fire.cpp:116-131 on a copy (reference build only)."""
        x = self._c(x).copy()
        self._call("orc_ref_quantize", x, _CODES[x.dtype], x.size, float(lower), float(middle), float(upper))
        return x

    def zca_fit(self, x, epsilon: float, transform: bool = False):
        """cpu/zca.cpp:67-105 on samples [N, ...] (F32/F64; reference build
        only): (mean [D], trans [D, D], x whitened in place if `transform`)."""
        x = self._c(x).copy()
        n, d = x.shape[0], int(np.prod(x.shape[1:]))
        mean = np.zeros(d, dtype=x.dtype)
        trans = np.zeros((d, d), dtype=x.dtype)
        self._call("orc_ref_zca_fit", x, _CODES[x.dtype], n, d, mean, trans, float(epsilon), int(transform))
        return mean, trans, x

    def zca_trans(self, x, mean, trans):
        """cpu/zca.cpp:107-118: (x - mean) trans on a copy (reference build only)."""
        x = self._c(x).copy()
        n, d = x.shape[0], int(np.prod(x.shape[1:]))
        mean = np.ascontiguousarray(mean, dtype=x.dtype)
        trans = np.ascontiguousarray(trans, dtype=x.dtype)
        self._call("orc_ref_zca_trans", x, _CODES[x.dtype], n, d, mean, trans)
        return x

    def zca_split(self, x):
        """cpu/zca.cpp:139-155: [N, ...] -> [N, 2, ...] (reference build only)."""
        x = self._c(x)
        n, d = x.shape[0], int(np.prod(x.shape[1:]))
        out = np.zeros((n, 2) + x.shape[1:], dtype=x.dtype)
        self._call("orc_ref_zca_split", x, _CODES[x.dtype], n, d, out)
        return out

    # -- sparse event lists (offsets [U*T+1], zyx [N, 3]) -----------------
    def sparse_code(self, x, time: int, sort: bool = True):
        x = self._c(x)
        u, c, h, w = x.shape
        return self._events_out("orc_sparse_code", u, time, x, _CODES[x.dtype], u, c, h, w, time, int(sort))

    def sparse_from_dense(self, x, thr: float = 0.0):
        x = self._c(x)
        u, t, c, h, w = x.shape
        return self._events_out("orc_sparse_from_dense", u, t, x, _CODES[x.dtype], u, t, c, h, w, float(thr))

    def sparse_to_dense(self, ev, shape, dtype=np.uint8) -> np.ndarray:
        off, zyx = ev
        out = np.zeros(shape, dtype=dtype)
        self._call("orc_sparse_to_dense", self._c(off, np.int64), self._c(zyx, np.uint8), *shape, out,
                   _CODES[out.dtype])
        return out

    def sparse_gather(self, ev, shape, dtype=np.uint8) -> np.ndarray:
        off, zyx = ev
        u, t, c, h, w = shape
        out = np.zeros((u, c, h, w), dtype=dtype)
        self._call("orc_sparse_gather", self._c(off, np.int64), self._c(zyx, np.uint8), u, t, c, h, w, out,
                   _CODES[out.dtype])
        return out

    def sparse_conv(self, ev, shape, kernel, thr: float, pad4=(0, 0, 0, 0)):
        off, zyx = ev
        u, t, c, h, w = shape
        kernel = self._c(kernel, np.float32)
        cout, _, kh, kw = kernel.shape
        oh = h + pad4[0] + pad4[2] - kh + 1
        ow = w + pad4[1] + pad4[3] - kw + 1
        res = self._events_out("orc_sparse_conv", u, t, self._c(off, np.int64), self._c(zyx, np.uint8), u, t, c, h, w,
                               kernel, cout, kh, kw, float(thr), _i64(1, 1), _i64(*pad4), oh, ow)
        return res, (u, t, cout, oh, ow)

    def sparse_pad(self, ev, shape, pad4):
        off, zyx = ev
        u, t, c, h, w = shape
        res = self._events_out("orc_sparse_pad", u, t, self._c(off, np.int64), self._c(zyx, np.uint8), u, t, c, h, w,
                               _i64(*pad4))
        return res, (u, t, c, h + pad4[0] + pad4[2], w + pad4[1] + pad4[3])

    def sparse_pool(self, ev, shape, kernel2, pad4=(0, 0, 0, 0)):
        off, zyx = ev
        u, t, c, h, w = shape
        oh = (h + pad4[0] + pad4[2] - kernel2[0]) // kernel2[0] + 1
        ow = (w + pad4[1] + pad4[3] - kernel2[1]) // kernel2[1] + 1
        res = self._events_out("orc_sparse_pool", u, t, self._c(off, np.int64), self._c(zyx, np.uint8), u, t, c, h, w,
                               _i64(*kernel2), _i64(*kernel2), _i64(*pad4), oh, ow)
        return res, (u, t, c, oh, ow)

    def sparse_inhibit(self, ev, shape):
        off, zyx = ev
        return self._events_out("orc_sparse_inhibit", shape[0], shape[1], self._c(off, np.int64),
                                self._c(zyx, np.uint8), *shape)

    def sparse_convwta(self, ev, shape, radius2, count: int):
        off, zyx = ev
        u = shape[0]
        win = np.zeros((u, count, 5), dtype=np.int64)
        cnt = np.zeros(u, dtype=np.int64)
        self._call("orc_sparse_convwta", self._c(off, np.int64), self._c(zyx, np.uint8), *shape, _i64(*radius2), count,
                   win, cnt)
        return win, cnt

    def sparse_stdp(self, ev, shape, kernel, configs, winners, counts, pad4=(0, 0, 0, 0)) -> np.ndarray:
        off, zyx = ev
        kernel = self._c(kernel, np.float32).copy()
        cout, _, kh, kw = kernel.shape
        cfg = np.ascontiguousarray(np.array(configs, dtype=np.float64).reshape(-1, 5))
        winners = self._c(winners, np.int64)
        counts = self._c(counts, np.int64)
        self._call("orc_sparse_stdp", self._c(off, np.int64), self._c(zyx, np.uint8), *shape, kernel, cout, kh, kw, cfg,
                   cfg.shape[0], winners, counts, winners.shape[1], _i64(*pad4))
        return kernel


_cache: dict = {}


def get(kind: str = "port") -> Oracle:
    if kind not in _cache:
        _cache[kind] = Oracle(kind)
    return _cache[kind]


def available(kind: str) -> bool:
    return os.path.exists(PORT_PATH if kind == "port" else REF_PATH)
