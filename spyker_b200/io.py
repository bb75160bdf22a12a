"""Data input and output: MNIST IDX files into pinned host memory, batches
copied to the GPU on a side stream ahead of use, results read back on
another, CSV lines, and the examples' ``.npz`` kernel checkpoints.

Reference: helper/mnist.cpp:10-60 and utils.py:532-560 (``read_mnist``),
helper/csv.cpp:10-70 and bind.cpp:103-108 (``read_csv``),
examples/kheradpisheh_mnist_dense.py:81-89 (checkpoints).
"""

from __future__ import annotations

import ctypes
import os
from typing import Iterator, List, Optional, Sequence, Tuple

import numpy
import torch

from . import _lib


def _idx(path: str, magic: int) -> torch.Tensor:
    shape = (ctypes.c_int64 * 4)()
    ndim, offset = ctypes.c_int64(), ctypes.c_int64()
    p = os.fsencode(path)
    if _lib.lib.spk_idx_shape(p, magic, shape, ctypes.byref(ndim), ctypes.byref(offset)) != 0:
        return torch.empty(0, dtype=torch.uint8)
    dims = tuple(int(shape[i]) for i in range(ndim.value))
    out = torch.empty(dims, dtype=torch.uint8, pin_memory=torch.cuda.is_available())
    threads = min(8, os.cpu_count() or 1)
    if _lib.lib.spk_idx_read(p, offset.value, ctypes.c_void_p(out.data_ptr()), out.numel(), threads) != 0:
        return torch.empty(0, dtype=torch.uint8)
    return out


def mnist_data(path: str) -> torch.Tensor:
    """Images of an IDX file (magic 2051) as u8 [N, 1, rows, cols] in pinned
    host memory; an empty tensor when the file cannot be read, like
    ``Helper::mnistData``."""
    return _idx(path, 2051)


def mnist_label(path: str) -> torch.Tensor:
    """Labels of an IDX file (magic 2049) as u8 [N]; empty on failure."""
    return _idx(path, 2049)


def read_mnist(train_images: str, train_labels: str, test_images: str,
               test_labels: str) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor]:
    """(train images, train labels, test images, test labels)."""
    return mnist_data(train_images), mnist_label(train_labels), mnist_data(test_images), mnist_label(test_labels)


def write_idx(path: str, array) -> None:
    """Write u8 images [N, 1, rows, cols] / [N, rows, cols] (magic 2051) or
    labels [N] (magic 2049) in the IDX layout the reader takes."""
    a = numpy.ascontiguousarray(array.cpu().numpy() if torch.is_tensor(array) else array, dtype=numpy.uint8)
    if a.ndim == 1:
        head = [2049, a.shape[0]]
    elif a.ndim in (3, 4):
        head = [2051, a.shape[0], a.shape[-2], a.shape[-1]]
    else:
        raise ValueError("IDX arrays are [N] labels or [N, (1,) rows, cols] images")
    with open(path, "wb") as f:
        f.write(numpy.asarray(head, dtype=">i4").tobytes())
        f.write(a.tobytes())


class CSV:
    """Line reader of a delimited text file (helper/csv.cpp:10-70).

    A field ends at each occurrence of ``delim`` and the next one starts one
    character later, as in the reference, so with the default ``", "`` the
    fields after the first keep the space that follows the comma."""

    def __init__(self, path: str, delim: str = ", "):
        self.delim = delim
        try:
            self._file = open(path, "r", newline="")
        except OSError:
            self._file = None

    def _line(self) -> Optional[str]:
        if self._file is None:
            return None
        line = self._file.readline()
        if line == "":
            return None
        return line[:-1] if line.endswith("\n") else line

    def _split(self, line: str) -> List[str]:
        row, prev = [], 0
        while True:
            index = line.find(self.delim, prev)
            if index < 0:
                row.append(line[prev:])
                return row
            row.append(line[prev:index])
            prev = index + 1

    def readline(self) -> Tuple[bool, List[str]]:
        """(False, []) at the end; blank lines are skipped."""
        while True:
            line = self._line()
            if line is None:
                return False, []
            if line:
                return True, self._split(line)

    def skip(self, lines: int) -> int:
        """Skip up to ``lines`` lines; returns how many were skipped."""
        done = 0
        while done < lines and self._line() is not None:
            done += 1
        return done


def read_csv(path: str, delim: str = ", ") -> Tuple[bool, Sequence[str]]:
    """(ok, fields) of the first non-blank line, as the reference's binding."""
    return CSV(path, delim).readline()


class Prefetcher:
    """Batches of host data delivered on the GPU, each copied on a side
    stream while the batches before it are processed.

    ``source`` is a host tensor split into batches of ``batch`` samples
    (the last one ragged) or a sequence of host tensors, one per batch; it
    should be in pinned host memory (``read_mnist`` returns it so).  Batch
    ``k`` is a view of one of ``depth`` device buffers and stays valid until
    batch ``k + depth - 1`` is requested: the work queued on the consumer's
    stream between two requests is what a buffer waits for before it is
    refilled, so no host synchronisation happens."""

    def __init__(self, source, batch: Optional[int] = None, device=None, depth: int = 2):
        if torch.is_tensor(source):
            if batch is None or batch < 1:
                raise ValueError("batch must be positive")
            self.parts = [source[i: i + batch] for i in range(0, source.shape[0], batch)]
        else:
            self.parts = list(source)
        if any(p.is_cuda for p in self.parts):
            raise ValueError("Prefetcher copies from host memory")
        if depth < 1:
            raise ValueError("depth must be positive")
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.depth = depth
        self.stream = torch.cuda.Stream(self.device)
        if self.parts:
            rows = max(p.shape[0] for p in self.parts)
            tail, dtype = tuple(self.parts[0].shape[1:]), self.parts[0].dtype
            self.buffers = [torch.empty((rows,) + tail, dtype=dtype, device=self.device) for _ in range(depth)]
        self.ready = [torch.cuda.Event() for _ in range(depth)]
        self.free = [torch.cuda.Event() for _ in range(depth)]
        self.bytes = 0

    def __len__(self) -> int:
        return len(self.parts)

    def _issue(self, k: int, fresh: bool) -> None:
        slot, part = k % self.depth, self.parts[k]
        if not fresh:
            self.stream.wait_event(self.free[slot])
        with torch.cuda.stream(self.stream):
            self.buffers[slot][: part.shape[0]].copy_(part, non_blocking=True)
            self.ready[slot].record(self.stream)
        self.bytes += part.numel() * part.element_size()

    def __iter__(self) -> Iterator[torch.Tensor]:
        n = len(self)
        # the first copies start after the work already queued by the consumer
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        for k in range(min(self.depth, n)):
            self._issue(k, fresh=True)
        for k in range(n):
            slot = k % self.depth
            cur = torch.cuda.current_stream(self.device)
            cur.wait_event(self.ready[slot])
            yield self.buffers[slot][: self.parts[k].shape[0]]
            self.free[slot].record(cur)
            if k + self.depth < n:
                self._issue(k + self.depth, fresh=False)


class Readback:
    """Device results copied to pinned host buffers on a side stream, so the
    next step's kernels are queued meanwhile.  ``push`` returns the host
    tensor that will hold the copy; ``wait`` makes the current stream (and
    so a timing event recorded next) wait for every copy pushed."""

    def __init__(self, depth: int = 2, device=None):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.depth = depth
        self.stream = torch.cuda.Stream(self.device)
        self.host: List[Optional[torch.Tensor]] = [None] * depth
        self.done = [torch.cuda.Event() for _ in range(depth)]
        self.count = 0
        self.bytes = 0

    def push(self, tensor: torch.Tensor) -> torch.Tensor:
        slot = self.count % self.depth
        buf = self.host[slot]
        if buf is None or buf.shape != tensor.shape or buf.dtype != tensor.dtype:
            if buf is not None:
                self.done[slot].synchronize()
            buf = self.host[slot] = torch.empty(tensor.shape, dtype=tensor.dtype, pin_memory=True)
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(self.stream):
            buf.copy_(tensor, non_blocking=True)
            self.done[slot].record(self.stream)
        tensor.record_stream(self.stream)
        self.count += 1
        self.bytes += tensor.numel() * tensor.element_size()
        return buf

    def wait(self) -> None:
        torch.cuda.current_stream(self.device).wait_stream(self.stream)

    def synchronize(self) -> None:
        self.stream.synchronize()


def save_kernels(path: str, **kernels) -> None:
    """``numpy.savez(path, conv1_kernel=..., ...)`` of F32 kernels, the
    checkpoint layout of the reference's examples."""
    numpy.savez(path, **{k: (v.detach().cpu().numpy() if torch.is_tensor(v) else numpy.asarray(v))
                         for k, v in kernels.items()})


def load_kernels(path: str, **targets) -> None:
    """Copy each named array of an ``.npz`` checkpoint into the given kernel
    tensor in place (the examples' ``to_tensor(data[k]).to(kernel)``)."""
    data = numpy.load(path)
    for name, dst in targets.items():
        src = torch.from_numpy(numpy.ascontiguousarray(data[name]))
        if src.numel() != dst.numel():
            raise ValueError(f"{name}: {tuple(src.shape)} does not fit {tuple(dst.shape)}")
        dst.copy_(src.view(dst.shape))
