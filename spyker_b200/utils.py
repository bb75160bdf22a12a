"""Array interop: zero-copy for CUDA torch tensors, staged copies for host arrays.

Mirrors src/python/spyker/utils.py of the reference (``wrap_array`` /
``create_array`` / ``to_numpy`` / ``to_torch``).  The compute device is always a
CUDA GPU: CUDA tensors are used in place (no copy, the caller's stream), and
NumPy arrays or CPU tensors are copied to the device, processed, and the
result is returned in the caller's ecosystem (an in-place op writes back into
the caller's array), exactly as the reference returns results of the same
kind as its input (utils.py:294-340).
"""

from __future__ import annotations

from typing import Sequence, Tuple

import numpy
import torch

DataType = str  # "i8", "i16", "i32", "i64", "u8", "f16", "f32", "f64"

_TORCH = {
    "i8": torch.int8,
    "i16": torch.int16,
    "i32": torch.int32,
    "i64": torch.int64,
    "u8": torch.uint8,
    "f16": torch.float16,
    "f32": torch.float32,
    "f64": torch.float64,
}
_NAME = {v: k for k, v in _TORCH.items()}
# codes of the reference's `enum class Type` (src/spyker/utils.h:96-120)
_CODE = {torch.int8: 0, torch.int16: 1, torch.int32: 2, torch.int64: 3, torch.uint8: 4, torch.float16: 8,
         torch.float32: 9, torch.float64: 10}


def torch_dtype(dtype) -> torch.dtype:
    if isinstance(dtype, torch.dtype):
        return dtype
    if isinstance(dtype, str):
        if dtype not in _TORCH:
            raise TypeError(f"Given data type {dtype} is not supported.")
        return _TORCH[dtype]
    return torch.from_numpy(numpy.zeros(0, dtype=dtype)).dtype


def type_code(dtype: torch.dtype) -> int:
    if dtype not in _CODE:
        raise TypeError(f"Data type {dtype} is not supported.")
    return _CODE[dtype]


def dtype_name(dtype: torch.dtype) -> str:
    return _NAME[dtype]


_default_device: torch.device | None = None


def default_device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("spyker_b200 needs a CUDA GPU (there is no CPU backend)")
    global _default_device
    if _default_device is None:
        _default_device = torch.device("cuda", torch.cuda.current_device())
    return _default_device


def device(kind: str = "cuda", index: int = -1) -> torch.device:
    """``spyker.device(...)``: every device maps to a CUDA device here."""
    if kind == "cuda":
        return torch.device("cuda", index if index >= 0 else torch.cuda.current_device())
    return default_device()


class Bound:
    """An input array bound to a contiguous CUDA tensor view."""

    def __init__(self, array, dev: torch.device | None = None, writeable: bool = False):
        self.orig = array
        if torch.is_tensor(array):
            if not array.is_contiguous():
                raise TypeError('Input array is not contiguous. use "contiguous" function to make it contiguous.')
            if array.is_cuda:
                self.kind, self.dev = "cuda", array
            else:
                self.kind, self.dev = "torch", array.to(dev or default_device())
        elif isinstance(array, numpy.ndarray):
            if not array.flags["C_CONTIGUOUS"]:
                raise TypeError('Input array is not contiguous. use "numpy.ascontiguousarray" to make it contiguous.')
            if writeable and not array.flags["WRITEABLE"]:
                raise TypeError('Input array is not writable. use "numpy.array(..., copy=True)" to make it writable.')
            self.kind, self.dev = "numpy", torch.from_numpy(array).to(dev or default_device())
        else:
            raise TypeError(f"Input array {type(array)} can only be Numpy array or PyTorch tensor.")

    def back(self, out: torch.Tensor):
        """Return a device result in the caller's ecosystem."""
        if self.kind == "cuda":
            return out
        cpu = out.cpu()
        return cpu.numpy() if self.kind == "numpy" else cpu

    def write_back(self):
        """Finish an in-place op: copy the device tensor into a host array."""
        if self.kind == "numpy":
            numpy.copyto(self.orig, self.dev.cpu().numpy())
        elif self.kind == "torch":
            self.orig.copy_(self.dev.cpu())
        return self.orig


class _CudaBuffer:
    """A device pointer seen through ``__cuda_array_interface__``."""

    def __init__(self, ptr: int, shape, dtype: torch.dtype):
        typestr = numpy.dtype(torch.empty(0, dtype=dtype).numpy().dtype).str
        self.__cuda_array_interface__ = {"shape": tuple(int(v) for v in shape), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3}


def create_tensor(device, dtype, shape, pinned: bool = False, unified: bool = False, data: int | None = None):
    """A tensor of ``shape`` and ``dtype`` ("u8", "f32", ... or a torch dtype)
    on ``device`` (utils.py ``create_tensor`` of the reference): pinned host
    memory with ``pinned=True`` on the CPU; ``unified`` is treated as the
    device; ``data``, a raw pointer, is wrapped without a copy (the caller
    keeps the memory alive)."""
    dev = torch.device(device) if not isinstance(device, torch.device) else device
    dt = torch_dtype(dtype)
    shape = [int(v) for v in shape]
    if any(v < 0 for v in shape):
        raise ValueError("Tensor shape can't have negative dimensions.")
    if data is not None:
        if dev.type == "cuda":
            return torch.as_tensor(_CudaBuffer(data, shape, dt), device=dev)
        import ctypes

        nbytes = int(numpy.prod(shape)) * torch.empty(0, dtype=dt).element_size()
        buf = (ctypes.c_uint8 * nbytes).from_address(int(data))
        return torch.frombuffer(buf, dtype=dt).view(shape) if nbytes else torch.empty(shape, dtype=dt)
    if dev.type == "cpu":
        return torch.empty(shape, dtype=dt, pin_memory=bool(pinned) and torch.cuda.is_available())
    return torch.empty(shape, dtype=dt, device=dev)


def wrap_array(array, writeable: bool = False):
    """A zero-copy tensor view of a PyTorch tensor or NumPy array."""
    if torch.is_tensor(array):
        return array
    if isinstance(array, numpy.ndarray):
        if writeable and not array.flags["WRITEABLE"]:
            raise TypeError('Input array is not writable. use "numpy.array(..., copy=True)" to make it writable.')
        return torch.from_numpy(array)
    raise TypeError(f"Input array {type(array)} can only be Numpy array or PyTorch tensor.")


def create_array(array, dtype, shape):
    """A new array of ``array``'s kind (NumPy, or a tensor on its device)."""
    shape = [int(v) for v in shape]
    if isinstance(array, numpy.ndarray):
        dt = dtype if not isinstance(dtype, (str, torch.dtype)) else torch.empty(0, dtype=torch_dtype(dtype)).numpy().dtype
        return numpy.empty(shape, dtype=dt)
    if torch.is_tensor(array):
        return torch.empty(shape, dtype=torch_dtype(dtype), device=array.device)
    raise TypeError(f"Input array {type(array)} can only be Numpy array or PyTorch tensor.")


def clone_array(array):
    if torch.is_tensor(array):
        return array.clone()
    if isinstance(array, numpy.ndarray):
        return numpy.array(array, copy=True)
    raise TypeError(f"Input array {type(array)} can only be Numpy array or PyTorch tensor.")


def to_numpy(*arrays):
    out = [a.detach().cpu().numpy() if torch.is_tensor(a) else numpy.asarray(a) for a in arrays]
    return out[0] if len(out) == 1 else tuple(out)


def to_torch(*arrays):
    out = [a if torch.is_tensor(a) else torch.from_numpy(numpy.ascontiguousarray(a)) for a in arrays]
    return out[0] if len(out) == 1 else tuple(out)


class Tensor(torch.Tensor):
    """A torch tensor whose ``to(other_tensor)`` copies its values into
    ``other`` in place (casting, any devices, same element count) and
    returns None, as the reference's ``Tensor::to(Tensor)``
    (utils.cpp:149-170), which the examples use to load checkpoints into
    kernels.  Every other form of ``to`` and every op are torch's, and op
    results are plain tensors."""

    __torch_function__ = torch._C._disabled_torch_function_impl

    def to(self, *args, **kwargs):
        if len(args) == 1 and not kwargs and torch.is_tensor(args[0]):
            other = args[0]
            if other.numel() != self.numel():
                raise ValueError("Tensors must have the same numel.")
            other.copy_(self.as_subclass(torch.Tensor).reshape(other.shape))
            return None
        return torch.Tensor.to(self.as_subclass(torch.Tensor), *args, **kwargs)


def to_tensor(*arrays, pinned: bool = False, unified: bool = False):
    """A new tensor holding each array: on the GPU, or in pinned host memory
    with ``pinned=True`` (``unified`` is accepted and treated as the GPU)."""
    out = []
    for a in arrays:
        if pinned:
            t = to_torch(a).detach().cpu().clone()
            t = t.pin_memory() if torch.cuda.is_available() else t
        else:
            t = Bound(a).dev.clone() if not (torch.is_tensor(a) and a.is_cuda) else a.clone()
        out.append(t.as_subclass(Tensor))
    return out[0] if len(out) == 1 else tuple(out)


def copy_array(source, destin) -> None:
    src = to_torch(source)
    if torch.is_tensor(destin):
        destin.copy_(src)
    else:
        numpy.copyto(destin, to_numpy(src))


# ---- shape helpers (src/python/spyker/private.py, src/spyker/opers.cpp) ----

def expand2(shape) -> Tuple[int, int]:
    if isinstance(shape, int):
        return (shape, shape)
    if isinstance(shape, (list, tuple)) and len(shape) == 1:
        return int(shape[0]), int(shape[0])
    if isinstance(shape, (list, tuple)) and len(shape) == 2:
        return int(shape[0]), int(shape[1])
    raise ValueError("Given shape couldn't be expanded to 2D.")


def expand4(shape) -> Tuple[int, int, int, int]:
    """(top, left, bottom, right), the order src/spyker/shape.cpp:44-45 uses."""
    if isinstance(shape, int):
        return (shape, shape, shape, shape)
    if isinstance(shape, (list, tuple)) and len(shape) == 1:
        return (int(shape[0]),) * 4
    if isinstance(shape, (list, tuple)) and len(shape) == 2:
        return int(shape[0]), int(shape[1]), int(shape[0]), int(shape[1])
    if isinstance(shape, (list, tuple)) and len(shape) == 4:
        return tuple(int(s) for s in shape)
    raise ValueError("Given shape couldn't be expanded to 4D.")


def _at_least(shape: Sequence[int], n: int, exact: bool, what: str):
    shape = list(shape)
    if len(shape) == n - 1:
        shape.insert(0, 1)
    if (exact and len(shape) != n) or (not exact and len(shape) < n):
        raise ValueError(f"Input dimensions couldn't be viewed as {'' if exact else 'at least '}{n}D.")
    return shape


def least2(s):
    return _at_least(s, 2, False, "2")


def least3(s):
    return _at_least(s, 3, False, "3")


def to2(s):
    return _at_least(s, 2, True, "2")


def to3(s):
    return _at_least(s, 3, True, "3")


def to4(s):
    return _at_least(s, 4, True, "4")


def to5(s):
    return _at_least(s, 5, True, "5")


class shape:
    """Output-shape inference of src/spyker/shape.cpp:35-154."""

    @staticmethod
    def conv(input, kernel, stride, pad):
        if len(input) != 5 or len(kernel) != 4:
            raise ValueError("Input dimensions must be 5 and kernel dimensions must be 4.")
        if input[2] != kernel[1]:
            raise ValueError("Input and kernel channels are not compatible.")
        oh = (input[3] + pad[0] + pad[2] - kernel[2]) // stride[0] + 1
        ow = (input[4] + pad[1] + pad[3] - kernel[3]) // stride[1] + 1
        if oh <= 0 or ow <= 0 or input[3] + pad[0] + pad[2] < kernel[2] or input[4] + pad[1] + pad[3] < kernel[3]:
            raise ValueError("Input and kernel shapes are not compatible.")
        return [input[0], input[1], kernel[0], oh, ow]

    @staticmethod
    def fc(input, kernel):
        if len(input) != 3 or len(kernel) != 2 or input[2] != kernel[1]:
            raise ValueError("Input and kernel shapes don't match.")
        return [input[0], input[1], kernel[0]]

    @staticmethod
    def pool(input, kernel, stride, pad):
        if len(input) != 5:
            raise ValueError("Input dimensions must be 5.")
        oh = (input[3] + pad[0] + pad[2] - kernel[0]) // stride[0] + 1
        ow = (input[4] + pad[1] + pad[3] - kernel[1]) // stride[1] + 1
        if oh <= 0 or ow <= 0:
            raise ValueError("Input and kernel shapes are not compatible.")
        return [input[0], input[1], input[2], oh, ow]

    @staticmethod
    def pad(input, pad):
        return [input[0], input[1], input[2], input[3] + pad[0] + pad[2], input[4] + pad[1] + pad[3]]

    @staticmethod
    def filt(input, kh, kw, pad, channels):
        oh = input[2] + pad[0] + pad[2] - kh + 1
        ow = input[3] + pad[1] + pad[3] - kw + 1
        if oh <= 0 or ow <= 0:
            raise ValueError("Input and kernel shapes are not compatible.")
        return [input[0], input[1] * channels, oh, ow]

    @staticmethod
    def code(input, time):
        return [input[0], time] + list(input[1:])

    @staticmethod
    def gather(input):
        return [input[0]] + list(input[2:])


def read_mnist(train_images: str, train_labels: str, test_images: str, test_labels: str):
    """``spyker.utils.read_mnist``: the IDX reader of ``spyker_b200.io``."""
    from .io import read_mnist as read

    return read(train_images, train_labels, test_images, test_labels)


def read_csv(path: str, delim: str = ", "):
    """``spyker.utils.read_csv``: the CSV reader of ``spyker_b200.io``."""
    from .io import read_csv as read

    return read(path, delim)


def to_sparse(*arrays, threshold: float = 0.0):
    """``spyker.utils.to_sparse``: event lists of ``spyker_b200.sparse``."""
    from .sparse import to_sparse as convert

    return convert(*arrays, threshold=threshold)
