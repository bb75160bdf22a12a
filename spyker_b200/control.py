"""Device and memory control of the reference's `spyker.control` module
(opers.h:44-121, bind.cpp:136-163), on torch's CUDA runtime and caching
allocator.

The reference keeps its own CUDA memory cache and cuDNN convolution knobs;
here device memory comes from torch's caching allocator (the cache calls
act on it) and convolutions are this library's own kernels, so the cuDNN
knobs are recorded and reported but select nothing.  CPU threads bound the
host-side work (IDX reads, torch's CPU ops); every spiking op runs on the
GPU.
"""

from __future__ import annotations

import os
from typing import List

import torch

from . import utils

# compute capabilities the shared library is built for (sm_100a)
_ARCHS = [100]
_cache_enabled = {}
_conv = {"light": False, "heuristic": True, "force": False}


def _dev(device: int) -> int:
    return torch.cuda.current_device() if device < 0 else int(device)


def cuda_set_device(device: int) -> None:
    if not 0 <= int(device) < torch.cuda.device_count():
        raise ValueError(f"CUDA device {device} is not available.")
    torch.cuda.set_device(int(device))
    utils._default_device = torch.device("cuda", int(device))


def cuda_current_device() -> int:
    return torch.cuda.current_device()


def cuda_arch_list() -> List[int]:
    """Architectures the library is compiled for (major * 10 + minor)."""
    return list(_ARCHS)


def cuda_device_arch() -> List[int]:
    """Architecture of every visible device (major * 10 + minor)."""
    out = []
    for i in range(torch.cuda.device_count()):
        major, minor = torch.cuda.get_device_capability(i)
        out.append(major * 10 + minor)
    return out


def cuda_memory_total() -> int:
    return int(torch.cuda.mem_get_info()[1])


def cuda_memory_free() -> int:
    return int(torch.cuda.mem_get_info()[0])


def cuda_memory_taken(device: int = -1) -> int:
    """Bytes held by the caching allocator (in use or cached)."""
    return int(torch.cuda.memory_reserved(_dev(device)))


def cuda_memory_used(device: int = -1) -> int:
    """Bytes of live tensors."""
    return int(torch.cuda.memory_allocated(_dev(device)))


def cuda_cache_enabled(device: int = -1) -> bool:
    return _cache_enabled.get(_dev(device), True)


def cuda_cache_enable(enable: bool, device: int = -1) -> None:
    """Record the setting; disabling releases the cached blocks now (torch's
    allocator keeps caching later frees)."""
    d = _dev(device)
    _cache_enabled[d] = bool(enable)
    if not enable:
        cuda_cache_clear(d)


def cuda_cache_clear(device: int = -1) -> None:
    with torch.cuda.device(_dev(device)):
        torch.cuda.empty_cache()


def clear_context() -> None:
    """Release every cached block on every device."""
    for i in range(torch.cuda.device_count()):
        cuda_cache_clear(i)


def cuda_cache_print(device: int = -1) -> None:
    print(torch.cuda.memory_summary(_dev(device), abbreviated=True))


def cuda_conv_light(light: bool) -> None:
    _conv["light"] = bool(light)


def cuda_conv_heuristic(heuristic: bool) -> None:
    _conv["heuristic"] = bool(heuristic)


def cuda_conv_force(force: bool) -> None:
    _conv["force"] = bool(force)


def conv_settings() -> dict:
    """The recorded cuDNN-knob values (they select nothing here)."""
    return dict(_conv)


def all_devices() -> List[torch.device]:
    return [torch.device("cpu")] + [torch.device("cuda", i) for i in range(torch.cuda.device_count())]


def max_threads() -> int:
    return torch.get_num_threads()


def set_max_threads(threads: int = -1) -> None:
    torch.set_num_threads(int(threads) if threads > 0 else (os.cpu_count() or 1))
