"""spyker_b200 — B200-native (sm_100a) spiking-CNN hot path with Spyker's API.

``import spyker_b200 as spyker`` gives the names of the reference's Python
package (src/python/spyker/__init__.py): coding, filters, Conv with
``.stdp()``, fire/threshold/infinite, pool, inhibit, convwta/fcwta, the
temporal-backprop helpers and the sparse event-list path.  Every operation
runs on the GPU through the C ABI of ``include/spyker_b200.h``.
"""

from . import control, io, sparse, temporal
from ._lib import SpykerError, set_nvtx
from .control import (all_devices, clear_context, cuda_arch_list, cuda_cache_clear, cuda_cache_enable, cuda_cache_enabled,
                      cuda_cache_print, cuda_conv_force, cuda_conv_heuristic, cuda_conv_light, cuda_current_device,
                      cuda_device_arch, cuda_memory_free, cuda_memory_taken, cuda_memory_total, cuda_memory_used,
                      cuda_set_device, max_threads, set_max_threads)
from .io import CSV, Prefetcher, Readback, mnist_data, mnist_label, read_csv, read_mnist
from .module import (FC, ZCA, BPConfig, Conv, conv_fire_wta, DoG, DoGFilter, Gabor, GaborFilter, LoG, STDPConfig, Winner, Winners,
                     backward, canny, code, conv, conv_precision, convwta, fc, fcwta, fire, gather, infinite,
                     inhibit, labelize, pad, pool, quantize, random_seed, scatter, set_conv_precision, stdp,
                     threshold)
from .sparse import SparseTensor, to_sparse
from .utils import (Tensor, copy_array, create_array, create_tensor, device, expand2, expand4, shape, to_numpy, to_tensor,
                    to_torch, wrap_array)

__version__ = "0.1.0"


def version() -> str:
    from ._lib import lib

    return lib.spk_version().decode()


def cuda_available() -> bool:
    import torch

    return torch.cuda.is_available()


def cuda_device_count() -> int:
    from ._lib import lib

    return max(0, int(lib.spk_device_count()))
