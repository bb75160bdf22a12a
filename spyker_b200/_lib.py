"""Loader of the sm_100a C-ABI library (``include/spyker_b200.h``).

The library is required: importing this module fails loudly when
``spyker_b200/lib/libspyker_b200.so`` has not been built, and every entry point
raises on a non-zero status.  There is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libspyker_b200.so")

_P, _I, _D, _S, _INT = C.c_void_p, C.c_int64, C.c_double, C.c_size_t, C.c_int

# name -> (restype, argtypes)
SIGNATURES = {
    "spk_last_error": (C.c_char_p, []),
    "spk_version": (C.c_char_p, []),
    "spk_device_count": (_INT, []),
    "spk_launch_count": (C.c_uint64, []),
    "spk_device_status": (_INT, [_INT]),
    "spk_recheck_count": (C.c_ulonglong, [_INT]),
    "spk_recompute_count": (C.c_ulonglong, [_INT]),
    "spk_set_conv_schedule": (_INT, [_INT, _INT, _INT]),
    "spk_random_seed": (None, [C.c_uint64]),
    "spk_normal_kernel": (_INT, [_P, _I, _D, _D]),
    "spk_gaussian_kernel": (_INT, [_P, _I, _D]),
    "spk_gabor_kernel": (_INT, [_P, _I, _D, _D, _D, _D, _D]),
    "spk_log_kernel": (_INT, [_P, _I, _D]),
    "spk_rank_code_workspace": (_S, [_I, _I, _INT]),
    "spk_rank_code": (_INT, [_P, _INT, _P, _INT, _I, _I, _I, _INT, _P, _S, _P]),
    "spk_canny_workspace": (_I, [_I, _I, _I]),
    "spk_canny": (_INT, [_P, _P, _I, _I, _I, _D, _D, _P, _I, _P]),
    "spk_quantize": (_INT, [_P, _INT, _I, _D, _D, _D, _P]),
    "spk_idx_shape": (_INT, [C.c_char_p, _INT, _P, _P, _P]),
    "spk_idx_read": (_INT, [C.c_char_p, _I, _P, _I, _INT]),
    "spk_zca_stats_workspace": (_I, [_I, _I]),
    "spk_zca_stats": (_INT, [_P, _I, _I, _P, _P, _P, _I, _P]),
    "spk_zca_matrix": (_INT, [_P, _P, _I, _D, _P, _P, _P]),
    "spk_zca_transform": (_INT, [_P, _I, _I, _P, _P, _P, _P]),
    "spk_zca_split": (_INT, [_P, _INT, _P, _I, _I, _P]),
    "spk_rate_code_workspace": (_S, [_I, _I, _I, _INT]),
    "spk_rate_code": (_INT, [_P, _INT, _P, _INT, _I, _I, _I, _INT, _P, _S, _P]),
    "spk_rate_interval_table": (None, [_I, _P]),
    "spk_rate_fire": (_INT, [_P, _INT, _P, _INT, _I, _I, _I, _D, _P]),
    "spk_rate_gather": (_INT, [_P, _INT, _P, _INT, _I, _I, _I, _P]),
    "spk_rate_pool": (_INT, [_P, _P, _INT, _INT, _P, _I, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P]),
    "spk_threshold": (_INT, [_P, _INT, _I, _D, _D, _P]),
    "spk_rank_infinite": (_INT, [_P, _INT, _I, _I, _I, _D, _P]),
    "spk_rank_fire": (_INT, [_P, _INT, _P, _INT, _I, _D, _P]),
    "spk_rank_gather": (_INT, [_P, _INT, _P, _INT, _I, _I, _I, _D, _P]),
    "spk_rank_scatter": (_INT, [_P, _INT, _P, _INT, _I, _I, _I, _P]),
    "spk_pad": (_INT, [_P, _P, _INT, _I, _I, _I, _P, _D, _P]),
    "spk_rank_pool": (_INT, [_P, _P, _INT, _I, _I, _I, _I, _I, _I, _I, _I, _I, _P, _P]),
    "spk_rank_inhibit": (_INT, [_P, _INT, _I, _I, _I, _I, _D, _P]),
    "spk_rank_convwta_workspace": (_S, [_I, _I, _I, _I, _I]),
    "spk_rank_convwta": (_INT, [_P, _INT, _I, _I, _I, _I, _I, _I, _I, _I, _D, _P, _P, _P, _S, _P]),
    "spk_rank_fcwta_workspace": (_S, [_I, _I, _I]),
    "spk_rank_fcwta": (_INT, [_P, _INT, _I, _I, _I, _I, _I, _D, _P, _P, _P, _S, _P]),
    "spk_rank_convstdp_workspace": (_S, [_I, _I, _I, _I, _I, _I, _I]),
    "spk_rank_convstdp": (_INT, [_P, _INT, _I, _I, _I, _I, _I, _P, _I, _I, _I, _P, _I, _I, _P, _I, _P, _P, _I,
                                 _I, _I, _P, _P, _S, _P]),
    "spk_rank_convstdp_noalloc": (_INT, [_P, _INT, _I, _I, _I, _I, _I, _P, _I, _I, _I, _P, _I, _I, _P, _I, _P, _P,
                                         _I, _I, _I, _P, _P]),
    "spk_rank_convstdp_prepost_workspace": (_S, [_I, _I, _I, _I]),
    "spk_rank_convstdp_prepost": (_INT, [_P, _INT, _I, _I, _I, _I, _I, _I, _I, _I, _P, _I, _I, _P, _P, _I, _I, _I, _P,
                                         _P, _P, _P, _S, _P]),
    "spk_stdp_scan": (_INT, [_P, _I, _I, _I, _I, _I, _P, _P, _P, _I, _I, _P, _P, _I, _INT, _P]),
    "spk_stdp_scan_nets": (_INT, [_P, _I, _I, _I, _I, _I, _I, _P, _P, _P, _I, _I, _P, _P, _P, _P, _I, _INT, _P]),
    "spk_conv_fire_wta_nets_workspace": (_S, [_I, _I, _I, _I, _I, _I, _I, _I, _I, _I, _I, _P, _INT]),
    "spk_conv_fire_wta_nets": (_INT, [_P, _INT, _P, _I, _P, _P, _P, _I, _I, _I, _I, _I, _I, _I, _I, _I, _I, _P, _D,
                                      _D, _D, _I, _I, _I, _D, _P, _P, _P, _I, _I, _P, _INT, _P, _S, _P]),
    "spk_rank_fcstdp_workspace": (_S, [_I, _I, _I]),
    "spk_rank_fcstdp": (_INT, [_P, _INT, _I, _I, _I, _P, _I, _P, _P, _I, _P, _P, _I, _P, _S, _P]),
    "spk_conv_workspace": (_S, [_I, _I, _I, _I, _I, _I, _I, _INT]),
    "spk_conv": (_INT, [_P, _INT, _P, _P, _I, _I, _I, _I, _I, _I, _I, _I, _I, _P, _INT, _P, _S, _P]),
    "spk_conv_fire_wta_workspace": (_S, [_I, _I, _I, _I, _I, _I, _I, _I, _I, _I, _P, _INT]),
    "spk_conv_fire_wta": (_INT, [_P, _INT, _P, _I, _I, _I, _I, _I, _I, _I, _I, _I, _I, _P, _D, _D, _D, _D, _I, _I,
                                 _I, _D, _P, _P, _P, _I, _I, _P, _INT, _P, _S, _P]),
    "spk_fc": (_INT, [_P, _INT, _P, _P, _I, _I, _I, _INT, _P]),
    "spk_filter": (_INT, [_INT, _P, _P, _P, _I, _I, _I, _I, _I, _I, _I, _I, _P, _P]),
    "spk_backward": (_INT, [_P, _P, _P, _I, _I, _I, _D, _P]),
    "spk_labelize": (_INT, [_P, _INT, _P, _I, _I, _I, _D, _P]),
    "spk_fcbackward_workspace": (_S, [_I, _I]),
    "spk_fcbackward": (_INT, [_P, _I, _I, _P, _P, _P, _P, _I, _P, _P, _S, _P]),
    "spk_fst_pool": (_INT, [_P, _I, _I, _I, _I, _P, _I, _I, _P, _P, _P, _D, _P]),
    "spk_fst_pool_backward": (_INT, [_P, _I, _I, _I, _I, _P, _I, _I, _P, _P, _P, _P, _P]),
    "spk_fst_conv_backward_workspace": (_S, [_I, _I, _I, _I, _I]),
    "spk_fst_conv_backward": (_INT, [_P, _I, _I, _I, _I, _P, _I, _I, _I, _P, _P, _I, _I, _P, _P, _P, _P, _P, _S,
                                     _P]),
    "spk_fst_conv_times_workspace": (_S, [_I, _I, _I, _I, _I, _I, _I, _I, _INT]),
    "spk_fst_conv_times": (_INT, [_P, _I, _I, _I, _I, _P, _I, _I, _I, _I, _I, _P, _I, _D, _P, _INT, _P, _S, _P]),
    "spk_fst_conv_prespike": (_INT, [_P, _I, _I, _I, _I, _P, _I, _I, _I, _P, _I, _I, _P, _P, _P, _P]),
    "spk_sparse_code_workspace": (_S, [_I, _I, _I, _I, _I]),
    "spk_sparse_code": (_INT, [_P, _INT, _I, _I, _I, _I, _I, _INT, _P, _P, _I, _P, _S, _P]),
    "spk_sparse_from_dense_workspace": (_S, [_I, _I, _I, _I, _I]),
    "spk_sparse_from_dense": (_INT, [_P, _INT, _I, _I, _I, _I, _I, _D, _P, _P, _I, _P, _S, _P]),
    "spk_sparse_dense_workspace": (_S, [_I, _I, _I, _I]),
    "spk_sparse_to_dense": (_INT, [_P, _P, _I, _I, _I, _I, _I, _P, _INT, _P, _S, _P]),
    "spk_sparse_gather": (_INT, [_P, _P, _I, _I, _I, _I, _I, _P, _INT, _P, _S, _P]),
    "spk_sparse_pad": (_INT, [_P, _P, _I, _I, _I, _I, _I, _I, _P, _P, _P, _I, _P]),
    "spk_sparse_pool_workspace": (_S, [_I, _I, _I, _I, _I]),
    "spk_sparse_pool": (_INT, [_P, _P, _I, _I, _I, _I, _I, _I, _P, _P, _P, _I, _I, _P, _P, _I, _P, _S, _P]),
    "spk_sparse_inhibit_workspace": (_S, [_I, _I, _I, _I]),
    "spk_sparse_inhibit": (_INT, [_P, _P, _I, _I, _I, _I, _I, _I, _P, _P, _I, _P, _S, _P]),
    "spk_sparse_conv_workspace": (_S, [_I, _I, _I, _I, _I, _I, _I, _P]),
    "spk_sparse_conv": (_INT, [_P, _P, _I, _I, _I, _I, _I, _P, _I, _I, _I, _D, _P, _P, _P, _P, _I, _P, _S, _P]),
    "spk_sparse_convwta": (_INT, [_P, _P, _I, _I, _I, _I, _I, _P, _I, _P, _P, _P]),
    "spk_sparse_stdp_workspace": (_S, [_I, _I, _I, _I, _I, _I, _I, _P]),
    "spk_sparse_stdp": (_INT, [_P, _P, _I, _I, _I, _I, _I, _P, _I, _I, _I, _P, _I, _P, _P, _I, _P, _P, _S, _P]),
}


class SpykerError(RuntimeError):
    """A failure reported by the C ABI (bad arguments, CUDA error...)."""


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"spyker_b200: the CUDA library {LIB_PATH} is not built; run "
            f"`python {os.path.join(os.path.dirname(os.path.abspath(__file__)), 'build.py')}` "
            "(a script: importing the package needs the library; there is no CPU fallback)"
        )
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status: int) -> None:
    if status != 0:
        raise SpykerError(lib.spk_last_error().decode())


# NVTX ranges around every C-ABI call, named after the entry point (for
# nsys timelines and `ncu --nvtx --nvtx-include`); off unless SPYKER_NVTX is
# set to a non-zero value or set_nvtx(True) is called.  Without a profiler
# attached a range costs a no-op call.
_nvtx = os.environ.get("SPYKER_NVTX", "0") not in ("", "0")


def set_nvtx(enabled: bool) -> None:
    """Turn the per-call NVTX ranges on or off."""
    global _nvtx
    _nvtx = bool(enabled)


def call(name: str, *args) -> None:
    if _nvtx:
        torch.cuda.nvtx.range_push(name)
        try:
            check(getattr(lib, name)(*args))
        finally:
            torch.cuda.nvtx.range_pop()
        return
    check(getattr(lib, name)(*args))


def stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def i64(*v) -> C.Array:
    return (C.c_int64 * len(v))(*[int(x) for x in v])


def f64(v) -> C.Array:
    v = [float(x) for x in v]
    return (C.c_double * len(v))(*v)
