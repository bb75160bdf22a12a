"""The control functions of the reference's `spyker.control` module
(opers.h:44-121): every exported name exists, the CPU-side ones behave, and
on a GPU the device / memory queries answer from the CUDA runtime."""

import re

import pytest
import torch

import spyker_b200 as spyker

NAMES = ["all_devices", "clear_context", "cuda_arch_list", "cuda_cache_clear", "cuda_cache_enable",
         "cuda_cache_enabled", "cuda_cache_print", "cuda_conv_force", "cuda_conv_heuristic", "cuda_conv_light",
         "cuda_current_device", "cuda_device_arch", "cuda_memory_free", "cuda_memory_taken", "cuda_memory_total",
         "cuda_memory_used", "cuda_set_device", "max_threads", "set_max_threads", "cuda_available",
         "cuda_device_count", "version"]


def test_names_exported():
    missing = [n for n in NAMES if not callable(getattr(spyker, n, None))]
    assert not missing


def test_threads_archs_and_knobs():
    keep = spyker.max_threads()
    spyker.set_max_threads(2)
    assert spyker.max_threads() == 2
    spyker.set_max_threads()
    assert spyker.max_threads() >= 1
    spyker.set_max_threads(keep)
    assert spyker.cuda_arch_list() == [100]
    assert spyker.all_devices()[0] == torch.device("cpu")
    spyker.cuda_conv_light(True)
    spyker.cuda_conv_force(True)
    spyker.cuda_conv_heuristic(False)
    assert spyker.control.conv_settings() == {"light": True, "heuristic": False, "force": True}
    spyker.cuda_conv_light(False)
    spyker.cuda_conv_force(False)
    spyker.cuda_conv_heuristic(True)


@pytest.mark.gpu
def test_device_and_memory_queries():
    assert spyker.cuda_available() and spyker.cuda_device_count() >= 1
    spyker.cuda_set_device(0)
    assert spyker.cuda_current_device() == 0
    assert spyker.cuda_device_arch()[0] == 100
    total, free = spyker.cuda_memory_total(), spyker.cuda_memory_free()
    assert total > 100 * 2**30 and 0 < free <= total
    x = torch.empty(64 * 2**20, dtype=torch.uint8, device="cuda")
    assert spyker.cuda_memory_used() >= x.numel() and spyker.cuda_memory_taken() >= spyker.cuda_memory_used()
    del x
    spyker.cuda_cache_enable(False)
    assert not spyker.cuda_cache_enabled()
    spyker.cuda_cache_enable(True)
    spyker.clear_context()
    assert len(spyker.all_devices()) == 1 + spyker.cuda_device_count()
    with pytest.raises(ValueError):
        spyker.cuda_set_device(spyker.cuda_device_count())
    assert re.search(r"\d+\.\d+", spyker.version())
