"""Array interop of the reference's utils.py (create_tensor, wrap_array,
create_array, to_tensor(...).to(other)) on CPU, and wrapping a raw device
pointer on the GPU."""

import numpy as np
import pytest
import torch

import spyker_b200 as spyker
from spyker_b200 import utils


def test_create_and_wrap():
    t = spyker.create_tensor("cpu", "u8", [2, 3])
    assert t.shape == (2, 3) and t.dtype == torch.uint8
    a = np.arange(6, dtype=np.float32)
    v = spyker.wrap_array(a)
    v[0] = 7
    assert a[0] == 7
    b = spyker.create_tensor("cpu", "f32", [2, 3], data=a.ctypes.data)
    assert b[0, 0] == 7 and b[1, 2] == 5
    ro = np.zeros(3)
    ro.flags.writeable = False
    with pytest.raises(TypeError):
        spyker.wrap_array(ro, writeable=True)
    with pytest.raises(ValueError):
        spyker.create_tensor("cpu", "f32", [-1])
    assert spyker.create_array(a, "u8", [4]).dtype == np.uint8
    assert spyker.create_array(torch.zeros(1), "f64", [2]).dtype == torch.float64
    assert callable(utils.read_mnist) and callable(utils.read_csv) and callable(utils.to_sparse)


@pytest.mark.gpu
def test_wrap_device_pointer():
    x = torch.arange(12, dtype=torch.float32, device="cuda")
    y = spyker.create_tensor(torch.device("cuda", 0), "f32", [3, 4], data=x.data_ptr())
    y[0, 0] = -1
    torch.cuda.synchronize()
    assert y.is_cuda and float(x[0]) == -1 and float(y[2, 3]) == 11
