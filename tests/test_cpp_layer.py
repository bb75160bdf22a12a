"""The C++ ``Spyker::`` layer (include/spyker_b200.hpp) over the C ABI.

CPU: the header compiles with the reference's names, and a program using
it links against the library.  GPU: that program runs one layer step (DoG,
rank code, the plain FP32 ops, the fused tensor-core layer with pooling, STDP
on its winners) and every result equals the Python API's on the same
inputs."""

import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "layer_check.cpp")
LIB = os.path.join(ROOT, "spyker_b200", "lib")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")

pytestmark = pytest.mark.skipif(shutil.which("g++") is None or not os.path.exists(os.path.join(CUDA, "include")),
                                reason="needs g++ and the CUDA headers")


def _flags():
    return ["-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(ROOT, "include"),
            "-I" + os.path.join(CUDA, "include")]


def _build(tmp_path) -> str:
    exe = str(tmp_path / "layer_check")
    subprocess.check_call(["g++", *_flags(), SRC, "-o", exe, "-L" + LIB, "-lspyker_b200",
                           "-L" + os.path.join(CUDA, "lib64"), "-lcudart", "-Wl,-rpath," + LIB,
                           "-Wl,-rpath," + os.path.join(CUDA, "lib64")])
    return exe


def test_header_compiles():
    subprocess.check_call(["g++", *_flags(), "-fsyntax-only", SRC])


def test_program_links(tmp_path):
    if not os.path.exists(os.path.join(LIB, "libspyker_b200.so")):
        pytest.skip("library not built")
    assert os.path.exists(_build(tmp_path))


def _load(d, name, dtype, shape=None):
    a = np.fromfile(os.path.join(d, name + ".bin"), dtype=dtype)
    return a.reshape(shape) if shape is not None else a


def _winners(w):
    rows = []
    for i, lst in enumerate(w):
        for x in lst:
            rows.append((i, x.c, x.t, x.z, x.y, x.x))
    return np.array(rows, dtype=np.int64).reshape(-1, 6)


@pytest.mark.gpu
def test_cpp_layer_matches_python(tmp_path):
    import torch

    import spyker_b200 as spyker

    exe = _build(tmp_path)
    out = tmp_path / "out"
    out.mkdir()
    r = subprocess.run([exe, str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    b, t, h, w = 6, 15, 20, 18
    dev = torch.device("cuda", 0)
    images = torch.from_numpy(_load(out, "images", np.float32, (b, 1, h, w))).to(dev)
    dog = spyker.DoG(3, [spyker.DoGFilter(1, 2), spyker.DoGFilter(2, 1)], pad=3, device=dev)
    codes = spyker.code(dog(images), t)
    assert np.array_equal(codes.cpu().numpy(), _load(out, "codes", np.uint8, (b, t, 2, h, w)))
    conv = spyker.Conv(2, 12, 5, pad=2, device=dev)
    conv.kernel.copy_(torch.from_numpy(_load(out, "kernel0", np.float32, (12, 2, 5, 5))))
    conv.stdpconfig = [spyker.STDPConfig(0.004, -0.003)]
    conv.precision = "fp32"
    o = spyker.inhibit(spyker.threshold(conv(codes), 4.0))
    spk = spyker.fire(o)
    assert np.array_equal(spk.cpu().numpy().ravel(), _load(out, "spikes_ops", np.uint8))
    assert np.array_equal(spyker.pool(spk, 2).cpu().numpy().ravel(), _load(out, "pooled_ops", np.uint8))
    assert np.array_equal(_winners(spyker.convwta(o, 2, 3)), _load(out, "winners_ops", np.int64).reshape(-1, 6))
    conv.precision = "bf16x3"
    spk, wins, pooled = spyker.conv_fire_wta(codes, conv, 4.0, 2, 3, pool=2)
    assert np.array_equal(spk.cpu().numpy().ravel(), _load(out, "spikes_fused", np.uint8))
    assert np.array_equal(pooled.cpu().numpy().ravel(), _load(out, "pooled_fused", np.uint8))
    got_w = _load(out, "winners_fused", np.int64).reshape(-1, 6)
    assert np.array_equal(_winners(wins), got_w) and got_w.shape[0] > 0
    conv.stdp(codes, wins, spk)
    k1 = _load(out, "kernel1", np.float32, (12, 2, 5, 5))
    assert np.array_equal(conv.kernel.cpu().numpy(), k1)
    assert not np.array_equal(k1, _load(out, "kernel0", np.float32, (12, 2, 5, 5)))
