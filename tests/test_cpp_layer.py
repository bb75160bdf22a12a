"""The C++ ``Spyker::`` layer (include/spyker_b200.hpp) over the C ABI.

CPU: the header compiles with the reference's names, and programs using
it (the layer step, and every module and function of the layer) link
against the library.  GPU: that program runs one layer step (DoG,
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


def test_full_surface_links(tmp_path):
    """Every module and function of the layer named after the reference's
    opers.h (Gabor, LoG, FC with stdp / backward, fc, backward, labelize
    beside the layer-step ones) compiles with the reference's argument forms
    and links against the library."""
    if not os.path.exists(os.path.join(LIB, "libspyker_b200.so")):
        pytest.skip("library not built")
    exe = str(tmp_path / "api_surface")
    subprocess.check_call(["g++", *_flags(), os.path.join(ROOT, "tests", "cpp", "api_surface.cpp"), "-o", exe,
                           "-L" + LIB, "-lspyker_b200", "-L" + os.path.join(CUDA, "lib64"), "-lcudart",
                           "-Wl,-rpath," + LIB])
    assert os.path.exists(exe)


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


def _plugin():
    import importlib.util
    import sysconfig

    path = os.path.join(LIB, "spyker_b200_plugin" + sysconfig.get_config_var("EXT_SUFFIX"))
    if not os.path.exists(path):
        pytest.skip("plugin not built")
    spec = importlib.util.spec_from_file_location("spyker_b200_plugin", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_plugin_surface():
    """The pybind11 module exposes the reference plugin's hot-path names
    (bind.cpp:241-407): modules with their ``_forward`` / ``_stdp`` /
    ``_backward`` methods, the free functions and the ``sparse`` submodule."""
    p = _plugin()
    for name in ("Tensor", "tensor", "from_numpy", "Winner", "DoGFilter", "GaborFilter", "STDPConfig", "BPConfig",
                 "SparseTensor", "DoG", "Gabor", "LoG", "FC", "Conv", "conv", "fc", "pad", "threshold", "code",
                 "infinite", "fire", "gather", "scatter", "pool", "inhibit", "fcwta", "convwta", "backward",
                 "labelize", "conv_fire_wta", "synchronize", "sparse"):
        assert hasattr(p, name), name
    for cls, methods in (("DoG", ["_forward"]), ("Gabor", ["_forward"]), ("LoG", ["_forward"]),
                         ("FC", ["_forward", "_stdp", "_backward"]), ("Conv", ["_forward", "_stdp"]),
                         ("SparseTensor", ["dense", "sparsity"])):
        for meth in methods:
            assert hasattr(getattr(p, cls), meth), f"{cls}.{meth}"
    for name in ("conv", "pad", "code", "gather", "pool", "inhibit", "convwta"):
        assert hasattr(p.sparse, name), f"sparse.{name}"
    assert p.GaborFilter(2.0, 90.0, 0.5, 4.0, 0.0).theta == pytest.approx(np.pi / 2)
    bp = p.BPConfig(1.0, 0.01, 0.1, 0.001)
    assert (bp.sfactor, bp.lrf) == (1.0, pytest.approx(0.1))


@pytest.mark.gpu
def test_plugin_matches_python():
    """A layer step through the plugin on views of torch CUDA tensors equals
    the Python API's: rank code into a given output, the plain ops, the fused
    layer, and STDP with the fused layer's winners."""
    import torch

    import spyker_b200 as spyker

    p = _plugin()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(5)
    b, t = 4, 15
    img = torch.from_numpy(rng.random((b, 2, 20, 22), dtype=np.float32)).to(dev)
    img[img < 0.5] = 0
    codes = torch.empty((b, t, 2, 20, 22), dtype=torch.uint8, device=dev)
    view = lambda x, ty: p.tensor(x.data_ptr(), ty, list(x.shape))  # noqa: E731
    p.code(view(img, "f32"), view(codes, "u8"), t, True, "rank")
    p.synchronize()
    assert torch.equal(codes, spyker.code(img, t))
    w = torch.from_numpy(rng.uniform(0.3, 1.0, size=(10, 2, 5, 5)).astype(np.float32)).to(dev)
    pot = torch.empty((b, t, 10, 20, 22), dtype=torch.float32, device=dev)
    p.conv(view(codes, "u8"), view(w, "f32"), view(pot, "f32"), [1], [2])
    p.threshold(view(pot, "f32"), 4.0, 0.0)
    p.inhibit(view(pot, "f32"), 0.0)
    spk = torch.empty_like(pot, dtype=torch.uint8)
    p.fire(view(pot, "f32"), view(spk, "u8"), 0.0, "rank")
    wins = p.convwta(view(pot, "f32"), [2], 3, 0.0)
    p.synchronize()
    conv = spyker.Conv(2, 10, 5, pad=2)
    conv.kernel.copy_(w)
    conv.precision = "fp32"
    ref = spyker.inhibit(spyker.threshold(conv(codes), 4.0))
    assert torch.equal(spk, spyker.fire(ref))
    rw = spyker.convwta(ref, 2, 3)
    assert [[(x.c, x.t, x.z, x.y, x.x) for x in s] for s in wins] == [[(x.c, x.t, x.z, x.y, x.x) for x in s] for s in rw]
    layer = p.Conv(2, 10, [5], [1], [2], 0.5, 0.02)
    p.from_numpy(w.cpu().numpy())  # host round trip
    layer.kernel = p.from_numpy(w.cpu().numpy())
    layer.precision = p.CONV_BF16X3
    layer.stdpconfig = [p.STDPConfig(0.004, -0.003)]
    fspk, fwins, fpool = p.conv_fire_wta(view(codes, "u8"), layer, 4.0, [2], 3, [2])
    conv.precision = "bf16x3"
    gspk, gwins, gpool = spyker.conv_fire_wta(codes, conv, 4.0, 2, 3, pool=2)
    assert np.array_equal(fspk.numpy(), gspk.cpu().numpy()) and np.array_equal(fpool.numpy(), gpool.cpu().numpy())
    layer._stdp(view(codes, "u8"), fwins, fspk)
    conv.stdpconfig = [spyker.STDPConfig(0.004, -0.003)]
    conv.stdp(codes, gwins, gspk)
    assert np.array_equal(layer.kernel.numpy(), conv.kernel.cpu().numpy())
