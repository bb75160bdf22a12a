"""Build the sm_100a C-ABI library ``spyker_b200/lib/libspyker_b200.so``.

Every ``csrc/*.cu`` is compiled by ``nvcc`` for ``sm_100a`` (objects under
``spyker_b200/_build``) and linked, with the CUDA runtime linked statically,
into one shared library that exports the ``spk_*`` entry points declared in
``include/spyker_b200.h``.  The build is incremental (object newer than its
source and the shared headers is reused).
"""

from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libspyker_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Host code is built like the reference's CPU library (-O3, AVX2 + FMA with
# GCC's default contraction) so the host-side kernel generators round alike.
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3,-march=x86-64-v3", "--expt-relaxed-constexpr",
         "-I", os.path.join(ROOT, "include")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, hmtime: float, verbose: bool) -> str:
    obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hmtime):
        return obj
    cmd = [nvcc(), *ARCH, *FLAGS, "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{res.stdout}\n{res.stderr}")
    return obj


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hm = float("inf") if force else _headers_mtime()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, hm, verbose), srcs))
    if not os.path.exists(LIB) or force or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIB


def build_plugin(verbose: bool = False, force: bool = False) -> str:
    """The pybind11 module ``spyker_b200_plugin`` (plugin/plugin.cpp over the
    C++ layer include/spyker_b200.hpp) next to the library, which it links."""
    import sysconfig

    import pybind11

    src = os.path.join(HERE, "plugin", "plugin.cpp")
    out = os.path.join(LIB_DIR, "spyker_b200_plugin" + sysconfig.get_config_var("EXT_SUFFIX"))
    deps = [src, LIB, os.path.join(ROOT, "include", "spyker_b200.hpp"), os.path.join(ROOT, "include", "spyker_b200.h")]
    if os.path.exists(out) and not force and os.path.getmtime(out) >= max(os.path.getmtime(d) for d in deps):
        return out
    cuda = os.path.dirname(os.path.dirname(nvcc()))
    cmd = [shutil.which("g++") or "g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(cuda, "include"), "-I", pybind11.get_include(), "-I", sysconfig.get_paths()["include"],
           src, "-o", out, "-L", LIB_DIR, "-lspyker_b200", "-L", os.path.join(cuda, "lib64"), "-lcudart",
           "-Wl,-rpath,$ORIGIN", "-Wl,-rpath," + os.path.join(cuda, "lib64")]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"plugin build failed:\n{res.stdout}\n{res.stderr}")
    return out


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
    print(build_plugin(verbose="-v" in sys.argv, force="-f" in sys.argv))
