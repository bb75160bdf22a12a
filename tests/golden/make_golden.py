"""Generate the golden fixtures from the reference CPU build.

Runs Spyker's own CPU backend (``oracle/_ref/libspyker_ref.so``, compiled from
the reference sources by ``oracle/Makefile``) on seeded synthetic inputs of
the config-0 pipeline and stores every intermediate result in
``tests/golden/cfg0_small.npz``:

  strokes u8 [16, 28, 28] -> /255 -> DoG(7x7, (1,2), (2,1), pad 3)
  -> rank code T=15 -> conv 30x5x5 pad 2 (weights N(0.8, 0.05) clipped)
  -> threshold 15 -> inhibit -> convwta(r=3, k=5) -> fire -> conv STDP
  (0.004, -0.003, soft bound) -> pool 2x2; plus the latency code, the sparse
  event-list path (code, conv+fire, inhibit, convwta, STDP, pool) and the
  fc / temporal-backprop helpers on small seeded inputs.

Large float tensors are stored as SHA-256 digests of their bytes.

Usage: python tests/golden/make_golden.py   (needs the reference tree to build
oracle/_ref; the fixture is committed, the GPU box never runs this).
"""

from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
import importlib.util  # noqa: E402

# the synthetic-data module by file path: the package itself would load the
# GPU library, which the CPU-only users of this file (bench.py's reference
# arm) must not do
_spec = importlib.util.spec_from_file_location("spyker_synth", os.path.join(ROOT, "spyker_b200", "synth.py"))
synth = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(synth)

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cfg0_small.npz")
CFG = [(0.004, -0.003, 1.0, 0.0, 1.0)]


def digest(a: np.ndarray) -> np.ndarray:
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest(), dtype=np.uint8)


def dog_kernel(o) -> np.ndarray:
    k = np.zeros((2, 2, 7, 7))
    k[0, 0], k[1, 0] = o.gaussian_kernel(7, 1.0), o.gaussian_kernel(7, 2.0)
    k[0, 1], k[1, 1] = o.gaussian_kernel(7, 2.0), o.gaussian_kernel(7, 1.0)
    return k.astype(np.float32)


def run(o, n: int = 16) -> dict:
    d = {}
    img = synth.strokes(n, seed=0)
    d["images"] = img
    x = img.astype(np.float32) / np.float32(255)
    dk = dog_kernel(o)
    d["dog_kernel"] = dk
    dog = o.filter("dog", x[:, None], dk, (3, 3, 3, 3))
    d["dog"] = dog
    codes = o.rank_code(dog, 15)
    d["codes"] = codes
    d["codes_latency"] = o.rank_code(dog, 15, sort=False)
    w = synth.conv_weights(30, 2, 5, seed=1)
    d["kernel"] = w
    pot = o.conv(codes, w, (1, 1), (2, 2, 2, 2))
    d["potentials_sha"] = digest(pot)
    th = o.threshold(pot, 15.0)
    inh = o.inhibit(th)
    d["inhibited_sha"] = digest(inh)
    win, cnt = o.convwta(inh, (3, 3), 5)
    d["winners"], d["counts"] = win, cnt
    spk = o.fire(inh)
    d["fire"] = spk
    d["stdp_kernel"] = o.convstdp(codes, w, spk, CFG, win, cnt, (1, 1), (2, 2, 2, 2))
    d["pooled"] = o.pool(spk, (2, 2))
    d["gather"] = o.gather(spk)
    # sparse event-list path
    ev = o.sparse_code(dog, 15)
    d["sp_code_off"], d["sp_code_zyx"] = ev
    shp = (n, 15, 2, 28, 28)
    (so, sz), oshape = o.sparse_conv(ev, shp, w, 15.0, (2, 2, 2, 2))
    d["sp_conv_off"], d["sp_conv_zyx"] = so, sz
    ih = o.sparse_inhibit((so, sz), oshape)
    d["sp_inhibit_off"], d["sp_inhibit_zyx"] = ih
    sw, sc = o.sparse_convwta(ih, oshape, (3, 3), 5)
    d["sp_winners"], d["sp_counts"] = sw, sc
    d["sp_stdp_kernel"] = o.sparse_stdp(ev, shp, w, CFG, sw, sc, (2, 2, 2, 2))
    (po, pz), _ = o.sparse_pool((so, sz), oshape, (2, 2), (1, 1, 1, 1))
    d["sp_pool_off"], d["sp_pool_zyx"] = po, pz
    # fc / temporal-backprop helpers
    rng = np.random.default_rng(4)
    fx = (rng.random((8, 15, 40)) * 3).astype(np.float32)
    d["fc_in"] = fx
    d["fcwta_winners"], d["fcwta_counts"] = o.fcwta(fx, 2, 3, 1.0)
    tim = (rng.random((16, 10)) * 20).astype(np.float32)
    tg = rng.integers(0, 10, 16).astype(np.int64)
    d["bw_in"], d["bw_target"] = tim, tg
    d["bw_out"] = o.backward(tim, tg, 15, 2.0)
    d["labels"] = o.labelize(fx, 2.5)
    return d


def main() -> None:
    oracle.build()
    if not oracle.available("reference"):
        raise SystemExit("the reference CPU build is required to generate fixtures")
    d = run(oracle.get("reference"))
    np.savez_compressed(OUT, **d)
    print(f"wrote {OUT} ({os.path.getsize(OUT)} bytes)")


if __name__ == "__main__":
    main()
