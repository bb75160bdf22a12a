"""Canny and quantize of the reference build (cpu/canny.cpp, cpu/fire.cpp,
compiled in oracle/_ref) on CPU: quantize against its NumPy statement, and
Canny's defining behaviour on a step edge (a strong edge along the step,
nothing in flat regions, u8 out)."""

import numpy as np


def test_quantize_matches_statement(ref):
    rng = np.random.default_rng(0)
    for dt in (np.float32, np.float64, np.int32, np.uint8):
        x = (rng.random(1000) * 200).astype(dt)
        got = ref.quantize(x, 3, 100.5, 250)
        mid = dt(100.5)  # the middle value converted to the type first
        assert np.array_equal(got, np.where(x < mid, dt(3), dt(250)).astype(dt))


def test_canny_step_edge(ref):
    img = np.zeros((2, 32, 32), dtype=np.uint8)
    img[:, :, 16:] = 200
    out = ref.canny(img, 50, 100)
    assert out.dtype == np.uint8 and out.shape == img.shape
    # the strongest response sits on the step, away from the borders
    cols = out[0, 4:28].astype(int).sum(axis=0)
    assert cols.argmax() in (15, 16)
    assert out[0, 4:28, 14:18].max() == 255
    assert (out[0, 4:28, :10] == 0).all() and (out[0, 4:28, 23:] == 0).all()
    assert np.array_equal(out[0], out[1])


def test_canny_reference_is_run_deterministically(ref):
    # the shim runs cpu/canny.cpp on one thread: its per-image scratch planes
    # alias other images' buffers, so threads would race
    from spyker_b200 import synth
    img = synth.strokes(24, seed=5)
    assert np.array_equal(ref.canny(img, 30, 120), ref.canny(img, 30, 120))
