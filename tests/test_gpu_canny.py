"""Canny edges and quantize on the GPU against the reference build
(cpu/canny.cpp, cpu/fire.cpp compiled in oracle/_ref): quantize bit for
bit in four types; Canny on smooth synthetic textures, stroke images and
edge cases (flat, tiny, 3-D input).  The direction is F32 atan2 on both
sides (CUDA's and glibc's may differ in the last place), so Canny is
checked for pixel agreement >= 99.99 %, and exactly on images whose
directions sit away from the bin edges."""

import numpy as np
import pytest
import torch

import spyker_b200 as spyker
from spyker_b200 import synth

pytestmark = pytest.mark.gpu
DEV = "cuda"


@pytest.mark.parametrize("dtype", [np.uint8, np.int32, np.float32, np.float64])
def test_quantize_bit_exact(ref, dtype):
    x = (np.random.default_rng(1).random((7, 33, 5)) * 200).astype(dtype)
    want = ref.quantize(x, 3, 100.5, 250)
    t = torch.from_numpy(x.copy()).to(DEV)
    got = spyker.quantize(t, 3, 100.5, 250)
    assert got is t and np.array_equal(t.cpu().numpy(), want)
    keep = x.copy()
    y = spyker.quantize(x, 3, 100.5, 250, inplace=False)
    assert np.array_equal(x, keep) and np.array_equal(y, want)


def _agree(a, b):
    return float((a == b).mean())


def test_canny_textures_and_strokes(ref):
    tex = (synth.textures(6, size=96, seed=4) * 255).astype(np.uint8)[:, None]
    strokes = synth.strokes(64, seed=5)[:, None]
    for img, lo, hi in ((tex, 40, 90), (tex, 0, 255), (strokes, 30, 120), (strokes, 0, 255), (strokes, 255, 255)):
        got = spyker.canny(torch.from_numpy(img).to(DEV), lo, hi).cpu().numpy()
        want = ref.canny(img, lo, hi)
        assert got.shape == img.shape and got.dtype == np.uint8
        assert _agree(got, want) >= 0.9999, _agree(got, want)
        assert (want == 255).any()


def test_canny_axis_aligned_exact(ref):
    # edges along rows / columns: directions of 0 or 90 degrees exactly
    img = np.zeros((3, 1, 40, 50), dtype=np.uint8)
    img[0, 0, :, 20:] = 180
    img[1, 0, 10:30, :] = 90
    img[2, 0, 5:35, 8:40] = 250
    got = spyker.canny(img, 20, 60)
    assert isinstance(got, np.ndarray)
    assert np.array_equal(got, ref.canny(img, 20, 60))


def test_canny_edge_cases(ref):
    cases = [np.zeros((2, 16, 16), np.uint8), np.full((1, 9, 9), 77, np.uint8),
             np.random.default_rng(2).integers(0, 256, (4, 2, 2), dtype=np.uint8),
             np.random.default_rng(3).integers(0, 256, (1, 3, 7), dtype=np.uint8)]
    for img in cases:
        for lo, hi in ((0, 0), (10, 200)):
            got = spyker.canny(torch.from_numpy(img).to(DEV), lo, hi).cpu().numpy()
            assert np.array_equal(got, ref.canny(img, lo, hi)), (img.shape, lo, hi)
    with pytest.raises(TypeError):
        spyker.canny(torch.zeros((1, 8, 8), device=DEV), 1, 2)


def test_canny_multichannel_and_3d(ref):
    # [N, C, H, W] is processed as N * C images; 3-D input as one batch
    img = (synth.textures(3, size=40, seed=9) * 255).astype(np.uint8).reshape(3, 1, 40, 40)
    img = np.concatenate([img, img[:, :, ::-1].copy()], axis=1)  # 2 channels
    got = spyker.canny(torch.from_numpy(img).to(DEV), 35, 80).cpu().numpy()
    assert got.shape == img.shape
    assert np.array_equal(got, ref.canny(img, 35, 80))
    flat = img.reshape(6, 40, 40)
    assert np.array_equal(spyker.canny(torch.from_numpy(flat).to(DEV), 35, 80).cpu().numpy(),
                          ref.canny(flat, 35, 80))
