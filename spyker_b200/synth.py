"""Seeded synthetic inputs with the geometry of the reference's examples.

MNIST (used by every reference example) is not available offline, so the
workloads use generated stand-ins with the same shapes and value ranges:

* :func:`strokes` — 28x28 u8 images, zero background, 1-4 anti-aliased
  line/arc strokes 2-3 px wide with intensity U[180, 255];
* :func:`textures` — 256x256 f32 images in [0, 1]: a 1/f-noise texture plus
  8-32 Gaussian blobs (sigma 2-12 px).

Everything is drawn from ``numpy.random.default_rng(seed)``.
"""

from __future__ import annotations

import numpy as np


def _segment_distance(py, px, y0, x0, y1, x1):
    dy, dx = y1 - y0, x1 - x0
    den = dy * dy + dx * dx
    t = np.clip(((py - y0) * dy + (px - x0) * dx) / max(den, 1e-9), 0.0, 1.0)
    return np.hypot(py - (y0 + t * dy), px - (x0 + t * dx))


def _arc_distance(py, px, cy, cx, r, a0, a1):
    ang = np.arctan2(py - cy, px - cx)
    span = (a1 - a0) % (2 * np.pi)
    rel = (ang - a0) % (2 * np.pi)
    inside = rel <= span
    dist_ring = np.abs(np.hypot(py - cy, px - cx) - r)
    e0 = np.hypot(py - (cy + r * np.sin(a0)), px - (cx + r * np.cos(a0)))
    e1 = np.hypot(py - (cy + r * np.sin(a1)), px - (cx + r * np.cos(a1)))
    return np.where(inside, dist_ring, np.minimum(e0, e1))


def strokes(n: int, seed: int = 0, size: int | tuple = 28) -> np.ndarray:
    """``n`` stroke images ``[n, size, size]`` u8 (``size`` may vary per call)."""
    rng = np.random.default_rng(seed)
    h = w = int(size)
    py, px = np.mgrid[0:h, 0:w].astype(np.float64) + 0.5
    out = np.zeros((n, h, w), dtype=np.uint8)
    for i in range(n):
        img = np.zeros((h, w), dtype=np.float64)
        for _ in range(int(rng.integers(1, 5))):
            width = rng.uniform(2.0, 3.0)
            level = rng.uniform(180.0, 255.0)
            if rng.random() < 0.5:
                y0, x0, y1, x1 = rng.uniform(0.15 * h, 0.85 * h, size=4)
                d = _segment_distance(py, px, y0, x0, y1, x1)
            else:
                cy, cx = rng.uniform(0.3 * h, 0.7 * h, size=2)
                r = rng.uniform(0.12 * h, 0.35 * h)
                a0 = rng.uniform(0, 2 * np.pi)
                a1 = a0 + rng.uniform(0.5 * np.pi, 1.6 * np.pi)
                d = _arc_distance(py, px, cy, cx, r, a0, a1)
            cover = np.clip(width / 2.0 + 0.5 - d, 0.0, 1.0)
            img = np.maximum(img, level * cover)
        out[i] = np.clip(np.rint(img), 0, 255).astype(np.uint8)
    return out


def labelled_strokes(n: int, classes: int = 10, seed: int = 4, size: int = 28):
    """``n`` images ``[n, size, size]`` u8 of ``classes`` seeded stroke
    templates (2-3 lines / arcs each) with per-image jitter (shift of up to 2
    px, control points moved by up to 1.5 px, width U[2, 3], intensity
    U[180, 255]), and their labels ``[n]`` int64."""
    rng = np.random.default_rng(seed)
    h = w = int(size)
    templates = []
    for _ in range(classes):
        parts = []
        for _ in range(int(rng.integers(2, 4))):
            if rng.random() < 0.5:
                parts.append(("line", rng.uniform(0.2 * h, 0.8 * h, size=4)))
            else:
                a0 = rng.uniform(0, 2 * np.pi)
                parts.append(("arc", np.array([*rng.uniform(0.35 * h, 0.65 * h, size=2), rng.uniform(0.15 * h, 0.3 * h),
                                               a0, a0 + rng.uniform(0.6 * np.pi, 1.5 * np.pi)])))
        templates.append(parts)
    py, px = np.mgrid[0:h, 0:w].astype(np.float64) + 0.5
    labels = rng.integers(0, classes, size=n).astype(np.int64)
    out = np.zeros((n, h, w), dtype=np.uint8)
    for i in range(n):
        dy, dx = rng.uniform(-2.0, 2.0, size=2)
        img = np.zeros((h, w), dtype=np.float64)
        for kind, prm in templates[labels[i]]:
            width, level = rng.uniform(2.0, 3.0), rng.uniform(180.0, 255.0)
            if kind == "line":
                y0, x0, y1, x1 = prm + rng.uniform(-1.5, 1.5, size=4) + np.array([dy, dx, dy, dx])
                d = _segment_distance(py, px, y0, x0, y1, x1)
            else:
                cy, cx, r, a0, a1 = prm
                d = _arc_distance(py, px, cy + dy + rng.uniform(-1.5, 1.5), cx + dx + rng.uniform(-1.5, 1.5),
                                  r + rng.uniform(-1.0, 1.0), a0, a1)
            img = np.maximum(img, level * np.clip(width / 2.0 + 0.5 - d, 0.0, 1.0))
        out[i] = np.clip(np.rint(img), 0, 255).astype(np.uint8)
    return out, labels


def textures(n: int, seed: int = 2, size: int = 256) -> np.ndarray:
    """``n`` texture images ``[n, size, size]`` f32 in [0, 1]."""
    rng = np.random.default_rng(seed)
    fy = np.fft.fftfreq(size)[:, None]
    fx = np.fft.rfftfreq(size)[None, :]
    f = np.hypot(fy, fx)
    f[0, 0] = 1.0
    amp = 1.0 / f
    amp[0, 0] = 0.0
    yy, xx = np.mgrid[0:size, 0:size].astype(np.float32)
    out = np.zeros((n, size, size), dtype=np.float32)
    for i in range(n):
        phase = rng.uniform(0, 2 * np.pi, size=amp.shape)
        tex = np.fft.irfft2(amp * np.exp(1j * phase), s=(size, size)).astype(np.float32)
        tex = (tex - tex.min()) / max(float(tex.max() - tex.min()), 1e-12)
        img = 0.5 * tex
        for _ in range(int(rng.integers(8, 33))):
            cy, cx = rng.uniform(0, size, size=2)
            s = rng.uniform(2.0, 12.0)
            a = rng.uniform(0.3, 1.0)
            img += a * np.exp(-((yy - cy) ** 2 + (xx - cx) ** 2) / (2 * s * s)).astype(np.float32)
        img = (img - img.min()) / max(float(img.max() - img.min()), 1e-12)
        out[i] = img
    return out


def conv_weights(cout: int, cin: int, k: int, seed: int, mean: float = 0.8, std: float = 0.05) -> np.ndarray:
    """Weights ~ N(mean, std) clipped to [0, 1], f32 ``[cout, cin, k, k]``."""
    rng = np.random.default_rng(seed)
    return np.clip(rng.normal(mean, std, size=(cout, cin, k, k)), 0.0, 1.0).astype(np.float32)
