"""ORACLE — test infrastructure only: NumPy FP64 restatement of first-spike
layers and of the temporal-backprop rule, the checker of
``spyker_b200/csrc/temporal.cu`` (never the product).

Rule (src/spyker/cpu/backprop.cpp, fc backward):
  * target rule ``(desired - t) / T``                       backprop.cpp:40-52
  * ``select = (t_in < t_out) * grad``                      backprop.cpp:116-119
  * ``next   = sum_j kernel * select``                      backprop.cpp:140-144
Here written for a conv weight shared over output pixels, in autograd's sign
(``grad_out = dL/dt_out = -grad``).  Layer forward: the potential at step t
is the conv of the cumulative input spikes ``[t_in <= t]`` (cpu/conv.cpp
semantics: cross-correlation, zero pad, stride; shape.cpp:35-50); the output
time is the first step with potential > threshold, else T (cpu/time.cpp:40-58).
"""

from __future__ import annotations

import numpy as np


def _windows(t_in, kh, kw, stride, pad, never):
    """Padded input times and the (iy, ix) index grids of every output pixel."""
    b, c, h, w = t_in.shape
    top, left, bottom, right = pad
    sy, sx = stride
    xp = np.full((b, c, h + top + bottom, w + left + right), never, dtype=np.float64)
    xp[:, :, top:top + h, left:left + w] = t_in
    oh = (h + top + bottom - kh) // sy + 1
    ow = (w + left + right - kw) // sx + 1
    # [B, C, OH, OW, KH, KW]
    iy = (np.arange(oh) * sy)[:, None] + np.arange(kh)[None, :]
    ix = (np.arange(ow) * sx)[:, None] + np.arange(kw)[None, :]
    patches = xp[:, :, iy[:, None, :, None], ix[None, :, None, :]]
    return patches, oh, ow


def conv_forward(t_in, kernel, threshold, time, stride=(1, 1), pad=(0, 0, 0, 0)):
    """Output first-spike times [B, Z, OH, OW] (float64; ``time`` = never)."""
    kernel = np.asarray(kernel, dtype=np.float64)
    z, c, kh, kw = kernel.shape
    patches, oh, ow = _windows(np.asarray(t_in, np.float64), kh, kw, stride, pad, float(time))
    out = np.full((t_in.shape[0], z, oh, ow), float(time))
    for t in range(time - 1, -1, -1):
        spk = (patches <= t).astype(np.float64)  # [B, C, OH, OW, KH, KW]
        pot = np.einsum("bcyxij,zcij->bzyx", spk, kernel)
        out = np.where(pot > threshold, float(t), out)
    return out


def prespike(t_in, kernel, t_out, stride=(1, 1), pad=(0, 0, 0, 0), time=None):
    """Potential one step before each output spike: sum W * [t_in < t_out]."""
    kernel = np.asarray(kernel, dtype=np.float64)
    z, c, kh, kw = kernel.shape
    never = float(time if time is not None else np.inf)
    patches, oh, ow = _windows(np.asarray(t_in, np.float64), kh, kw, stride, pad, never)
    mask = patches[:, None] < np.asarray(t_out, np.float64)[:, :, None, :, :, None, None]  # [B,Z,C,OH,OW,KH,KW]
    return np.einsum("bzcyxij,zcij->bzyx", mask.astype(np.float64), kernel)


def conv_backward(t_in, kernel, t_out, grad_out, stride=(1, 1), pad=(0, 0, 0, 0)):
    """(grad_in [B, C, H, W], grad_kernel [Z, C, KH, KW]) of the rule above."""
    t_in = np.asarray(t_in, np.float64)
    kernel = np.asarray(kernel, np.float64)
    go = np.asarray(grad_out, np.float64)
    b, c, h, w = t_in.shape
    z, _, kh, kw = kernel.shape
    top, left, bottom, right = pad
    sy, sx = stride
    patches, oh, ow = _windows(t_in, kh, kw, stride, pad, np.inf)
    mask = (patches[:, None] < np.asarray(t_out, np.float64)[:, :, None, :, :, None, None]).astype(np.float64)
    gk = -np.einsum("bzcyxij,bzyx->zcij", mask, go)
    # grad_in: scatter W * go * mask back to the (padded) input positions
    contrib = mask * kernel[None, :, :, None, None, :, :] * go[:, :, None, :, :, None, None]
    contrib = contrib.sum(axis=1)  # [B, C, OH, OW, KH, KW]
    gpad = np.zeros((b, c, h + top + bottom, w + left + right))
    for i in range(kh):
        for j in range(kw):
            gpad[:, :, i:i + sy * (oh - 1) + 1:sy, j:j + sx * (ow - 1) + 1:sx] += contrib[:, :, :, :, i, j]
    return gpad[:, :, top:top + h, left:left + w], gk


def pool_forward(t_in, kernel2, stride2=None, pad=(0, 0, 0, 0), time=None):
    """Earliest time of each window (cpu/pool.cpp:41-86 on cumulative spikes)."""
    kh, kw = kernel2
    stride2 = stride2 or kernel2
    patches, oh, ow = _windows(np.asarray(t_in, np.float64), kh, kw, stride2, pad, float(time))
    return patches.min(axis=(-2, -1))


def pool_backward(t_in, grad_out, kernel2, stride2=None, pad=(0, 0, 0, 0)):
    """Each window's gradient to its earliest in-range input, first in raster
    order on ties."""
    t_in = np.asarray(t_in, np.float64)
    kh, kw = kernel2
    sy, sx = stride2 or kernel2
    top, left = pad[0], pad[1]
    b, c, h, w = t_in.shape
    go = np.asarray(grad_out, np.float64)
    gi = np.zeros_like(t_in)
    for oy in range(go.shape[2]):
        for ox in range(go.shape[3]):
            ys = [y for y in range(oy * sy - top, oy * sy - top + kh) if 0 <= y < h]
            xs = [x for x in range(ox * sx - left, ox * sx - left + kw) if 0 <= x < w]
            win = t_in[:, :, ys][:, :, :, xs].reshape(b, c, -1)
            k = win.argmin(axis=-1)  # first minimum in raster order
            yy = np.array(ys)[k // len(xs)]
            xx = np.array(xs)[k % len(xs)]
            for bi in range(b):
                for ci in range(c):
                    gi[bi, ci, yy[bi, ci], xx[bi, ci]] += go[bi, ci, oy, ox]
    return gi


def target_rule(t_out, target, time, gamma):
    """(desired - t) / T of cpu/backprop.cpp:40-52 ([B, N] float64)."""
    t_out = np.asarray(t_out, np.float64)
    out = np.empty_like(t_out)
    for i in range(t_out.shape[0]):
        o = t_out[i].copy()
        mn = o.min()
        upper = mn + gamma
        value = min(float(time), upper)
        if mn != time:
            o = np.where(o < upper, value, o)
        o[target[i]] = max(0.0, mn)
        out[i] = (o - t_out[i]) / time
    return out
