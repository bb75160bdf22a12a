"""Temporal backprop through first-spike layers, on torch.autograd.

A rank-coded layer maps input first-spike times to output first-spike times:
the input times become cumulative spikes (``scatter``), the tensor-core conv
gives the potentials at every step, and the output time of a neuron is the
first step whose potential exceeds the threshold (``gather``; T = never).
The backward is the reference's temporal-backprop rule (the fc backward of
src/spyker/cpu/backprop.cpp:105-160: ``select = (t_in < t_out) * grad``,
``next = sum kernel * select``) for conv and fc layers, run by the
hand-written kernels of ``csrc/temporal.cu`` (``spk_fst_conv_backward``,
``spk_fst_pool_backward``).  Only the first-spike times are saved for the
backward, never the [B, T, ...] potentials; the kernel gradient is the exact
derivative of the potential-level loss ``sum g * V(t_out - 1)`` that
:func:`prespike` recomputes in FP64.

Times are F32 tensors ``[B, C, H, W]`` (fc: ``[B, N]``) holding 0..T.
"""

from __future__ import annotations

import numpy
import torch

from . import _lib
from . import module as M
from ._lib import call, i64, ptr, stream
from .utils import expand2, expand4

# Potentials of at most this many bytes are materialised at once (the batch
# is split into chunks beyond it).
_CHUNK_BYTES = 4 << 30


def _ws(nbytes: int, dev: torch.device):
    return M._workspace(nbytes, dev)


def times_of(spikes: torch.Tensor) -> torch.Tensor:
    """First-spike times F32 ``[B, ...]`` of cumulative spikes ``[B, T, ...]``."""
    return M.gather(spikes, 0.0, dtype="f32")


def conv_forward(t_in: torch.Tensor, kernel: torch.Tensor, threshold: float, time: int, stride=1, pad=0,
                 precision: str = "bf16x3") -> torch.Tensor:
    """Output first-spike times of a conv layer (no gradient tracking).

    On the tensor-core precisions one fused kernel (``spk_fst_conv_times``)
    writes the times without materialising the potentials; otherwise (FP32,
    or layers that do not fit one CTA) the potentials of every step are
    computed and gathered, in batch chunks."""
    s2, p4 = expand2(stride), expand4(pad)
    b = t_in.shape[0]
    if precision != "fp32" and time <= 126:
        k = kernel.float().contiguous()
        ti = t_in.float().contiguous()
        _, c, h, w = ti.shape
        z, _, kh, kw = k.shape
        nb = _lib.lib.spk_fst_conv_times_workspace(b, c, h, w, z, kh, kw, time, M._PRECISION[precision])
        if nb > 0:
            oh = (h + p4[0] + p4[2] - kh) // s2[0] + 1
            ow = (w + p4[1] + p4[3] - kw) // s2[1] + 1
            out = torch.empty((b, z, oh, ow), dtype=torch.float32, device=ti.device)
            ws, wsb = _ws(nb, ti.device)
            call("spk_fst_conv_times", ptr(ti), b, c, h, w, ptr(k), z, kh, kw, s2[0], s2[1], i64(*p4), int(time),
                 float(threshold), ptr(out), M._PRECISION[precision], ptr(ws), wsb, stream())
            return out
    z = kernel.shape[0]
    oh = (t_in.shape[2] + p4[0] + p4[2] - kernel.shape[2]) // s2[0] + 1
    ow = (t_in.shape[3] + p4[1] + p4[3] - kernel.shape[3]) // s2[1] + 1
    per_sample = time * z * oh * ow * 4
    step = max(1, min(b, _CHUNK_BYTES // max(per_sample, 1)))
    outs = []
    for s in range(0, b, step):
        ti = t_in[s:s + step]
        spikes = M.scatter(ti.reshape(ti.shape[0], -1), time).view(ti.shape[0], time, *ti.shape[1:])
        pot = M.conv(spikes, kernel, s2, p4, precision=precision)
        outs.append(M.gather(pot, float(threshold), dtype="f32"))
        del spikes, pot
    return outs[0] if len(outs) == 1 else torch.cat(outs)


def conv_backward(t_in, kernel, t_out, grad_out, stride=1, pad=0, need_input: bool = True, need_kernel: bool = True):
    """(grad_in, grad_kernel) of a first-spike conv layer (either may be None)."""
    s2, p4 = expand2(stride), expand4(pad)
    t_in, kernel = t_in.contiguous(), kernel.contiguous()
    t_out, grad_out = t_out.contiguous(), grad_out.float().contiguous()
    b, c, h, w = t_in.shape
    z, _, kh, kw = kernel.shape
    oh, ow = t_out.shape[2], t_out.shape[3]
    gi = torch.empty_like(t_in) if need_input else None
    gk = torch.empty_like(kernel) if need_kernel else None
    nb = _lib.lib.spk_fst_conv_backward_workspace(b, c, z, kh, kw) if need_kernel else 0
    ws, wsb = _ws(nb, t_in.device)
    call("spk_fst_conv_backward", ptr(t_in), b, c, h, w, ptr(kernel), z, kh, kw, ptr(t_out), ptr(grad_out), oh, ow,
         i64(*s2), i64(*p4), ptr(gi), ptr(gk), ptr(ws), wsb, stream())
    return gi, gk


def prespike(t_in, kernel, t_out, stride=1, pad=0) -> torch.Tensor:
    """FP64 potential one step before each output spike, [B, Z, OH, OW]."""
    s2, p4 = expand2(stride), expand4(pad)
    t_in, kernel, t_out = t_in.contiguous(), kernel.contiguous(), t_out.contiguous()
    b, c, h, w = t_in.shape
    z, _, kh, kw = kernel.shape
    out = torch.empty(t_out.shape, dtype=torch.float64, device=t_in.device)
    call("spk_fst_conv_prespike", ptr(t_in), b, c, h, w, ptr(kernel), z, kh, kw, ptr(t_out), t_out.shape[2],
         t_out.shape[3], i64(*s2), i64(*p4), ptr(out), stream())
    return out


def pool_forward(t_in: torch.Tensor, kernel, time: int, stride=None, pad=0) -> torch.Tensor:
    """Earliest spike time of each window (pool of cumulative spikes)."""
    k2 = expand2(kernel)
    s2 = expand2(kernel if stride is None else stride)
    p4 = expand4(pad)
    t_in = t_in.contiguous()
    b, c, h, w = t_in.shape
    oh = (h + p4[0] + p4[2] - k2[0]) // s2[0] + 1
    ow = (w + p4[1] + p4[3] - k2[1]) // s2[1] + 1
    out = torch.empty((b, c, oh, ow), dtype=torch.float32, device=t_in.device)
    call("spk_fst_pool", ptr(t_in), b, c, h, w, ptr(out), oh, ow, i64(*k2), i64(*s2), i64(*p4), float(time), stream())
    return out


def pool_backward(t_in, grad_out, kernel, stride=None, pad=0) -> torch.Tensor:
    k2 = expand2(kernel)
    s2 = expand2(kernel if stride is None else stride)
    p4 = expand4(pad)
    t_in, grad_out = t_in.contiguous(), grad_out.float().contiguous()
    b, c, h, w = t_in.shape
    gi = torch.empty_like(t_in)
    call("spk_fst_pool_backward", ptr(t_in), b, c, h, w, ptr(grad_out), grad_out.shape[2], grad_out.shape[3],
         i64(*k2), i64(*s2), i64(*p4), ptr(gi), stream())
    return gi


class FirstSpikeConv(torch.autograd.Function):
    """t_out = first-spike conv layer(t_in; kernel)."""

    @staticmethod
    def forward(ctx, t_in, kernel, threshold, time, stride, pad, precision):
        t_out = conv_forward(t_in, kernel, threshold, time, stride, pad, precision)
        ctx.save_for_backward(t_in, kernel, t_out)
        ctx.geo = (stride, pad)
        return t_out

    @staticmethod
    def backward(ctx, grad_out):
        t_in, kernel, t_out = ctx.saved_tensors
        stride, pad = ctx.geo
        gi, gk = conv_backward(t_in, kernel, t_out, grad_out, stride, pad, ctx.needs_input_grad[0],
                               ctx.needs_input_grad[1])
        return gi, gk, None, None, None, None, None


class FirstSpikePool(torch.autograd.Function):
    @staticmethod
    def forward(ctx, t_in, kernel, time, stride, pad):
        ctx.save_for_backward(t_in)
        ctx.geo = (kernel, stride, pad)
        return pool_forward(t_in, kernel, time, stride, pad)

    @staticmethod
    def backward(ctx, grad_out):
        (t_in,) = ctx.saved_tensors
        kernel, stride, pad = ctx.geo
        return pool_backward(t_in, grad_out, kernel, stride, pad), None, None, None, None


class FirstSpikeLoss(torch.autograd.Function):
    """Loss of the reference's target rule (cpu/backprop.cpp:40-52):
    L = sum (desired - t)^2 / (2 T), desired held fixed, so dL/dt =
    -(desired - t) / T = -backward(t, target, T, gamma)."""

    @staticmethod
    def forward(ctx, t_out, target, time, gamma):
        g = M.backward(t_out, target, time, gamma)
        ctx.save_for_backward(g)
        return (g.double() ** 2).sum() * (0.5 * time)

    @staticmethod
    def backward(ctx, gl):
        (g,) = ctx.saved_tensors
        return -g * gl.to(g.dtype), None, None, None


def first_spike_conv(t_in, kernel, threshold: float, time: int, stride=1, pad=0, precision: str = "bf16x3"):
    return FirstSpikeConv.apply(t_in, kernel, float(threshold), int(time), stride, pad, precision)


def first_spike_pool(t_in, kernel, time: int, stride=None, pad=0):
    return FirstSpikePool.apply(t_in, kernel, int(time), stride, pad)


def first_spike_fc(t_in, kernel, threshold: float, time: int, precision: str = "bf16x3"):
    """fc layer [B, N] -> [B, O] as the 1x1 conv of [B, N, 1, 1]."""
    b, n = t_in.shape[0], t_in[0].numel()
    o = kernel.shape[0]
    out = FirstSpikeConv.apply(t_in.reshape(b, n, 1, 1), kernel.reshape(o, n, 1, 1), float(threshold), int(time), 1,
                               0, precision)
    return out.reshape(b, o)


def first_spike_loss(t_out, target, time: int, gamma: float):
    return FirstSpikeLoss.apply(t_out, target, int(time), float(gamma))


class TemporalNet:
    """conv 32x5x5 -> pool 2 -> conv 64x3x3 -> pool 2 -> fc 10 over rank-coded
    28x28 images, trained through the output first-spike times.  Weights F32
    ~U(0, 0.1) (seeded)."""

    def __init__(self, time: int = 64, thresholds=(0.5, 2.0, 40.0), gamma: float = 3.0, seed: int = 4,
                 device=None, precision: str = "bf16x3", in_channels: int = 1, size: int = 28):
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        rng = numpy.random.default_rng(seed)
        s = size // 2 // 2
        shapes = [(32, in_channels, 5, 5), (64, 32, 3, 3), (10, 64 * s * s)]
        self.weights = [torch.from_numpy(rng.uniform(0.0, 0.1, size=sh).astype(numpy.float32)).to(dev)
                        .requires_grad_(True) for sh in shapes]
        self.time, self.thresholds, self.gamma, self.precision = time, thresholds, gamma, precision

    def input_times(self, images: torch.Tensor) -> torch.Tensor:
        """Rank-order first-spike times of images [B, C, H, W] in [0, 1]."""
        return times_of(M.code(images, self.time))

    def forward(self, t0: torch.Tensor) -> torch.Tensor:
        T, th, p = self.time, self.thresholds, self.precision
        w1, w2, w3 = self.weights
        x = first_spike_conv(t0, w1, th[0], T, 1, 2, p)
        x = first_spike_pool(x, 2, T)
        x = first_spike_conv(x, w2, th[1], T, 1, 1, p)
        x = first_spike_pool(x, 2, T)
        return first_spike_fc(x.reshape(x.shape[0], -1), w3, th[2], T, p)

    def loss(self, t_out, target) -> torch.Tensor:
        return first_spike_loss(t_out, target, self.time, self.gamma)

    def step(self, images, target, lrate: float = 1e-4):
        """One training step (forward, loss, backward, SGD); returns the loss
        and the output times.  The loss sums the samples, as the reference's
        fc backward applies one update per sample (cpu/backprop.cpp:112-124)."""
        t_out = self.forward(self.input_times(images))
        loss = self.loss(t_out, target)
        grads = torch.autograd.grad(loss, self.weights)
        with torch.no_grad():
            for w, g in zip(self.weights, grads):
                w.sub_(g, alpha=lrate)
        return loss.detach(), t_out.detach()
