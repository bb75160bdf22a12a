"""First-spike layers trained through their spike times, on the GPU: the
hand-written backward kernels (csrc/temporal.cu, through the C ABI) against
the NumPy FP64 restatement (oracle/temporal.py), against the reference's fc
backward (oracle/_ref), and against central finite differences of the
potential-level loss, recomputed in FP64 on the GPU."""

import numpy as np
import pytest
import torch

import spyker_b200 as spyker
from spyker_b200 import synth, temporal
from oracle import temporal as tr

pytestmark = pytest.mark.gpu
DEV = "cuda"


def cuda(a, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV, dtype)


def host(t):
    return t.detach().cpu().numpy()


GEOS = [
    # b, c, h, w, z, k, stride, pad, time
    (3, 4, 9, 8, 5, 3, (1, 1), (1, 1, 1, 1), 16),
    (2, 3, 11, 10, 6, 5, (2, 1), (2, 0, 1, 2), 20),
    (4, 32, 14, 14, 16, 3, (1, 1), (1, 1, 1, 1), 64),
    (5, 70, 1, 1, 10, 1, (1, 1), (0, 0, 0, 0), 32),  # fc as a 1x1 conv
    (2, 1, 28, 28, 8, 5, (1, 1), (2, 2, 2, 2), 64),
    (3, 3136, 1, 1, 10, 1, (1, 1), (0, 0, 0, 0), 64),  # the network's fc: two weight blocks
    (2, 64, 14, 14, 8, 3, (1, 1), (1, 1, 1, 1), 32),  # input times read from global memory
]


def _case(g, seed):
    b, c, h, w, z, k, stride, pad, time = g
    rng = np.random.default_rng(seed)
    t_in = rng.integers(0, time + 1, size=(b, c, h, w)).astype(np.float32)
    kern = rng.uniform(0.0, 0.3, size=(z, c, k, k)).astype(np.float32)
    oh = (h + pad[0] + pad[2] - k) // stride[0] + 1
    ow = (w + pad[1] + pad[3] - k) // stride[1] + 1
    t_out = rng.integers(0, time + 1, size=(b, z, oh, ow)).astype(np.float32)
    go = rng.normal(size=t_out.shape).astype(np.float32)
    return t_in, kern, t_out, go


@pytest.mark.parametrize("g", GEOS)
def test_conv_backward_matches_oracle(g):
    stride, pad = g[6], g[7]
    t_in, kern, t_out, go = _case(g, sum(g[:6]))
    gi, gk = temporal.conv_backward(cuda(t_in), cuda(kern), cuda(t_out), cuda(go), stride, pad)
    wi, wk = tr.conv_backward(t_in, kern, t_out, go, stride, pad)
    np.testing.assert_allclose(host(gk), wk, rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(host(gi), wi, rtol=1e-5, atol=1e-5)
    assert np.abs(wk).sum() > 0 and np.abs(wi).sum() > 0
    # either gradient alone
    gi2, gk2 = temporal.conv_backward(cuda(t_in), cuda(kern), cuda(t_out), cuda(go), stride, pad, need_kernel=False)
    assert gk2 is None and torch.equal(gi2, gi)
    gi3, gk3 = temporal.conv_backward(cuda(t_in), cuda(kern), cuda(t_out), cuda(go), stride, pad, need_input=False)
    assert gi3 is None and torch.equal(gk3, gk)


@pytest.mark.parametrize("g", GEOS[:3])
def test_prespike_matches_oracle(g):
    stride, pad, time = g[6], g[7], g[8]
    t_in, kern, t_out, _ = _case(g, 11)
    got = temporal.prespike(cuda(t_in), cuda(kern), cuda(t_out), stride, pad)
    np.testing.assert_allclose(host(got), tr.prespike(t_in, kern, t_out, stride, pad, time), rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("geo", [((2, 2), None, (0, 0, 0, 0)), ((3, 3), (2, 2), (1, 1, 1, 1)), ((2, 3), (1, 2), (0, 1, 1, 0))])
def test_pool_forward_backward(geo):
    k2, s2, p4 = geo
    rng = np.random.default_rng(3)
    t = rng.integers(0, 9, size=(3, 4, 10, 11)).astype(np.float32)  # many ties
    out = temporal.pool_forward(cuda(t), k2, 9, s2, p4)
    want = tr.pool_forward(t, k2, s2, p4, 9)
    assert np.array_equal(host(out), want)
    go = rng.normal(size=want.shape).astype(np.float32)
    gi = temporal.pool_backward(cuda(t), cuda(go), k2, s2, p4)
    np.testing.assert_allclose(host(gi), tr.pool_backward(t, go, k2, s2, p4), rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
@pytest.mark.parametrize("g", [GEOS[0], GEOS[1], GEOS[2], GEOS[4]])
def test_forward_times_match_oracle(g, precision):
    b, c, h, w, z, k, stride, pad, time = g
    rng = np.random.default_rng(b + c)
    t_in = rng.integers(0, time + 1, size=(b, c, h, w)).astype(np.float32)
    kern = rng.uniform(0.0, 0.1, size=(z, c, k, k)).astype(np.float32)
    thr = 0.02 * c * k * k
    got = temporal.conv_forward(cuda(t_in), cuda(kern), thr, time, stride, pad, precision)
    want = tr.conv_forward(t_in, kern, thr, time, stride, pad)
    assert np.array_equal(host(got), want)
    assert 0 < (want < time).mean() < 1


@pytest.mark.parametrize("g", [
    (3, 4, 9, 8, 5, 3, (1, 1), (1, 1, 1, 1), 16),
    (2, 3, 11, 10, 6, 5, (2, 1), (2, 0, 1, 2), 20),
    (2, 8, 12, 12, 40, 3, (1, 1), (1, 1, 1, 1), 64),  # 2 pixels per tile, 2 warps per pixel
    (2, 2, 6, 7, 12, 3, (1, 1), (1, 1, 1, 1), 100),  # 1 pixel per tile, 4 warps per pixel
    (3, 2, 10, 10, 8, 3, (1, 1), (1, 1, 1, 1), 2),
    (2, 64, 7, 7, 10, 1, (1, 1), (0, 0, 0, 0), 64),
])
@pytest.mark.parametrize("precision", ["bf16x3", "bf16x2"])
def test_fused_times_equal_potentials_then_gather(g, precision):
    """The fused first-spike kernel equals the tensor-core potentials of
    every step followed by gather, bit for bit."""
    b, c, h, w, z, k, stride, pad, time = g
    rng = np.random.default_rng(b * 5 + c + time)
    t_in = rng.integers(0, time + 1, size=(b, c, h, w)).astype(np.float32)
    kern = rng.uniform(0.0, 0.2, size=(z, c, k, k)).astype(np.float32)
    thr = 0.05 * c * k * k
    ti = cuda(t_in)
    got = temporal.conv_forward(ti, cuda(kern), thr, time, stride, pad, precision)
    spikes = spyker.scatter(ti.reshape(b, -1), time).view(b, time, c, h, w)
    want = spyker.gather(spyker.conv(spikes, cuda(kern), stride, pad, precision), thr, dtype="f32")
    assert torch.equal(got, want)
    assert 0 < float((want < time).float().mean()) < 1
    assert spyker._lib.lib.spk_device_status(1) == 0


@pytest.mark.parametrize("seed", [0, 1])
def test_fc_gradients_are_reference_fcbackward(ref, seed):
    """The GPU fc backward against the reference's own (cpu/backprop.cpp:105-160)."""
    rng = np.random.default_rng(seed)
    b, ni, no, time = 4, 300, 10, 64
    t_in = rng.integers(0, time + 1, size=(b, ni)).astype(np.float32)
    t_out = rng.integers(0, time + 1, size=(b, no)).astype(np.float32)
    grad = (rng.normal(size=(b, no)) / time).astype(np.float32)
    w = rng.uniform(0.0, 0.1, size=(no, ni)).astype(np.float32)
    gi, gk = temporal.conv_backward(cuda(t_in).view(b, ni, 1, 1), cuda(w).view(no, ni, 1, 1),
                                    cuda(t_out).view(b, no, 1, 1), -cuda(grad).view(b, no, 1, 1))
    _, nxt, _ = ref.fcbackward(w, t_in, t_out, grad, (0.0, 0.0, 0.0, 0.0))
    np.testing.assert_allclose(host(gi).reshape(b, ni), -nxt, rtol=1e-6, atol=1e-7)
    k, _, _ = ref.fcbackward(w, t_in[:1], t_out[:1], grad[:1], (0.0, 1.0, 0.0, 0.0))
    _, gk1 = temporal.conv_backward(cuda(t_in[:1]).view(1, ni, 1, 1), cuda(w).view(no, ni, 1, 1),
                                    cuda(t_out[:1]).view(1, no, 1, 1), -cuda(grad[:1]).view(1, no, 1, 1))
    np.testing.assert_allclose(host(gk1).reshape(no, ni), w - k, rtol=0, atol=2e-7)


def _net_and_data(b=6, seed=4):
    imgs, labels = synth.labelled_strokes(b, seed=seed)
    net = temporal.TemporalNet(time=64, seed=seed)
    x = cuda(imgs.astype(np.float32) / 255)[:, None]
    return net, x, torch.from_numpy(labels).to(DEV)


def _layers(net, x):
    """Forward with the intermediate times kept (and their gradients)."""
    T, th, p = net.time, net.thresholds, net.precision
    w1, w2, w3 = net.weights
    t0 = net.input_times(x)
    t1 = temporal.first_spike_conv(t0, w1, th[0], T, 1, 2, p)
    p1 = temporal.first_spike_pool(t1, 2, T)
    t2 = temporal.first_spike_conv(p1, w2, th[1], T, 1, 1, p)
    p2 = temporal.first_spike_pool(t2, 2, T)
    f = p2.reshape(p2.shape[0], -1)
    t3 = temporal.first_spike_fc(f, w3, th[2], T, p)
    for t in (t1, p1, t2, p2, t3):
        t.retain_grad()
    return t0, t1, p1, t2, p2, f, t3


def test_network_gradients_match_oracle_chain():
    net, x, y = _net_and_data()
    t0, t1, p1, t2, p2, f, t3 = _layers(net, x)
    loss = net.loss(t3, y)
    loss.backward()
    w1, w2, w3 = [host(w) for w in net.weights]
    T = net.time
    g3 = -tr.target_rule(host(t3), host(y), T, net.gamma)
    np.testing.assert_allclose(host(t3.grad), g3, rtol=1e-6, atol=1e-7)
    gf, gk3 = tr.conv_backward(host(f)[:, :, None, None], w3[:, :, None, None], host(t3)[:, :, None, None],
                               g3[:, :, None, None])
    np.testing.assert_allclose(host(net.weights[2].grad), gk3[:, :, 0, 0], rtol=1e-5, atol=1e-6)
    gp2 = gf.reshape(host(p2).shape)
    np.testing.assert_allclose(host(p2.grad), gp2, rtol=1e-5, atol=1e-6)
    gt2 = tr.pool_backward(host(t2), host(p2.grad), (2, 2))
    np.testing.assert_allclose(host(t2.grad), gt2, rtol=1e-5, atol=1e-6)
    gp1, gk2 = tr.conv_backward(host(p1), w2, host(t2), host(t2.grad), (1, 1), (1, 1, 1, 1))
    np.testing.assert_allclose(host(net.weights[1].grad), gk2, rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(host(p1.grad), gp1, rtol=1e-5, atol=1e-5)
    gt1 = tr.pool_backward(host(t1), host(p1.grad), (2, 2))
    _, gk1 = tr.conv_backward(host(t0), w1, host(t1), gt1, (1, 1), (2, 2, 2, 2))
    np.testing.assert_allclose(host(net.weights[0].grad), gk1, rtol=1e-5, atol=1e-5)
    assert all(float(w.grad.abs().sum()) > 0 for w in net.weights)


def test_finite_differences_of_potential_loss_all_layers():
    """dL/dW of every layer is the derivative of its potential-level loss
    sum(-dL/dt_out * V(t_out - 1)) (times held fixed), by central differences
    with h = 1e-3 on FP64 potentials recomputed on the GPU."""
    net, x, y = _net_and_data(b=4, seed=9)
    t0, t1, p1, t2, p2, f, t3 = _layers(net, x)
    net.loss(t3, y).backward()
    b = t3.shape[0]
    layers = [(t0, net.weights[0], t1, t1.grad, (1, 1), (2, 2, 2, 2)),
              (p1, net.weights[1], t2, t2.grad, (1, 1), (1, 1, 1, 1)),
              (f.reshape(b, -1, 1, 1), net.weights[2], t3.reshape(b, -1, 1, 1), t3.grad.reshape(b, -1, 1, 1), (1, 1),
               (0, 0, 0, 0))]
    rng = np.random.default_rng(0)
    h = 1e-3
    for t_in, w, t_out, go, stride, pad in layers:
        w4 = w.detach().reshape(w.shape[0], -1, *(w.shape[2:] if w.dim() == 4 else (1, 1)))
        grad = w.grad.reshape(w4.shape)

        def loss(wx):
            return float((-go.double() * temporal.prespike(t_in.detach(), wx, t_out.detach(), stride, pad)).sum())

        flat = np.flatnonzero(host(grad).reshape(-1) != 0)
        picks = rng.choice(flat, size=min(6, flat.size), replace=False).tolist() + [0]
        for i in picks:
            wp, wm = w4.clone(), w4.clone()
            wp.view(-1)[i] += h
            wm.view(-1)[i] -= h
            # the loss is linear in W: divide by the perturbation actually stored in F32
            fd = (loss(wp) - loss(wm)) / (float(wp.view(-1)[i]) - float(wm.view(-1)[i]))
            assert abs(fd - float(grad.view(-1)[i])) <= 1e-6 * max(1.0, abs(fd)), (i, fd, float(grad.view(-1)[i]))


def test_training_steps_run_and_change_weights():
    net, x, y = _net_and_data(b=32, seed=5)
    w0 = [w.detach().clone() for w in net.weights]
    losses = [float(net.step(x, y, lrate=0.05)[0]) for _ in range(3)]
    assert all(np.isfinite(losses))
    assert all(not torch.equal(a, b.detach()) for a, b in zip(w0, net.weights))
    assert spyker._lib.lib.spk_device_status(1) == 0
