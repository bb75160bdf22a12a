"""The temporal-backprop rule of the first-spike layers, on CPU.

The NumPy restatement (oracle/temporal.py) is pinned to the reference's own
fc backward (src/spyker/cpu/backprop.cpp:105-160, compiled in oracle/_ref):
with lrate = lambda = 0 its `next` is minus our input gradient, and with
lrate = 1 on one sample its weight change is minus our kernel gradient.
Its kernel gradient is also the exact derivative of the potential-level
loss, checked by central finite differences (h = 1e-3)."""

import numpy as np
import pytest

from oracle import temporal as tr


def _fc_case(seed, b=3, ni=40, no=6, time=20):
    rng = np.random.default_rng(seed)
    t_in = rng.integers(0, time + 1, size=(b, ni)).astype(np.float32)
    t_out = rng.integers(0, time + 1, size=(b, no)).astype(np.float32)
    grad = rng.normal(size=(b, no)).astype(np.float32) / time  # (desired - t) / T
    w = rng.uniform(0.0, 0.1, size=(no, ni)).astype(np.float32)
    return t_in, t_out, grad, w


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_fc_input_gradient_is_reference_next(ref, seed):
    t_in, t_out, grad, w = _fc_case(seed)
    _, nxt, _ = ref.fcbackward(w, t_in, t_out, grad, (0.0, 0.0, 0.0, 0.0))
    gi, _ = tr.conv_backward(t_in[:, :, None, None], w[:, :, None, None], t_out[:, :, None, None],
                             -grad.astype(np.float64)[:, :, None, None])
    np.testing.assert_allclose(gi[:, :, 0, 0], -nxt, rtol=1e-6, atol=1e-7)
    assert np.abs(nxt).sum() > 0


@pytest.mark.parametrize("seed", [3, 4])
def test_fc_kernel_gradient_is_reference_update(ref, seed):
    t_in, t_out, grad, w = _fc_case(seed, b=1)
    k, _, _ = ref.fcbackward(w, t_in, t_out, grad, (0.0, 1.0, 0.0, 0.0))
    _, gk = tr.conv_backward(t_in[:, :, None, None], w[:, :, None, None], t_out[:, :, None, None],
                             -grad.astype(np.float64)[:, :, None, None])
    # reference: kernel -= lrate * select, select = dL/dW
    np.testing.assert_allclose(w - k, gk[:, :, 0, 0], rtol=0, atol=2e-7)
    assert np.abs(gk).sum() > 0


def test_target_rule_matches_reference(ref):
    rng = np.random.default_rng(7)
    t = rng.integers(0, 33, size=(6, 10)).astype(np.float32)
    t[2] = 32  # a silent sample
    target = rng.integers(0, 10, size=6).astype(np.int64)
    want = ref.backward(t, target, 32, 3.0)
    np.testing.assert_allclose(tr.target_rule(t, target, 32, 3.0), want, rtol=1e-6, atol=1e-7)


@pytest.mark.parametrize("geo", [((1, 1), (1, 1, 1, 1), 3), ((2, 1), (0, 2, 1, 0), 3), ((1, 1), (2, 2, 2, 2), 5)])
def test_kernel_gradient_is_derivative_of_potential_loss(geo):
    stride, pad, k = geo
    rng = np.random.default_rng(k + stride[0])
    time = 12
    t_in = rng.integers(0, time + 1, size=(2, 3, 7, 6)).astype(np.float64)
    w = rng.uniform(0.0, 0.3, size=(4, 3, k, k))
    t_out = tr.conv_forward(t_in, w, 1.2, time, stride, pad)
    go = rng.normal(size=t_out.shape)
    _, gk = tr.conv_backward(t_in, w, t_out, go, stride, pad)

    def loss(wx):
        return float(np.sum(-go * tr.prespike(t_in, wx, t_out, stride, pad, time)))

    h = 1e-3
    for idx in [(0, 0, 0, 0), (1, 2, k - 1, 0), (3, 1, k // 2, k - 1), (2, 0, k - 1, k - 1)]:
        wp, wm = w.copy(), w.copy()
        wp[idx] += h
        wm[idx] -= h
        fd = (loss(wp) - loss(wm)) / (2 * h)
        assert abs(fd - gk[idx]) <= 1e-9 * max(1.0, abs(fd)), (idx, fd, gk[idx])


def test_pool_gradient_goes_to_first_earliest():
    t = np.array([[[[3, 1, 1, 5], [1, 4, 2, 2], [7, 7, 9, 9], [7, 7, 9, 9]]]], dtype=np.float64)
    p = tr.pool_forward(t, (2, 2), None, (0, 0, 0, 0), 10)
    assert np.array_equal(p[0, 0], [[1, 1], [7, 9]])
    g = tr.pool_backward(t, np.array([[[[1.0, 2.0], [3.0, 4.0]]]]), (2, 2))
    want = np.zeros((4, 4))
    want[0, 1], want[0, 2], want[2, 0], want[2, 2] = 1, 2, 3, 4
    assert np.array_equal(g[0, 0], want)
