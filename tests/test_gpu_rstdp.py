"""R-STDP (the reference's Mozafari example, examples/mozafari_mnist_original.py)
on the GPU: one layer-3 reward/punish step against the same step composed
from the oracle's ops (FP64 convolutions, the reference's STDP rule with two
configs selected per winner)."""

import numpy as np
import pytest
import torch

from spyker_b200 import rstdp, synth

pytestmark = pytest.mark.gpu
DEV = "cuda"


def host(t):
    return t.detach().cpu().numpy()


def test_layer3_rstdp_step_matches_oracle(port):
    imgs, labels = synth.labelled_strokes(4, seed=8)
    net = rstdp.MozafariNetwork(device=DEV, seed=3)
    x = net.transform(torch.from_numpy(imgs).to(DEV).float().div_(255)[:, None])
    target = torch.from_numpy(labels).to(DEV)
    codes = host(x)
    w1, w2, w3 = host(net.conv1.kernel), host(net.conv2.kernel), host(net.conv3.kernel)
    got_labels = host(net.train_layer3(x, target))

    a = port.pool(port.fire(port.conv(codes, w1, (1, 1), (2, 2, 2, 2)), 15.0), (2, 2))
    b = port.pool(port.fire(port.conv(a, w2, (1, 1), (1, 1, 1, 1)), 5.0), (3, 3))
    out = port.infinite(port.conv(b, w3, (1, 1), (2, 2, 2, 2)))
    win, cnt = port.convwta(out, (0, 0), 1)
    want_labels = np.where(cnt == 1, win[:, 0, 2] // 20, -1)
    assert np.array_equal(got_labels, want_labels)
    win[:, 0, 0] = (want_labels != labels).astype(np.int64)
    cfg = [(0.004, -0.003, 0.0, 0.2, 0.8), (-0.004, 0.0005, 0.0, 0.2, 0.8)]
    want = port.convstdp(b, w3, port.fire(out), cfg, win, cnt, (1, 1), (2, 2, 2, 2))
    assert np.array_equal(host(net.conv3.kernel), want)
    assert not np.array_equal(want, w3)


def test_training_phases_run():
    imgs, labels = synth.labelled_strokes(16, seed=9)
    net = rstdp.MozafariNetwork(device=DEV, seed=4)
    x = net.transform(torch.from_numpy(imgs).to(DEV).float().div_(255)[:, None])
    k1, k2 = net.conv1.kernel.clone(), net.conv2.kernel.clone()
    net.train_layer1(x)
    net.train_layer2(x)
    assert not torch.equal(k1, net.conv1.kernel) and not torch.equal(k2, net.conv2.kernel)
    pred = net(x)
    assert pred.shape == (16,) and int(pred.min()) >= -1 and int(pred.max()) <= 9
    perf = rstdp.accuracy(pred.cpu(), torch.from_numpy(labels))
    assert perf.sum() - perf[3] == perf[3]
