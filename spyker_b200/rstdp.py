"""Reward-modulated STDP (R-STDP): the three-layer network of the reference's
Mozafari example (examples/mozafari_mnist_original.py:60-138) on the GPU.

Layers 1 and 2 learn with STDP (convwta + `Conv.stdp`), layer 3 with R-STDP:
its potentials are read only at the last step (`infinite`), one winner per
image (`convwta(x, 0, 1)`) gives the label `z // (C / 10)`, and the winner's
STDP config is 0 (reward) when the label is right, 1 (punish) when it is
wrong.  The reference assigns that config in a Python loop over the winner
lists; here it is one tensor operation on the device records, so a training
step makes no host round trip.
"""

from __future__ import annotations

import numpy
import torch

from . import module as M


class MozafariNetwork:
    """DoG (6 filters, 7x7) -> threshold 0.02 -> rank code T=15 -> conv1 30x5x5
    (th 15) -> pool 2 -> conv2 250x3x3 (th 5) -> pool 3 -> conv3 200x5x5
    (infinite readout, 10 classes of 20 maps)."""

    def __init__(self, device=None, precision: str = "bf16x3", seed: int = 0):
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        M.random_seed(seed)
        F = M.DoGFilter
        filters = [F(3 / 9, 6 / 9), F(6 / 9, 3 / 9), F(7 / 9, 14 / 9), F(14 / 9, 7 / 9), F(13 / 9, 26 / 9),
                   F(26 / 9, 13 / 9)]
        self.filters = M.DoG(3, filters, pad=3, device=dev)
        self.conv1 = M.Conv(6, 30, 5, pad=2, mean=0.8, std=0.05, device=dev)
        self.conv2 = M.Conv(30, 250, 3, pad=1, mean=0.8, std=0.05, device=dev)
        self.conv3 = M.Conv(250, 200, 5, pad=2, mean=0.8, std=0.05, device=dev)
        for c in (self.conv1, self.conv2, self.conv3):
            c.precision = precision
        self.conv1.stdpconfig = [M.STDPConfig(0.004, -0.003)]
        self.conv2.stdpconfig = [M.STDPConfig(0.004, -0.003)]
        reward = M.STDPConfig(0.004, -0.003, False, 0.2, 0.8)
        punish = M.STDPConfig(-0.004, 0.0005, False, 0.2, 0.8)
        self.conv3.stdpconfig = [reward, punish]
        self.thresh1, self.thresh2 = 15.0, 5.0

    def transform(self, images):
        return M.code(M.threshold(self.filters(images), 0.02), 15)

    def _features(self, x):
        x = M.pool(M.fire(self.conv1(x), self.thresh1), 2)
        return M.pool(M.fire(self.conv2(x), self.thresh2), 3)

    def train_layer1(self, x):
        out = M.inhibit(M.threshold(self.conv1(x), self.thresh1))
        self.conv1.stdp(x, M.convwta(out, 3, 5), M.fire(out))

    def train_layer2(self, x):
        x = M.pool(M.fire(self.conv1(x), self.thresh1), 2)
        out = M.inhibit(M.threshold(self.conv2(x), self.thresh2))
        self.conv2.stdp(x, M.convwta(out, 1, 8), M.fire(out))

    def _readout(self, x):
        out = M.infinite(self.conv3(x))
        wins = M.convwta(out, 0, 1)
        per = out.shape[2] // 10
        labels = torch.where(wins.counts == 1, wins.records[:, 0, 2] // per, torch.full_like(wins.counts, -1))
        return out, wins, labels.long()

    def train_layer3(self, x, target: torch.Tensor) -> torch.Tensor:
        """One R-STDP step; returns the labels (-1: no winner)."""
        x = self._features(x)
        out, wins, labels = self._readout(x)
        # config 0 (reward) when right, 1 (punish) when wrong, for samples
        # with a winner (records of samples without one are not read)
        wins.records[:, 0, 0] = (labels != target.to(labels.device)).to(torch.int32)
        self.conv3.stdp(x, wins, M.fire(out))
        return labels

    def __call__(self, x) -> torch.Tensor:
        return self._readout(self._features(x))[2]


def accuracy(labels: torch.Tensor, target: torch.Tensor) -> numpy.ndarray:
    """(correct, wrong, silent, total) as the example's `perform`."""
    silent = int((labels == -1).sum())
    right = int((labels == target).sum())
    return numpy.array([right, len(target) - right - silent, silent, len(target)])
