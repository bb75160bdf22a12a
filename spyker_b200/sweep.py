"""Many independent STDP networks trained in one step (a hyperparameter sweep).

Every network has the 2-layer architecture of the Kheradpisheh example
(DoG -> rank code -> conv1 30x5x5 -> threshold -> inhibit -> WTA -> fire ->
STDP -> pool 2 -> conv2 100x5x5 -> ... -> STDP -> global pool), its own
weights, threshold and learning rates, and its own stream of images of
uneven sizes.  One step trains every network on its whole stream:

* images are grouped by size; per size and layer ONE fused tcgen05 launch
  (``spk_conv_fire_wta_nets``) runs all networks, each tile reading its
  network's weight image and threshold (``path="dense"``); or, with
  ``path="search"``, each network's share of the group takes the
  single-network fused layer (``spk_conv_fire_wta``), whose first-crossing
  search on u8 tensor cores evaluates about log2(T) + 2 of a pixel's T
  potential rows where the weights are non-negative (more launches, much
  less work per image);
* per layer ONE ordered STDP scan (``spk_stdp_scan_nets``) updates all
  networks, each walking its winners in the order of its own image stream
  (the reference's per-sample sequential rule, cpu/stdp.cpp:99-169), across
  the size groups;
* the whole step can be captured once as a CUDA graph and replayed;
* the launch schedule of each (size, layer) is chosen by
  :mod:`spyker_b200.autotune`.

A network's result equals training that network alone on its images, in
stream order, with the batch semantics of the single-network step (forward of
the batch with the weights at its start, then the sequential updates).
"""

from __future__ import annotations

import numpy
import torch

from . import _lib
from . import autotune
from . import module as M
from . import synth
from ._lib import call, i64, ptr, stream

T = 15
C1, C2 = 30, 100
COUNT1, COUNT2 = 5, 8
RADIUS1, RADIUS2 = 3, 1


def _pp(t: int) -> int:
    tp = 1
    while tp < t:
        tp <<= 1
    return 128 // tp


class NetworkSpec:
    """Hyperparameters of network n (numpy default_rng(seed + n))."""

    def __init__(self, n: int, seed: int, images: int, sizes):
        rng = numpy.random.default_rng(seed + n)
        self.theta = float(rng.uniform(8.0, 20.0))
        self.pos = float(rng.uniform(0.001, 0.01))
        self.neg = -0.75 * self.pos
        self.w1 = synth.conv_weights(C1, 2, 5, seed=1000 + seed + n)
        self.w2 = synth.conv_weights(C2, C1, 5, seed=2000 + seed + n)
        self.sizes = rng.choice(numpy.asarray(sizes), size=images)
        self.image_seed = 3000 + seed + n

    @property
    def theta2(self) -> float:
        # the second layer's threshold keeps the example's 10 / 15 ratio
        return self.theta * (10.0 / 15.0)


class _Group:
    """The images of one size, network by network (each network's share padded
    with blank images to a whole number of tiles at both layers)."""

    def __init__(self, size, per_net, dev):
        self.size = size
        self.per_net = per_net  # list of (network, [stream positions], images [k, S, S] u8)
        counts = []
        for _, pos, _ in per_net:
            k = len(pos)
            # layer 1: k * S^2 and layer 2: k * (S/2)^2 pixels per network must
            # be multiples of the tile's 8 pixels
            while (k * size * size) % _pp(T) or (k * (size // 2) ** 2) % _pp(T):
                k += 1
            counts.append(k)
        self.counts = counts
        self.offsets = numpy.concatenate([[0], numpy.cumsum(counts)]).astype(numpy.int64)
        self.batch = int(self.offsets[-1])
        imgs = numpy.zeros((self.batch, size, size), dtype=numpy.uint8)
        snet = numpy.zeros(self.batch, dtype=numpy.int32)
        for (n, pos, x), o, k in zip(per_net, self.offsets[:-1], counts):
            imgs[o:o + len(pos)] = x
            snet[o:o + k] = n
        self.host = torch.from_numpy(imgs).pin_memory()
        self.images = self.host.to(dev).float().div_(255.0)[:, None]
        self.sample_net = torch.from_numpy(snet).to(dev)


class Sweep:
    """``nets`` networks, each with ``images`` stroke images of sides drawn
    uniformly from ``sizes``."""

    def __init__(self, nets: int = 32, images: int = 512, sizes=(20, 28, 40, 64), seed: int = 0, device=None,
                 precision: str = "bf16x3", tune: bool = True, path: str = "dense"):
        if path not in ("dense", "search"):
            raise ValueError("path must be 'dense' or 'search'")
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.dev, self.precision, self.nets, self.path = dev, precision, nets, path
        self.specs = [NetworkSpec(n, seed, images, sizes) for n in range(nets)]
        self.dog = M.DoG(3, [M.DoGFilter(1, 2), M.DoGFilter(2, 1)], pad=3, device=dev)
        self.w1 = torch.from_numpy(numpy.stack([s.w1 for s in self.specs])).to(dev)
        self.w2 = torch.from_numpy(numpy.stack([s.w2 for s in self.specs])).to(dev)
        self.thr1 = torch.tensor([s.theta for s in self.specs], dtype=torch.float32, device=dev)
        self.thr2 = torch.tensor([s.theta2 for s in self.specs], dtype=torch.float32, device=dev)
        # STDP configs per network (positive, negative, stabilize, lower, upper)
        self.cfg = torch.tensor([[s.pos, s.neg, 1.0, 0.0, 1.0] for s in self.specs], dtype=torch.float64, device=dev)
        # groups by size; global sample index = group offset + index in group
        self.groups = []
        for size in sorted(set(int(v) for s in self.specs for v in s.sizes)):
            per_net = []
            for n, s in enumerate(self.specs):
                pos = numpy.flatnonzero(s.sizes == size)
                x = synth.strokes(len(pos), seed=s.image_seed * 7 + size, size=size) if len(pos) else \
                    numpy.zeros((0, size, size), numpy.uint8)
                per_net.append((n, pos, x))
            self.groups.append(_Group(size, per_net, dev))
        self.goff = numpy.concatenate([[0], numpy.cumsum([g.batch for g in self.groups])]).astype(numpy.int64)
        self.total = int(self.goff[-1])
        # each network's samples in its stream order (global indexes)
        order, noff = [], [0]
        for n, s in enumerate(self.specs):
            entries = []
            for gi, g in enumerate(self.groups):
                _, pos, _ = g.per_net[n]
                base = int(self.goff[gi] + g.offsets[n])
                entries += [(int(p), base + j) for j, p in enumerate(pos)]
            entries.sort()
            order += [e[1] for e in entries]
            noff.append(len(order))
        self.order = torch.tensor(order, dtype=torch.int32, device=dev)
        self.noff = torch.tensor(noff, dtype=torch.int64, device=dev)
        self.images_per_step = len(order)
        # winner records, (pre, post) times of both layers over all samples
        b = self.total
        self.rec = [torch.zeros((b, c, 5), dtype=torch.int32, device=dev) for c in (COUNT1, COUNT2)]
        self.cnt = [torch.zeros((b,), dtype=torch.int32, device=dev) for _ in range(2)]
        self.pre = [torch.zeros((b, COUNT1, 2 * 25), dtype=torch.int16, device=dev),
                    torch.zeros((b, COUNT2, C1 * 25), dtype=torch.int16, device=dev)]
        self.post = [torch.zeros((b, c), dtype=torch.int16, device=dev) for c in (COUNT1, COUNT2)]
        self.schedules = {}
        if tune and path == "dense":  # the schedules are the multi-network kernel's
            self.tune()
        self.graph = None

    # -- one layer of one size group, all networks -----------------------
    def _layer(self, gi, layer, x, pool, sched=None):
        if self.path == "search":
            return self._layer_search(gi, layer, x, pool)
        g = self.groups[gi]
        w, thr, cout, count, radius = ((self.w1, self.thr1, C1, COUNT1, RADIUS1) if layer == 0
                                       else (self.w2, self.thr2, C2, COUNT2, RADIUS2))
        s = list(x.shape)
        b, cin, h, wd = s[0], s[2], s[3], s[4]
        nb = _lib.lib.spk_conv_fire_wta_nets_workspace(self.nets, b, T, cin, h, wd, cout, 5, 5, 1, 1, i64(2, 2, 2, 2),
                                                       M._PRECISION[self.precision])
        if nb == 0:
            raise RuntimeError("layer does not fit the fused multi-network kernel")
        ws, wsb = M._workspace(nb, x.device)
        spikes = torch.empty((b, T, cout, h, wd), dtype=torch.uint8, device=x.device)
        ph, pw = (h, wd) if pool == "global" else (pool, pool)
        pooled = torch.empty((b, T, cout, h // ph, wd // pw), dtype=torch.uint8, device=x.device)
        o = int(self.goff[gi])
        rec, cnt = self.rec[layer][o:o + b], self.cnt[layer][o:o + b]
        st = sched if sched is not None else self.schedules.get((gi, layer), (0, 0, 0))
        call("spk_set_conv_schedule", *st)
        try:
            call("spk_conv_fire_wta_nets", ptr(x), 4, ptr(w), self.nets, i64(*g.offsets), ptr(g.sample_net), ptr(thr),
                 b, T, cin, h, wd, cout, 5, 5, 1, 1, i64(2, 2, 2, 2), 0.0, 0.0, 0.0, radius, radius, count, 0.0,
                 ptr(spikes), ptr(rec), ptr(cnt), ph, pw, ptr(pooled), M._PRECISION[self.precision], ptr(ws), wsb,
                 stream())
        finally:
            call("spk_set_conv_schedule", 0, 0, 0)
        return spikes, pooled

    def _layer_search(self, gi, layer, x, pool):
        """The group's layer as one single-network fused call per network, on
        that network's contiguous share of the group (its weights and
        threshold); records and counts land in the same slots as on the
        multi-network kernel."""
        g = self.groups[gi]
        w, cout, count, radius = ((self.w1, C1, COUNT1, RADIUS1) if layer == 0 else (self.w2, C2, COUNT2, RADIUS2))
        b, _, cin, h, wd = x.shape
        ph, pw = (h, wd) if pool == "global" else (pool, pool)
        spikes = torch.empty((b, T, cout, h, wd), dtype=torch.uint8, device=x.device)
        pooled = torch.empty((b, T, cout, h // ph, wd // pw), dtype=torch.uint8, device=x.device)
        o = int(self.goff[gi])
        rec, cnt = self.rec[layer][o:o + b], self.cnt[layer][o:o + b]
        rec.zero_()
        cnt.zero_()
        prec = M._PRECISION[self.precision]
        sizes = [int(g.offsets[n + 1] - g.offsets[n]) for n in range(self.nets)]
        nb = _lib.lib.spk_conv_fire_wta_workspace(max(sizes), T, cin, h, wd, cout, 5, 5, 1, 1, i64(2, 2, 2, 2), prec)
        if nb == 0:
            raise RuntimeError("layer does not fit the fused single-network kernel")
        ws, wsb = M._workspace(nb, x.device)
        for n, k in enumerate(sizes):
            if k == 0:
                continue
            lo = int(g.offsets[n])
            sl = slice(lo, lo + k)
            thr = self.specs[n].theta if layer == 0 else self.specs[n].theta2
            call("spk_conv_fire_wta", ptr(x[sl]), 4, ptr(w[n]), k, T, cin, h, wd, cout, 5, 5, 1, 1, i64(2, 2, 2, 2),
                 float(thr), 0.0, 0.0, 0.0, radius, radius, count, 0.0, ptr(spikes[sl]), ptr(rec[sl]), ptr(cnt[sl]),
                 ph, pw, ptr(pooled[sl]), prec, ptr(ws), wsb, stream())
        return spikes, pooled

    def _prepost(self, gi, layer, x, spikes):
        b, _, cin, h, wd = x.shape
        cout, count = (C1, COUNT1) if layer == 0 else (C2, COUNT2)
        o = int(self.goff[gi])
        nb = _lib.lib.spk_rank_convstdp_prepost_workspace(b, cin, h, wd)
        ws, wsb = M._workspace(nb, x.device)
        call("spk_rank_convstdp_prepost", ptr(x), 4, b, T, cin, h, wd, cout, 5, 5, ptr(spikes), h, wd,
             ptr(self.rec[layer][o:o + b]), ptr(self.cnt[layer][o:o + b]), count, 1, 1, i64(2, 2, 2, 2),
             ptr(self.pre[layer][o:o + b]), ptr(self.post[layer][o:o + b]), ptr(ws), wsb, stream())

    def _scan(self, layer):
        w, count, cin = (self.w1, COUNT1, 2) if layer == 0 else (self.w2, COUNT2, C1)
        k = cin * 25
        call("spk_stdp_scan_nets", ptr(w), self.nets, w.shape[1], k, self.total, count, 2, ptr(self.rec[layer]),
             ptr(self.cnt[layer]), ptr(self.pre[layer]), count * k, k, ptr(self.post[layer]), ptr(self.noff),
             ptr(self.order), ptr(self.cfg), 1, 0, stream())

    def _codes(self, gi):
        return M.code(self.dog(self.groups[gi].images), T)

    def step(self):
        """One training step of every network on its stream; returns the
        global-pool features of each size group."""
        codes = [self._codes(gi) for gi in range(len(self.groups))]
        pooled1 = []
        for gi, c in enumerate(codes):
            spk, pooled = self._layer(gi, 0, c, 2)
            self._prepost(gi, 0, c, spk)
            pooled1.append(pooled)
        self._scan(0)
        feats = []
        for gi, q in enumerate(pooled1):
            spk, f = self._layer(gi, 1, q, "global")
            self._prepost(gi, 1, q, spk)
            feats.append(f)
        self._scan(1)
        self.last_features = feats
        return feats

    # -- CUDA graph ------------------------------------------------------
    def capture(self):
        """Capture one step as a CUDA graph (replayed by :meth:`replay`)."""
        s = torch.cuda.Stream(self.dev)
        s.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(s):
            self.step()  # warm-up (allocator pools, kernel attributes)
        torch.cuda.current_stream(self.dev).wait_stream(s)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.graph_features = self.step()
        return self.graph

    def replay(self):
        self.graph.replay()
        return self.graph_features

    # -- autotuning ------------------------------------------------------
    def tune(self, reps: int = 3):
        """Pick the schedule of every (size group, layer) launch by timing the
        candidates (the weights are restored afterwards)."""
        w1, w2 = self.w1.clone(), self.w2.clone()
        for gi in range(len(self.groups)):
            codes = self._codes(gi)
            best = autotune.best_schedule(lambda st: self._layer(gi, 0, codes, 2, st), reps=reps)
            self.schedules[(gi, 0)] = best
            _, pooled = self._layer(gi, 0, codes, 2, best)
            self.schedules[(gi, 1)] = autotune.best_schedule(lambda st: self._layer(gi, 1, pooled, "global", st),
                                                             reps=reps)
        self.w1.copy_(w1)
        self.w2.copy_(w2)
        return self.schedules
