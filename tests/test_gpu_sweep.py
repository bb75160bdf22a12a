"""Several networks in one launch: the multi-network fused layer and STDP
scan against the single-network calls, and the sweep step (size groups,
per-network stream order, CUDA graph replay, autotuned schedules) against
training each network alone."""

import numpy as np
import pytest
import torch

import spyker_b200 as spyker
from spyker_b200 import _lib, sweep, synth
from spyker_b200._lib import i64

pytestmark = pytest.mark.gpu
DEV = "cuda"


def host(t):
    return t.cpu().numpy()


def _codes(n, size, seed):
    imgs = torch.from_numpy(synth.strokes(n, seed=seed, size=size)).to(DEV).float().div_(255)[:, None]
    dog = spyker.DoG(3, [spyker.DoGFilter(1, 2), spyker.DoGFilter(2, 1)], pad=3, device=DEV)
    return spyker.code(dog(imgs), 15)


def _nets_layer(x, kernels, offsets, thr, count, radius, pool, prec="bf16x3"):
    b, t, cin, h, w = x.shape
    n, cout = kernels.shape[0], kernels.shape[1]
    snet = torch.from_numpy(np.repeat(np.arange(n), np.diff(offsets)).astype(np.int32)).to(DEV)
    th = torch.tensor(thr, dtype=torch.float32, device=DEV)
    nb = _lib.lib.spk_conv_fire_wta_nets_workspace(n, b, t, cin, h, w, cout, 5, 5, 1, 1, i64(2, 2, 2, 2), 2 if prec == "bf16x3" else 1)
    ws = torch.empty(nb, dtype=torch.uint8, device=DEV)
    spikes = torch.empty((b, t, cout, h, w), dtype=torch.uint8, device=DEV)
    pooled = torch.empty((b, t, cout, h // pool, w // pool), dtype=torch.uint8, device=DEV)
    rec = torch.zeros((b, count, 5), dtype=torch.int32, device=DEV)
    cnt = torch.zeros((b,), dtype=torch.int32, device=DEV)
    _lib.call("spk_conv_fire_wta_nets", x.data_ptr(), 4, kernels.data_ptr(), n, i64(*offsets), snet.data_ptr(),
              th.data_ptr(), b, t, cin, h, w, cout, 5, 5, 1, 1, i64(2, 2, 2, 2), 0.0, 0.0, 0.0, radius, radius, count,
              0.0, spikes.data_ptr(), rec.data_ptr(), cnt.data_ptr(), pool, pool, pooled.data_ptr(),
              2 if prec == "bf16x3" else 1, ws.data_ptr(), nb, _lib.stream())
    return spikes, rec, cnt, pooled


@pytest.mark.parametrize("prec", ["bf16x3", "bf16x2"])
def test_nets_layer_equals_single_network_calls(prec):
    x = _codes(10, 28, seed=3)
    offsets = [0, 4, 6, 10]
    thr = [15.0, 11.0, 18.5]
    kernels = torch.from_numpy(np.stack([synth.conv_weights(30, 2, 5, seed=s) for s in (1, 2, 3)])).to(DEV)
    spikes, rec, cnt, pooled = _nets_layer(x, kernels, offsets, thr, 5, 3, 2, prec)
    assert _lib.lib.spk_device_status(1) == 0
    for n in range(3):
        sl = slice(offsets[n], offsets[n + 1])
        conv = spyker.Conv(2, 30, 5, pad=2, device=DEV)
        conv.kernel.copy_(kernels[n])
        conv.precision = prec
        s1, w1, p1 = spyker.conv_fire_wta(x[sl], conv, thr[n], 3, 5, pool=2)
        assert torch.equal(spikes[sl], s1) and torch.equal(pooled[sl], p1)
        assert torch.equal(cnt[sl], w1.counts)
        for i in range(offsets[n + 1] - offsets[n]):
            k = int(w1.counts[i])
            assert torch.equal(rec[offsets[n] + i, :k], w1.records[i, :k])
    assert int(cnt.sum()) > 0


def test_nets_layer_rejects_network_inside_a_tile():
    x = _codes(4, 20, seed=1)  # 400 pixels per image, 8-pixel tiles: fine
    k = torch.from_numpy(np.stack([synth.conv_weights(30, 2, 5, seed=s) for s in (1, 2)])).to(DEV)
    _nets_layer(x, k, [0, 1, 4], [15.0, 12.0], 5, 3, 2)
    q = spyker.pool(_nets_layer(x, k, [0, 1, 4], [15.0, 12.0], 5, 3, 2)[0], 2)  # 10x10: 100 pixels per image
    k2 = torch.from_numpy(np.stack([synth.conv_weights(100, 30, 5, seed=s) for s in (1, 2)])).to(DEV)
    with pytest.raises(spyker.SpykerError):
        _nets_layer(q, k2, [0, 1, 4], [10.0, 8.0], 8, 1, 10)  # sample 1 starts mid-tile


def test_scan_nets_equals_single_scans_in_order():
    rng = np.random.default_rng(0)
    x = _codes(12, 28, seed=5)
    conv = spyker.Conv(2, 30, 5, pad=2, device=DEV)
    conv.kernel.copy_(torch.from_numpy(synth.conv_weights(30, 2, 5, seed=1)))
    conv.precision = "bf16x3"
    spikes, wins = spyker.conv_fire_wta(x, conv, 13.0, 3, 5)
    b, k, count = 12, 50, 5
    pre = torch.zeros((b, count, k), dtype=torch.int16, device=DEV)
    post = torch.zeros((b, count), dtype=torch.int16, device=DEV)
    nb = _lib.lib.spk_rank_convstdp_prepost_workspace(b, 2, 28, 28)
    ws = torch.empty(max(int(nb), 1), dtype=torch.uint8, device=DEV)
    _lib.call("spk_rank_convstdp_prepost", x.data_ptr(), 4, b, 15, 2, 28, 28, 30, 5, 5, spikes.data_ptr(), 28, 28,
              wins.records.data_ptr(), wins.counts.data_ptr(), count, 1, 1, i64(2, 2, 2, 2), pre.data_ptr(),
              post.data_ptr(), ws.data_ptr(), int(nb), _lib.stream())
    # 3 networks over interleaved samples, each in a shuffled order
    owners = [np.array([0, 3, 5, 9]), np.array([1, 2, 6, 7, 11]), np.array([4, 8, 10])]
    orders = [rng.permutation(o) for o in owners]
    cfgs = [(0.004, -0.003, 1.0, 0.0, 1.0), (0.008, -0.006, 1.0, 0.0, 1.0), (0.002, -0.0015, 0.0, 0.0, 1.0)]
    kern = torch.from_numpy(np.stack([synth.conv_weights(30, 2, 5, seed=s) for s in (7, 8, 9)])).to(DEV)
    want = kern.clone()
    for n in range(3):
        idx = torch.from_numpy(orders[n]).to(DEV)
        # the gathered copies stay referenced until the scan has run
        rec, cnt = wins.records[idx].contiguous(), wins.counts[idx].contiguous()
        pr, po = pre[idx].contiguous(), post[idx].contiguous()
        _lib.call("spk_stdp_scan", want[n].data_ptr(), 30, k, len(idx), count, 2, rec.data_ptr(), cnt.data_ptr(),
                  pr.data_ptr(), count * k, k, po.data_ptr(), _lib.f64(cfgs[n]), 1, 0, _lib.stream())
        torch.cuda.synchronize()
    order = torch.from_numpy(np.concatenate(orders).astype(np.int32)).to(DEV)
    noff = torch.tensor([0, 4, 9, 12], dtype=torch.int64, device=DEV)
    cfg = torch.tensor(cfgs, dtype=torch.float64, device=DEV)
    got = kern.clone()
    _lib.call("spk_stdp_scan_nets", got.data_ptr(), 3, 30, k, b, count, 2, wins.records.data_ptr(),
              wins.counts.data_ptr(), pre.data_ptr(), count * k, k, post.data_ptr(), noff.data_ptr(), order.data_ptr(),
              cfg.data_ptr(), 1, 0, _lib.stream())
    assert torch.equal(got, want)
    assert all(not torch.equal(got[n], kern[n]) for n in range(3))


def _alone(sw, n):
    """Network n trained alone: per size group its own single-network layer
    calls, then its winners' updates in its stream order."""
    spec = sw.specs[n]
    w1 = torch.from_numpy(spec.w1).to(DEV)
    w2 = torch.from_numpy(spec.w2).to(DEV)
    per_layer = [[], []]  # (stream position, records, counts, pre, post) per sample
    pooled1 = {}
    c1 = spyker.Conv(2, 30, 5, pad=2, device=DEV)
    c2 = spyker.Conv(30, 100, 5, pad=2, device=DEV)
    c1.precision = c2.precision = "bf16x3"
    c1.kernel.copy_(w1)
    c2.kernel.copy_(w2)
    layers = [(c1, spec.theta, 3, 5, 2), (c2, spec.theta2, 1, 8, None)]
    inputs = {}
    for g in sw.groups:
        _, pos, imgs = g.per_net[n]
        if len(pos) == 0:
            continue
        x = torch.from_numpy(imgs).to(DEV).float().div_(255)[:, None]
        inputs[g.size] = (pos, sw.dog(x))
    for li, (conv, thr, radius, count, pool) in enumerate(layers):
        for size, (pos, xin) in inputs.items():
            x = spyker.code(xin, 15) if li == 0 else pooled1[size]
            if pool:
                spk, wins, pooled1[size] = spyker.conv_fire_wta(x, conv, thr, radius, count, pool=pool)
            else:
                spk, wins = spyker.conv_fire_wta(x, conv, thr, radius, count)
            b, _, cin, h, w = x.shape
            k = cin * 25
            pre = torch.zeros((b, count, k), dtype=torch.int16, device=DEV)
            post = torch.zeros((b, count), dtype=torch.int16, device=DEV)
            nb = _lib.lib.spk_rank_convstdp_prepost_workspace(b, cin, h, w)
            ws = torch.empty(max(int(nb), 1), dtype=torch.uint8, device=DEV)
            _lib.call("spk_rank_convstdp_prepost", x.data_ptr(), 4, b, 15, cin, h, w, conv.kernel.shape[0], 5, 5,
                      spk.data_ptr(), h, w, wins.records.data_ptr(), wins.counts.data_ptr(), count, 1, 1,
                      i64(2, 2, 2, 2), pre.data_ptr(), post.data_ptr(), ws.data_ptr(), int(nb), _lib.stream())
            for i, p in enumerate(pos):
                per_layer[li].append((int(p), wins.records[i], wins.counts[i], pre[i], post[i]))
        rows = sorted(per_layer[li], key=lambda e: e[0])
        rec = torch.stack([r[1] for r in rows]).contiguous()
        cnt = torch.stack([r[2] for r in rows]).contiguous()
        pr = torch.stack([r[3] for r in rows]).contiguous()
        po = torch.stack([r[4] for r in rows]).contiguous()
        k = pr.shape[-1]
        _lib.call("spk_stdp_scan", conv.kernel.data_ptr(), conv.kernel.shape[0], k, len(rows), count, 2,
                  rec.data_ptr(), cnt.data_ptr(), pr.data_ptr(), count * k, k, po.data_ptr(),
                  _lib.f64((spec.pos, spec.neg, 1.0, 0.0, 1.0)), 1, 0, _lib.stream())
    return c1.kernel, c2.kernel


@pytest.mark.parametrize("path", ["dense", "search"])
def test_sweep_step_equals_each_network_alone(path):
    sw = sweep.Sweep(nets=3, images=7, sizes=(20, 28), seed=1, device=DEV, tune=False, path=path)
    sw.step()
    assert _lib.lib.spk_device_status(1) == 0
    for n in range(3):
        k1, k2 = _alone(sw, n)
        assert torch.equal(sw.w1[n], k1), n
        assert torch.equal(sw.w2[n], k2), n
        assert not torch.equal(k1, torch.from_numpy(sw.specs[n].w1).to(DEV))


def test_sweep_graph_replay_and_tuned_schedules():
    eager = sweep.Sweep(nets=4, images=6, sizes=(20, 28, 40), seed=2, device=DEV, tune=False)
    eager.step()
    eager.step()
    tuned = sweep.Sweep(nets=4, images=6, sizes=(20, 28, 40), seed=2, device=DEV, tune=True)
    assert set(tuned.schedules) == {(g, l) for g in range(3) for l in range(2)}
    tuned.capture()  # runs one step while warming up
    tuned.replay()
    torch.cuda.synchronize()
    assert torch.equal(tuned.w1, eager.w1) and torch.equal(tuned.w2, eager.w2)
    for a, b in zip(tuned.graph_features, eager.last_features):
        assert torch.equal(a, b)


def test_sweep_search_path_equals_dense_path_and_replays():
    """Per-network single-network calls (path="search") against the
    multi-network kernel (path="dense") over all four image sizes: two
    steps, the search path's second one a CUDA-graph replay; weights and
    features equal bit for bit."""
    dense = sweep.Sweep(nets=4, images=6, sizes=(20, 28, 40, 64), seed=2, device=DEV, tune=False, path="dense")
    dense.step()
    dense.step()
    srch = sweep.Sweep(nets=4, images=6, sizes=(20, 28, 40, 64), seed=2, device=DEV, tune=False, path="search")
    assert srch.schedules == {}
    srch.capture()  # runs one step while warming up
    srch.replay()
    torch.cuda.synchronize()
    assert _lib.lib.spk_device_status(1) == 0
    assert torch.equal(srch.w1, dense.w1) and torch.equal(srch.w2, dense.w2)
    assert not torch.equal(srch.w2, torch.from_numpy(np.stack([s.w2 for s in srch.specs])).to(DEV))
    for a, b in zip(srch.graph_features, dense.last_features):
        assert torch.equal(a, b)
