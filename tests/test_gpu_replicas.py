"""Data-parallel STDP on one GPU: two shards' (pre, post) arrays, computed
separately and concatenated as the rank-ordered all-gather would, then one
ordered scan, give exactly the single-call conv STDP of the whole batch."""

import numpy as np
import pytest
import torch

import spyker_b200 as spyker
from spyker_b200 import _lib, replicas, synth

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_prepost_then_scan_equals_full_stdp(world):
    rng = np.random.default_rng(world)
    b, t, cin, h, w, cout = 13, 15, 2, 28, 28, 30
    fst = rng.integers(0, t + 3, size=(b, cin, h, w))
    x = torch.from_numpy((fst[:, None] <= np.arange(t)[None, :, None, None, None]).astype(np.uint8)).to(DEV)
    layer = spyker.Conv(cin, cout, 5, pad=2)
    layer.kernel.copy_(torch.from_numpy(synth.conv_weights(cout, cin, 5, seed=9)))
    layer.precision = "bf16x3"
    layer.stdpconfig = [spyker.STDPConfig(0.004, -0.003)]
    spikes, wins = spyker.conv_fire_wta(x, layer, 6.0, 3, 5)
    k0 = layer.kernel.clone()

    # per-shard (pre, post), concatenated in rank order
    k = cin * 25
    pres, posts = [], []
    for r in range(world):
        sl = replicas.shard(b, r, world)
        xs, ss = x[sl].contiguous(), spikes[sl].contiguous()
        rec, cnt = wins.records[sl].contiguous(), wins.counts[sl].contiguous()
        n = xs.shape[0]
        pre = torch.empty((n, wins.count, k), dtype=torch.int16, device=DEV)
        post = torch.empty((n, wins.count), dtype=torch.int16, device=DEV)
        nb = _lib.lib.spk_rank_convstdp_prepost_workspace(n, cin, h, w)
        ws = torch.empty(max(int(nb), 1), dtype=torch.uint8, device=DEV)
        _lib.call("spk_rank_convstdp_prepost", xs.data_ptr(), 4, n, t, cin, h, w, cout, 5, 5, ss.data_ptr(), 28, 28,
                  rec.data_ptr(), cnt.data_ptr(), wins.count, 1, 1, _lib.i64(2, 2, 2, 2), pre.data_ptr(),
                  post.data_ptr(), ws.data_ptr(), int(nb), _lib.stream())
        pres.append(pre), posts.append(post)
    pre, post = torch.cat(pres), torch.cat(posts)
    _lib.call("spk_stdp_scan", layer.kernel.data_ptr(), cout, k, b, wins.count, 2, wins.records.data_ptr(),
              wins.counts.data_ptr(), pre.data_ptr(), wins.count * k, k, post.data_ptr(), _lib.f64([0.004, -0.003, 1, 0, 1]),
              1, 0, _lib.stream())
    got = layer.kernel.clone()

    layer.kernel.copy_(k0)
    layer.stdp(x, wins, spikes)
    assert not torch.equal(layer.kernel, k0)
    assert torch.equal(got, layer.kernel)
    # without a process group, replicas.conv_stdp is the plain update
    layer.kernel.copy_(k0)
    replicas.conv_stdp(layer, x, wins, spikes)
    assert torch.equal(layer.kernel, got)
