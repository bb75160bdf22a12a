"""Host logic of the multi-GPU path on CPU ranks (gloo, world size 2).

The GPU kernels are the single-GPU ones; what is specific to several ranks
is the sharding of the batch, the rank-ordered gather of the winner records
and (pre, post) arrays, and the max over ranks of the step time.  These run
here as two gloo processes on CPU tensors.
"""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from spyker_b200 import replicas, synth
from tests.golden import make_golden


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank: int, world: int, port: int) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))


def test_shard_partitions():
    for n in (0, 1, 7, 4096):
        for world in (1, 2, 3, 8):
            parts = [replicas.shard(n, r, world) for r in range(world)]
            assert parts[0].start == 0 and parts[-1].stop == n
            assert all(a.stop == b.start for a, b in zip(parts, parts[1:]))
            sizes = [p.stop - p.start for p in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)


def _gather_worker(rank, world, port):
    _init(rank, world, port)
    try:
        rows = [3, 0] if world == 2 else [3]
        for dtype in (torch.int16, torch.int32, torch.uint8, torch.float64):
            mine = (torch.arange(rows[rank] * 6) + 100 * rank).reshape(rows[rank], 2, 3).to(dtype)
            got = replicas.gather_rows(mine)
            want = torch.cat([(torch.arange(r * 6) + 100 * q).reshape(r, 2, 3).to(dtype) for q, r in enumerate(rows)])
            assert got.dtype == dtype and got.shape == want.shape and torch.equal(got, want)
        # unequal non-empty shards
        mine = torch.full((rank + 2, 4), rank, dtype=torch.int16)
        got = replicas.gather_rows(mine)
        assert got.shape == (2 + 3, 4) and torch.equal(got[:2], torch.zeros(2, 4, dtype=torch.int16))
        assert replicas.max_over_ranks(1.5 + rank) == 2.5
    finally:
        dist.destroy_process_group()


def test_gather_rows_two_ranks():
    mp.spawn(_gather_worker, args=(2, _free_port()), nprocs=2, join=True)


def _stdp_worker(rank, world, port, root):
    """Each rank takes its shard of the images, selects its winners and
    gathers them: the gathered records are the single-process ones, in
    order, so the ordered STDP scan on them is the single-process update."""
    import sys

    sys.path.insert(0, root)
    import oracle

    _init(rank, world, port)
    try:
        port_ = oracle.get("port")
        imgs = synth.strokes(10, seed=4).astype(np.float32) / 255
        dog = port_.filter("dog", imgs[:, None], make_golden.dog_kernel(port_), (3, 3, 3, 3))
        codes = port_.rank_code(dog, 15)
        w = synth.conv_weights(30, 2, 5, seed=2)

        def winners(c):
            inh = port_.inhibit(port_.threshold(port_.conv(c, w, (1, 1), (2, 2, 2, 2)), 15.0))
            return port_.convwta(inh, (3, 3), 5), port_.fire(inh)

        (full_win, full_cnt), full_spk = winners(codes)
        sl = replicas.shard(codes.shape[0], rank, world)
        (win, cnt), spk = winners(codes[sl])
        g_win = replicas.gather_rows(torch.from_numpy(win.astype(np.int32))).numpy()
        g_cnt = replicas.gather_rows(torch.from_numpy(cnt.astype(np.int32))).numpy()
        g_spk = replicas.gather_rows(torch.from_numpy(spk)).numpy()
        assert np.array_equal(g_win, full_win.astype(np.int32)) and np.array_equal(g_cnt, full_cnt.astype(np.int32))
        assert np.array_equal(g_spk, full_spk)
        cfg = [(0.004, -0.003, 1.0, 0.0, 1.0)]
        got = port_.convstdp(codes, w, g_spk, cfg, g_win.astype(np.int64), g_cnt.astype(np.int64), (1, 1), (2, 2, 2, 2))
        want = port_.convstdp(codes, w, full_spk, cfg, full_win, full_cnt, (1, 1), (2, 2, 2, 2))
        assert np.array_equal(got, want) and not np.array_equal(want, w)
    finally:
        dist.destroy_process_group()


def test_stdp_winners_gathered_in_order(port):
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    mp.spawn(_stdp_worker, args=(2, _free_port(), root), nprocs=2, join=True)


def _packed_worker(rank, world, port):
    """The winners' records (int32) and (pre, post) first-spike times (int16)
    of unequal shards travel in one all-gather and come back bit for bit in
    rank order."""
    _init(rank, world, port)
    try:
        batch = 7
        sizes = [len(range(batch)[replicas.shard(batch, r, world)]) for r in range(world)]
        g = torch.Generator().manual_seed(5)
        full_rec = torch.randint(-2 ** 31, 2 ** 31 - 1, (batch, 3, 5), dtype=torch.int32, generator=g)
        full_cnt = torch.randint(0, 4, (batch,), dtype=torch.int32, generator=g)
        full_pre = torch.randint(-2 ** 15, 2 ** 15 - 1, (batch, 3, 50), dtype=torch.int16, generator=g)
        full_post = torch.randint(0, 16, (batch, 3), dtype=torch.int16, generator=g)
        sl = replicas.shard(batch, rank, world)
        got = replicas.gather_packed([full_rec[sl], full_cnt[sl], full_pre[sl], full_post[sl]], sizes)
        for a, b in zip(got, (full_rec, full_cnt, full_pre, full_post)):
            assert a.dtype == b.dtype and a.shape == b.shape and torch.equal(a, b)
        with pytest.raises(ValueError):
            replicas.gather_packed([full_rec[sl]], sizes[:1])
    finally:
        dist.destroy_process_group()


def test_gather_packed_int16_two_ranks():
    mp.spawn(_packed_worker, args=(2, _free_port()), nprocs=2, join=True)
