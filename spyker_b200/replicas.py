"""Several GPUs, one process per GPU (torch.distributed, NCCL over NVLink).

Forward passes, feature extraction and independent networks need no
exchange: each rank takes its shard of the images (``shard``) and works alone
("replicas").

STDP training of one network is sequential in its weights (the reference
applies the winners sample after sample, ``src/spyker/cpu/stdp.cpp:99-169``).
Across G ranks each rank runs the forward pass and the winner selection of its
shard, computes the (pre, post) first-spike times of its winners, and the
ranks all-gather those arrays (a few KB per image); every rank then applies
the same ordered STDP scan to its copy of the weights.  Shards are
consecutive and gathered in rank order, so the scan sees the winners in the
order of one GPU training on the whole batch: the copies stay identical,
and equal to the single-GPU weights, without an all-reduce.
"""

from __future__ import annotations

from typing import Optional

import torch
import torch.distributed as dist

from . import _lib
from ._lib import call, i64, ptr, stream


def shard(n: int, rank: int, world: int) -> slice:
    """Consecutive shard of ``n`` items for ``rank`` (the first ``n % world``
    ranks take one more)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("invalid rank / world size")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


def gather_rows(t: torch.Tensor, group: Optional[dist.ProcessGroup] = None) -> torch.Tensor:
    """Concatenation over ranks, in rank order, of each rank's ``t`` (same
    shape except the first dimension).  Moves raw bytes, so any dtype
    travels (NCCL has no 16-bit integer type)."""
    world = dist.get_world_size(group)
    if world == 1:
        return t
    t = t.contiguous()
    rows = torch.tensor([t.shape[0]], dtype=torch.int64, device=t.device)
    sizes = [torch.zeros_like(rows) for _ in range(world)]
    dist.all_gather(sizes, rows, group=group)
    sizes = [int(s.item()) for s in sizes]
    most = max(sizes)
    row_elems = 1
    for d in t.shape[1:]:
        row_elems *= int(d)
    row_bytes = row_elems * t.element_size()
    flat = t.reshape(t.shape[0], row_elems).view(torch.uint8)
    buf = torch.zeros((most, row_bytes), dtype=torch.uint8, device=t.device)
    buf[: t.shape[0]] = flat
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = torch.cat([p[:n] for p, n in zip(parts, sizes)], dim=0)
    return out.view(t.dtype).reshape((sum(sizes),) + tuple(t.shape[1:]))


def gather_packed(parts, rows_per_rank, group: Optional[dist.ProcessGroup] = None):
    """Rank-ordered concatenation of several per-sample tensors in ONE
    all-gather and without a host synchronisation: ``parts`` are this rank's
    tensors (same first dimension, any dtypes), ``rows_per_rank`` the first
    dimension of every rank (known from the shard arithmetic, e.g.
    :func:`shard`).  Each sample's rows of all parts travel as one byte row;
    shards shorter than the longest are padded.  Returns the gathered tensors
    in the order of ``parts``."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if len(rows_per_rank) != world:
        raise ValueError("rows_per_rank must give every rank's rows")
    if world == 1:
        return [p for p in parts]
    n = int(rows_per_rank[rank])
    dev = parts[0].device
    widths, flats = [], []
    for p in parts:
        if p.shape[0] != n:
            raise ValueError("every part must have this rank's rows")
        f = p.contiguous().reshape(n, -1).view(torch.uint8) if p.numel() else torch.empty((n, 0), dtype=torch.uint8,
                                                                                              device=dev)
        flats.append(f)
        widths.append(f.shape[1])
    most = max(int(r) for r in rows_per_rank)
    row = sum(widths)
    buf = torch.zeros((most, row), dtype=torch.uint8, device=dev)
    col = 0
    for f, w in zip(flats, widths):
        buf[:n, col:col + w] = f
        col += w
    out = torch.empty((world * most, row), dtype=torch.uint8, device=dev)
    dist.all_gather_into_tensor(out, buf, group=group)
    keep = torch.cat([torch.arange(q * most, q * most + int(r), device=dev) for q, r in enumerate(rows_per_rank)])
    rows = out.index_select(0, keep)
    total = int(sum(int(r) for r in rows_per_rank))
    res, col = [], 0
    for p, w in zip(parts, widths):
        piece = rows[:, col:col + w].contiguous()
        col += w
        res.append(piece.view(p.dtype).reshape((total,) + tuple(p.shape[1:])))
    return res


def max_over_ranks(x: float, group: Optional[dist.ProcessGroup] = None, device=None) -> float:
    """The largest ``x`` over the ranks (step times are reported this way)."""
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def conv_stdp(layer, array: torch.Tensor, winners, output: torch.Tensor,
              group: Optional[dist.ProcessGroup] = None, batch: Optional[int] = None) -> None:
    """``layer.stdp(array, winners, output)`` for the whole batch split over
    the ranks: ``array``, ``output`` and ``winners`` are this rank's shard
    (consecutive images, shards in rank order); every rank's ``layer.kernel``
    receives the update of the full batch.  With ``batch`` (the full batch,
    sharded by :func:`shard`) the winners and (pre, post) times of all ranks
    travel in one all-gather with no host synchronisation; without it the
    shard sizes are gathered first."""
    from .module import Winners, _check_winners, _configs
    from .utils import Bound, to5

    if len(layer.stdpconfig) == 0:
        raise ValueError("At least one STDP Config must be given.")
    x = Bound(array, layer.device).dev
    o = Bound(output, layer.device).dev
    s, so = to5(list(x.shape)), to5(list(o.shape))
    w = Winners.from_lists(winners, x.device)
    _check_winners(w, len(layer.stdpconfig), s[0])
    cout, cin, kh, kw = layer.kernel.shape
    k = cin * kh * kw
    pre = torch.empty((s[0], w.count, k), dtype=torch.int16, device=x.device)
    post = torch.empty((s[0], w.count), dtype=torch.int16, device=x.device)
    nb = _lib.lib.spk_rank_convstdp_prepost_workspace(s[0], cin, s[3], s[4])
    ws = torch.empty(max(int(nb), 1), dtype=torch.uint8, device=x.device)
    call("spk_rank_convstdp_prepost", ptr(x), _code(x.dtype), s[0], s[1], cin, s[3], s[4], cout, kh, kw, ptr(o), so[3],
         so[4], ptr(w.records), ptr(w.counts), w.count, layer._stride[0], layer._stride[1], i64(*layer._pad), ptr(pre),
         ptr(post), ptr(ws), int(nb), stream())
    if dist.is_initialized() and batch is not None:
        world = dist.get_world_size(group)
        sizes = [len(range(batch)[shard(batch, r, world)]) for r in range(world)]
        records, counts, pre, post = gather_packed([w.records, w.counts, pre, post], sizes, group)
    elif dist.is_initialized():
        records, counts = gather_rows(w.records, group), gather_rows(w.counts, group)
        pre, post = gather_rows(pre, group), gather_rows(post, group)
    else:
        records, counts = w.records, w.counts
    b = records.shape[0]
    call("spk_stdp_scan", ptr(layer.kernel), cout, k, b, w.count, 2, ptr(records), ptr(counts), ptr(pre), w.count * k,
         k, ptr(post), _configs(layer.stdpconfig), len(layer.stdpconfig), 0, stream())


def _code(dtype: torch.dtype) -> int:
    from .utils import type_code

    return type_code(dtype)
