"""Overlapped host->device batches (io.Prefetcher) and device->host results
(io.Readback): every batch arrives intact, in order, including the ragged
last one, for ring depths 1-3, while the consumer's kernels run on its own
stream; results read back equal the device values."""

import numpy as np
import pytest
import torch

import spyker_b200 as spyker
from spyker_b200 import io

pytestmark = pytest.mark.gpu
DEV = "cuda"


@pytest.mark.parametrize("depth", [1, 2, 3])
def test_prefetch_batches_in_order(depth, tmp_path):
    imgs = np.random.default_rng(depth).integers(0, 256, size=(1000, 28, 28), dtype=np.uint8)
    path = str(tmp_path / "x-idx3-ubyte")
    io.write_idx(path, imgs)
    host = spyker.mnist_data(path)
    assert host.is_pinned()
    pre = io.Prefetcher(host, 96, device=DEV, depth=depth)
    back = io.Readback(depth=2 * len(pre))  # every result kept
    outs, sums = [], []
    for x in pre:
        # a consumer that takes a while: several passes over the batch
        y = x.float()
        for _ in range(20):
            y = y * 1.0001
        sums.append(back.push(x.sum(dim=(1, 2, 3), dtype=torch.int64)))
        outs.append(back.push(x.clone()))
    back.synchronize()
    torch.cuda.synchronize()
    assert len(outs) == 11 and outs[-1].shape[0] == 1000 - 960
    got = torch.cat(outs).numpy()
    assert np.array_equal(got[:, 0], imgs)
    assert np.array_equal(torch.cat(sums).numpy(), imgs.reshape(1000, -1).sum(1))
    assert pre.bytes == imgs.nbytes


def test_prefetch_sequence_of_batches_and_readback_ring():
    parts = [torch.full((64, 3), k, dtype=torch.float32).pin_memory() for k in range(7)]
    pre = io.Prefetcher(parts, device=DEV, depth=2)
    back = io.Readback(depth=2)
    seen = []
    for k, x in enumerate(pre):
        h = back.push(x * 2)
        back.synchronize()
        seen.append(float(h[0, 0]))
        assert torch.equal(x, torch.full((64, 3), float(k), device=DEV))
    assert seen == [2.0 * k for k in range(7)]
    with pytest.raises(ValueError):
        io.Prefetcher([torch.zeros(3, device=DEV)])
