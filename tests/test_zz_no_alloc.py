"""spk_rank_convstdp_noalloc: conv STDP for callers that cannot allocate.

Such callers (hosts whose allocator owns all of the device's memory, C code
without a device allocator) cannot hand spk_rank_convstdp a
workspace; the no-alloc entry point keeps its scratch in a static device
array instead.  This checks, through the C ABI, that two calls in a row give
exactly the weights of the workspace entry point (STDP results are compared
bit-exactly, as in the other STDP tests), with the second call on a
different, larger problem so stale scratch from the first call would show.
It also checks the size limit is enforced.  Collected last on purpose.
"""

import numpy as np
import pytest
import torch

from spyker_b200 import _lib, synth

pytestmark = pytest.mark.gpu
CFG = [0.004, -0.003, 1.0, 0.0, 1.0]


def _case(port, n, seed, cout=30):
    rng = np.random.default_rng(seed)
    img = synth.strokes(n, seed=seed).astype(np.float32) / 255
    x = img[:, None] + rng.random((n, 2, 28, 28), dtype=np.float32) * 0.01
    codes = port.rank_code(x.astype(np.float32), 15)
    w = synth.conv_weights(cout, 2, 5, seed=seed + 1)
    pot = port.conv(codes, w, (1, 1), (2, 2, 2, 2))
    spk = port.fire(port.inhibit(port.threshold(pot, 15.0)))
    win, cnt = port.convwta(spk, (3, 3), 5)
    return codes, w, spk, win.astype(np.int32), cnt.astype(np.int32)


def _run(entry, codes, w, spk, win, cnt):
    dev = torch.device("cuda", 0)
    x = torch.from_numpy(codes).to(dev)
    o = torch.from_numpy(spk).to(dev)
    k = torch.from_numpy(w).to(dev)
    rec = torch.from_numpy(win).to(dev)
    cn = torch.from_numpy(cnt).to(dev)
    b, t, cin, h, wd = codes.shape
    cout, _, kh, kw = w.shape
    cfg = _lib.f64(CFG)
    pad = _lib.i64(2, 2, 2, 2)
    s = torch.cuda.current_stream().cuda_stream
    common = (x.data_ptr(), 4, b, t, cin, h, wd, k.data_ptr(), cout, kh, kw, o.data_ptr(), spk.shape[3],
              spk.shape[4], cfg, 1, rec.data_ptr(), cn.data_ptr(), win.shape[1], 1, 1, pad)
    if entry == "workspace":
        nb = _lib.lib.spk_rank_convstdp_workspace(b, win.shape[1], cin, h, wd, kh, kw)
        ws = torch.empty(nb, dtype=torch.uint8, device=dev)
        _lib.call("spk_rank_convstdp", *common, ws.data_ptr(), nb, s)
    else:
        _lib.call("spk_rank_convstdp_noalloc", *common, s)
    torch.cuda.synchronize()
    return k.cpu().numpy()


def test_noalloc_matches_workspace_entry_point_twice(port):
    first = _case(port, 12, seed=31)
    second = _case(port, 40, seed=57)
    for case in (first, second):
        want = _run("workspace", *case)
        got = _run("noalloc", *case)
        assert not np.array_equal(want, case[1]), "the update must change some weights"
        assert np.array_equal(got, want)


def test_noalloc_rejects_oversized_calls(port):
    # 2 * B * count * Cin*KH*KW bytes beyond 32 MiB: refused before any launch.
    b, count, cin, kh, kw = 4096, 8, 30, 11, 11
    assert _lib.lib.spk_rank_convstdp_workspace(b, count, cin, 14, 14, kh, kw) > (32 << 20)
    st = _lib.lib.spk_rank_convstdp_noalloc(None, 4, b, 15, cin, 14, 14, None, 100, kh, kw, None, 14, 14,
                                            _lib.f64(CFG), 1, None, None, count, 1, 1, _lib.i64(5, 5, 5, 5), None)
    assert st == 1
    assert b"static scratch" in _lib.lib.spk_last_error()


def _cumulative(rng, b, t, c, h, w):
    first = rng.integers(0, t + 1, size=(b, 1, c, h, w))
    return (np.arange(t)[None, :, None, None, None] >= first).astype(np.uint8)


def test_noalloc_limit_boundary():
    # 2*B*count*Cin*KH*KW + 2*B*count bytes, each rounded up to 256: exactly
    # 32 MiB for B=4088, count=8, Cin=8, 8x8 kernels (accepted, and equal to
    # the workspace entry point), 256 bytes more for B=5592402, count=1,
    # Cin=1, 1x2 kernels (refused before any launch).
    def need(b, count, k):
        a = lambda v: (v + 255) // 256 * 256
        return a(2 * b * count * k) + a(2 * b * count)

    assert need(4088, 8, 512) == 32 << 20 and need(5592402, 1, 2) == (32 << 20) + 256
    st = _lib.lib.spk_rank_convstdp_noalloc(None, 4, 5592402, 2, 1, 1, 2, None, 4, 1, 2, None, 1, 1,
                                            _lib.f64(CFG), 1, None, None, 1, 1, 1, _lib.i64(0, 0, 0, 0), None)
    assert st == 1 and b"static scratch" in _lib.lib.spk_last_error()

    rng = np.random.default_rng(5)
    b, t, cin, cout, count = 4088, 2, 8, 16, 8
    codes = _cumulative(rng, b, t, cin, 8, 8)
    out = _cumulative(rng, b, t, cout, 1, 1)
    win = np.zeros((b, count, 5), dtype=np.int32)
    win[:, :, 2] = rng.integers(0, cout, size=(b, count))
    cnt = rng.integers(0, count + 1, size=b).astype(np.int32)
    w = rng.uniform(0.2, 0.9, size=(cout, cin, 8, 8)).astype(np.float32)
    dev = torch.device("cuda", 0)
    x, o = torch.from_numpy(codes).to(dev), torch.from_numpy(out).to(dev)
    rec, cn = torch.from_numpy(win).to(dev), torch.from_numpy(cnt).to(dev)
    cfg, pad = _lib.f64(CFG), _lib.i64(0, 0, 0, 0)
    s = torch.cuda.current_stream().cuda_stream
    got = []
    for entry in ("workspace", "noalloc"):
        k = torch.from_numpy(w).to(dev)
        args = (x.data_ptr(), 4, b, t, cin, 8, 8, k.data_ptr(), cout, 8, 8, o.data_ptr(), 1, 1, cfg, 1,
                rec.data_ptr(), cn.data_ptr(), count, 1, 1, pad)
        if entry == "workspace":
            nb = _lib.lib.spk_rank_convstdp_workspace(b, count, cin, 8, 8, 8, 8)
            ws = torch.empty(nb, dtype=torch.uint8, device=dev)
            _lib.call("spk_rank_convstdp", *args, ws.data_ptr(), nb, s)
        else:
            _lib.call("spk_rank_convstdp_noalloc", *args, s)
        torch.cuda.synchronize()
        got.append(k.cpu().numpy())
    assert not np.array_equal(got[0], w)
    assert np.array_equal(got[0], got[1])
