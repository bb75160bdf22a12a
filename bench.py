"""Benchmark: images/s of Kheradpisheh-style 2-layer STDP training + forward.

Workload (one step = one batch of 4096 synthetic 28x28 stroke images, the
MNIST geometry of the reference's examples):
  DoG(7x7, (1,2), (2,1), pad 3) -> rank code T=15 ->
  conv1 30x5x5 pad 2 -> threshold 15 -> inhibit -> convwta(r3, k5) -> fire ->
  STDP(0.004, -0.003) -> pool 2 ->
  conv2 100x5x5 pad 2 -> threshold 10 -> inhibit -> convwta(r1, k8) -> fire ->
  STDP(0.004, -0.003) -> global max pool (the features).

``value``: images/s with the images already on the GPU; ``e2e``: the same
through the public API from pinned host images, with the H2D copy of the
images and the D2H copy of the features and both kernels inside the timed
region.  ``--impl reference`` times the reference's CPU implementation (its
own compiled CPU backend, oneDNN convolution through torch) on host cores.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BATCH, T, H = 4096, 15, 28
# DRAM bytes (read + write) of one conv2 layer call (its 27 launches, the
# 4096-image step): ncu's dram__bytes_read.sum + dram__bytes_write.sum summed
# over the call's launches, 611.6 MB read + 1169.6 MB written (1.20 GB of it
# the layer's [B, T, 100, 14, 14] spike output).
CONV2_TRAFFIC_BYTES = int((611.6 + 1169.6) * 1e6)
METRIC = "images/s (STDP train + fwd), BF16-split vs FP32 on 1 B200; spike match %"
WORKLOAD = "kheradpisheh-2layer-stdp: 4096 x 28x28 strokes, T=15, conv1 30x5x5 th15 r3k5, conv2 100x5x5 th10 r1k8"


def bf16_peak():
    """Sustained BF16 denominator: the pool's measured figure when the
    measurement file is present, else the profiling recipe's fallback."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        v = json.load(open(path)).get("bf16_tflops_sustained")
        if v:
            return float(v), "MEASURED_PEAKS.json bf16_tflops_sustained (of measured)"
    return 1400.0, "sustained cuBLAS BF16 of an earlier measurement on this pool (of fallback)"


def path_dtype(precision: str):
    """(dtype, arithmetic) of the fused layers.  With non-negative weights
    (STDP keeps them in [0, 1]) a fused layer takes the first-crossing search:
    u8 spikes x u8 base-256 weight digits on the tensor cores with exact S32
    sums, each potential rounded once from the exact sum; other weights take
    the dense split kernel of ``precision``."""
    if precision == "fp32":
        return "f32", "FP32 SIMT convolution, op by op"
    return "u8", (f"u8 spikes x 4 u8 weight digits (tcgen05 kind::i8, exact S32 sums, potentials rounded once "
                  f"from the exact sum); {precision}-split/f32-acc dense kernel when a weight is negative")


def headline_config(batch: int, world: int, mode: str = "replicas") -> dict:
    """The workload's `config`, shared by both arms of the bench."""
    return {"workload": WORKLOAD.replace("4096 x", f"{batch} x"), "global_batch": batch * world, "seq_len": T,
            "parallelism": f"{mode}{world}",
            "l2": "inputs larger than L2: each step writes its own 1.44 GB layer-1 spike tensor (126 MB L2)"}


def flops_per_image():
    c1 = 2 * T * 28 * 28 * 30 * 2 * 25
    c2 = 2 * T * 14 * 14 * 100 * 30 * 25
    return c1, c2


# ----------------------------------------------------------------------------
# clocks
# ----------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index, self.samples, self.stop = index, [], threading.Event()

    def _run(self):
        while not self.stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                self.samples.append([v.strip() for v in out.stdout.strip().split(",")])
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        self.th = threading.Thread(target=self._run, daemon=True)
        self.th.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.th.join(timeout=10)

    def summary(self):
        sm = [float(s[1]) for s in self.samples if len(s) >= 9 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) >= 9 and s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples if len(s) >= 9 for i in range(4) if s[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ----------------------------------------------------------------------------
# GPU arm
# ----------------------------------------------------------------------------
class Network:
    def __init__(self, spyker, torch, dev, precision):
        from spyker_b200 import synth

        self.sp, self.torch = spyker, torch
        self.dog = spyker.DoG(3, [spyker.DoGFilter(1, 2), spyker.DoGFilter(2, 1)], pad=3, device=dev)
        self.conv1 = spyker.Conv(2, 30, 5, pad=2, device=dev)
        self.conv2 = spyker.Conv(30, 100, 5, pad=2, device=dev)
        self.conv1.kernel.copy_(torch.from_numpy(synth.conv_weights(30, 2, 5, seed=1)))
        self.conv2.kernel.copy_(torch.from_numpy(synth.conv_weights(100, 30, 5, seed=2)))
        for c in (self.conv1, self.conv2):
            c.stdpconfig = [spyker.STDPConfig(0.004, -0.003)]
            c.precision = precision
        self.conv_events = []
        # Layer 1's STDP runs on `side` while layer 2's forward runs on the
        # main stream (layer 2 reads layer 1's spikes, not its weights),
        # joined before the next layer 1; layer 2's on `side2` while the next
        # step's front end and layer 1 run, joined before the next layer 2
        # (both by finish()).  The search rounds claim their tiles as CTAs
        # become free, so an SM held by an update's CTA delays no tile.
        self.side = torch.cuda.Stream(dev)
        self.side2 = torch.cuda.Stream(dev)
        # the STDP update of a layer: this rank's batch alone, or (data
        # parallel) the whole batch over the ranks
        self.stdp_fn = lambda layer, x, win, spk: layer.stdp(x, win, spk)

    def _conv(self, layer, x):
        t = self.torch
        a, b = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
        a.record()
        y = layer(x)
        b.record()
        self.conv_events.append((a, b, layer))
        return y

    def _layer(self, layer, x, theta, radius, count, pool):
        """conv -> threshold -> inhibit -> (fire, convwta) -> pool: one fused
        kernel on the tensor-core precisions, op by op on the FP32 path."""
        t = self.torch
        timed = not t.cuda.is_current_stream_capturing()  # no timing events inside a CUDA graph
        a, b = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
        if timed:
            a.record()
        if getattr(self, "probe", None):
            self.probe()
        if layer.precision == "fp32":
            out = self.sp.inhibit(self.sp.threshold(layer(x), theta))
            spk, wins = self.sp.fire(out), self.sp.convwta(out, radius, count)
            pooled = self.sp.pool(spk, pool)
        else:
            spk, wins, pooled = self.sp.conv_fire_wta(x, layer, theta, radius, count, pool=pool)
        if timed:
            b.record()
            self.conv_events.append((a, b, layer))
        if getattr(self, "probe", None):
            self.probe()
        return spk, wins, pooled

    def step(self, images_f32):
        sp = self.sp
        codes = sp.code(self.dog(images_f32), T)
        main = self.torch.cuda.current_stream()
        main.wait_stream(self.side)  # the previous step's layer-1 update
        spk1, win1, pooled = self._layer(self.conv1, codes, 15.0, 3, 5, 2)
        self.side.wait_stream(main)
        with self.torch.cuda.stream(self.side):
            self.stdp_fn(self.conv1, codes, win1, spk1)
        main.wait_stream(self.side2)  # the previous step's layer-2 update
        spk2, win2, feats = self._layer(self.conv2, pooled, 10.0, 1, 8, 14)
        self.side2.wait_stream(main)
        with self.torch.cuda.stream(self.side2):
            self.stdp_fn(self.conv2, pooled, win2, spk2)
        if not self.torch.cuda.is_current_stream_capturing():
            # not reused before the updates have read them
            for x in (codes, spk1, win1.records, win1.counts):
                x.record_stream(self.side)
            for x in (pooled, spk2, win2.records, win2.counts):
                x.record_stream(self.side2)
        self.last_spikes = (spk1, spk2)
        return feats

    def finish(self):
        """Join the last STDP updates into the current stream."""
        cur = self.torch.cuda.current_stream()
        cur.wait_stream(self.side)
        cur.wait_stream(self.side2)


def gpu_arm(args, rank, world):
    import torch

    import spyker_b200 as spyker
    from spyker_b200 import io, synth

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    BATCH = args.batch
    imgs = synth.strokes(BATCH, seed=100 + rank)
    host = torch.from_numpy(imgs).pin_memory()
    dev_imgs = host.to(dev).float().div_(255.0)[:, None]
    net = Network(spyker, torch, dev, args.precision)
    if args.mode == "dp":
        # one network over the ranks: each rank's 4096 images are its shard
        # of a BATCH * world batch; the winners' (pre, post) times of all
        # ranks are gathered (one all-gather per layer) and every rank applies
        # the ordered update of the whole batch
        from spyker_b200 import replicas

        net.stdp_fn = lambda layer, x, win, spk: replicas.conv_stdp(layer, x, win, spk, batch=BATCH * world)
        args.graph = False  # collectives stay outside the captured graph

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        net.step(dev_imgs)
    barrier()
    # Training state over the warm-up: per step and layer, the rows the fused
    # layers re-decided exactly and the layers' times (synchronised, untimed)
    trajectory = []
    for k in range(args.trajectory):
        rec = []
        net.conv_events.clear()
        net.probe = lambda: (torch.cuda.synchronize(), rec.append((spyker._lib.lib.spk_recheck_count(1),
                                                                  spyker._lib.lib.spk_recompute_count(1))))
        spyker._lib.lib.spk_recheck_count(1)
        spyker._lib.lib.spk_recompute_count(1)
        net.step(dev_imgs)
        net.finish()
        torch.cuda.synchronize()
        net.probe = None
        c1, c2 = (a.elapsed_time(b) for a, b, _ in net.conv_events[:2])
        # per layer: rows re-decided from exact term sums, rows recomputed from the weights
        trajectory.append({"step": args.warmup + k, "rechecks": [rec[1][0], rec[3][0]],
                           "recomputes": [rec[1][1], rec[3][1]], "conv_ms": [c1, c2]})
    barrier()
    net.conv_events.clear()
    # The step as one CUDA graph: images from a u8 device buffer (the e2e leg
    # copies each step's images into it) to the features, both layers' STDP
    # updates included, captured once and replayed; launch gaps and host work
    # leave the step.
    static_u8 = torch.from_numpy(imgs).to(dev)
    graph = None
    if args.graph:
        def gstep():
            # both side streams fork from the capturing stream first, so that
            # every wait of the step refers to captured work
            cur = torch.cuda.current_stream()
            net.side.wait_stream(cur)
            net.side2.wait_stream(cur)
            f = net.step(static_u8.float().div_(255.0)[:, None])
            net.finish()
            return f
        gstep()
        barrier()
        graph = torch.cuda.CUDAGraph()
        l0 = spyker._lib.lib.spk_launch_count()
        with torch.cuda.graph(graph):
            feats_g = gstep()
        launches = spyker._lib.lib.spk_launch_count() - l0
        graph.replay()
        barrier()
    else:
        l0 = spyker._lib.lib.spk_launch_count()
    spyker._lib.lib.spk_recheck_count(1)
    spyker._lib.lib.spk_recompute_count(1)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(dev.index) as clk:
        barrier()
        start.record()
        h0 = time.perf_counter()
        for _ in range(args.steps):
            if graph is not None:
                graph.replay()
            else:
                net.step(dev_imgs)
        net.finish()
        end.record()
        # host time to enqueue the steps (the GPU runs behind it unless the
        # host is the slower side)
        host_ms = (time.perf_counter() - h0) * 1e3 / max(args.steps, 1)
        barrier()
    if graph is None:
        launches = (spyker._lib.lib.spk_launch_count() - l0) // max(args.steps, 1)
    rechecks = spyker._lib.lib.spk_recheck_count(1) / max(args.steps, 1)
    recomputes = spyker._lib.lib.spk_recompute_count(1) / max(args.steps, 1)
    ms = start.elapsed_time(end) / args.steps
    if graph is not None:
        # per-layer times from two eager steps (timing events cannot sit in a graph)
        for _ in range(2):
            net.step(dev_imgs)
        net.finish()
        barrier()
    # fired neurons of one step: a cumulative spike tensor's last step
    spikes_per_step = sum(int(s[:, -1].sum().item()) for s in net.last_spikes)
    conv_ms = {}
    for a, b, layer in net.conv_events:
        conv_ms.setdefault(id(layer), []).append(a.elapsed_time(b))
    c1f, c2f = flops_per_image()
    c1_ms = statistics.mean(conv_ms[id(net.conv1)])
    c2_ms = statistics.mean(conv_ms[id(net.conv2)])

    # end to end: pinned host images -> features in pinned host memory.  The
    # images of step k+1 are uploaded on a side stream while step k runs
    # (io.Prefetcher) and each step's features are read back on another
    # (io.Readback, two host buffers in turn); the timed region starts before
    # the first upload and ends after the last read-back has landed.
    net.step(dev_imgs)
    back = io.Readback(depth=2, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if graph is not None:
        # each step: pinned host images -> the graph's input buffer, replay,
        # features read back on a side stream (two host buffers in turn)
        barrier()
        e0.record()
        for _ in range(args.steps):
            static_u8.copy_(host, non_blocking=True)
            graph.replay()
            feats = back.push(feats_g)
        back.wait()
        e1.record()
        barrier()
    else:
        uploads = io.Prefetcher([host] * args.steps, device=dev, depth=2)
        barrier()
        e0.record()
        for raw in uploads:
            feats = back.push(net.step(raw.float().div_(255.0)[:, None]))
        net.finish()
        back.wait()
        e1.record()
        barrier()
    e2e_ms = e0.elapsed_time(e1) / args.steps

    # the same step on the plain FP32 path (the comparison the metric names)
    fp32 = None
    if args.precision != "fp32" and not args.no_fp32_compare:
        ref_net = Network(spyker, torch, dev, "fp32")
        ref_net.step(dev_imgs)
        barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        for _ in range(2):
            ref_net.step(dev_imgs)
        ref_net.finish()
        f1.record()
        barrier()
        fp32_ms = f0.elapsed_time(f1) / 2
        fp32 = {"value": BATCH / (fp32_ms * 1e-3), "unit": "images/s", "ms_per_step": fp32_ms, "steps": 2}
        del ref_net

    t_max = torch.tensor([ms, e2e_ms], device=dev)
    if dist is not None:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
        dist.destroy_process_group()
    ms, e2e_ms = float(t_max[0]), float(t_max[1])
    if rank != 0:
        return
    peak, peak_source = bf16_peak()
    achieved = c2f * BATCH / (c2_ms * 1e-3) / 1e12
    line = {
        "metric": METRIC,
        "value": BATCH * world / (ms * 1e-3),
        "unit": "images/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": path_dtype(args.precision)[0],
        "arithmetic": path_dtype(args.precision)[1],
        "data": "synthetic (seeded stroke images, MNIST geometry)",
        "config": headline_config(BATCH, world, args.mode),
        "conv_precision": args.precision,
        "e2e": {"value": BATCH * world / (e2e_ms * 1e-3), "unit": "images/s", "h2d_bytes_per_step": BATCH * H * H,
                "d2h_bytes_per_step": int(feats.numel() * feats.element_size())},
        "gpu_launches": int(launches),
        "host_enqueue_ms_per_step": host_ms,
        "cuda_graph": graph is not None,
        "roofline": {"bound": "tensor", "kernel": "conv2 (30->100, 5x5, M=12.0M, K=750)", "achieved": achieved,
                     "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": CONV2_TRAFFIC_BYTES * BATCH // 4096 if args.precision != "fp32" else None,
                     "traffic_source": "ncu dram__bytes_read+write summed over the conv2 layer call's launches "
                                       "(4096 images; scaled by the batch)",
                     "peak_source": peak_source},
        "kernels_ms": {"conv1": c1_ms, "conv2": c2_ms, "rest": ms - c1_ms - c2_ms},
        "clocks": clk.summary(),
        "spikes_per_s": spikes_per_step * world / (ms * 1e-3),
        "near_threshold_rechecks_per_step": rechecks,
        "rows_recomputed_per_step": recomputes,
    }
    if trajectory:
        line["trajectory"] = trajectory
    if args.dump_weights:
        np.savez(args.dump_weights, conv1=net.conv1.kernel.cpu().numpy(), conv2=net.conv2.kernel.cpu().numpy())
    if fp32 is not None:
        line["fp32_path"] = fp32
    if not args.no_cpu_baseline and world == 1:
        # the CPU leg: the oracle as the timed baseline and as the checker
        line["cpu_baseline"] = cpu_baseline(args.cpu_seconds)
        if not args.no_spike_match:
            line["spike_match"] = spike_match(spyker, torch, dev, args.precision,
                                              (net.conv1.kernel.cpu().numpy(), net.conv2.kernel.cpu().numpy()))
    print(json.dumps(line), flush=True)


def spike_match(spyker, torch, dev, precision, weights, n=32):
    """Spike match %: both layers' fire spikes of this path against the
    oracle's FP64 pipeline on `n` images, with the weights the timed steps'
    STDP updates reached (the trained regime the bench measures)."""
    import oracle
    from spyker_b200 import synth
    from tests.golden.make_golden import dog_kernel

    kind = "reference" if oracle.available("reference") else "port"
    o = oracle.get(kind)
    imgs = synth.strokes(n, seed=7)
    w1, w2 = weights
    net = Network(spyker, torch, dev, precision)
    net.conv1.kernel.copy_(torch.from_numpy(w1))
    net.conv2.kernel.copy_(torch.from_numpy(w2))
    x = torch.from_numpy(imgs).to(dev).float().div_(255.0)[:, None]
    codes = spyker.code(net.dog(x), T)
    s1, _, p1 = net._layer(net.conv1, codes, 15.0, 3, 5, 2)
    s2, _, _ = net._layer(net.conv2, p1, 10.0, 1, 8, 14)
    g1, g2 = s1.cpu().numpy(), s2.cpu().numpy()

    ref_codes = o.rank_code(o.filter("dog", imgs.astype(np.float32)[:, None] / np.float32(255), dog_kernel(o),
                                     (3, 3, 3, 3)), T)
    r1 = o.fire(o.inhibit(o.threshold(o.conv(ref_codes, w1, (1, 1), (2, 2, 2, 2)), 15.0)))
    r2 = o.fire(o.inhibit(o.threshold(o.conv(o.pool(r1, (2, 2)), w2, (1, 1), (2, 2, 2, 2)), 10.0)))
    return {"layer1_pct": 100.0 * float(np.mean(g1 == r1)), "layer2_pct": 100.0 * float(np.mean(g2 == r2)),
            "images": n, "oracle": f"{kind} (FP64 convolution)", "weights": "after the timed steps"}


# ----------------------------------------------------------------------------
# CPU reference arm (the reference's own CPU backend)
# ----------------------------------------------------------------------------
def reference_step(o, torch, imgs, w1, w2, dk, ops=None):
    """The same pipeline with the reference's CPU code (oracle/_ref) and the
    oneDNN convolution its CPU backend uses (through torch), in place.  With
    a dict ``ops``, each op's wall time (s) is added under its name."""
    clock = [time.perf_counter()]

    def lap(name):
        if ops is not None:
            now = time.perf_counter()
            ops[name] = ops.get(name, 0.0) + now - clock[0]
            clock[0] = now

    x = imgs.astype(np.float32) / np.float32(255)
    dog = o.filter("dog", x[:, None], dk, (3, 3, 3, 3))
    lap("dog")
    codes = o.rank_code(dog, T)
    lap("code")
    b = codes.shape[0]
    f = torch.from_numpy(codes.reshape(b * T, 2, 28, 28).astype(np.float32))
    p1 = torch.nn.functional.conv2d(f, torch.from_numpy(w1), padding=2).numpy().reshape(b, T, 30, 28, 28)
    lap("conv1")
    inh1 = o.inhibit(o.threshold(p1, 15.0))
    lap("threshold+inhibit1")
    s1 = o.fire(inh1)
    lap("fire1")
    win, cnt = o.convwta(inh1, (3, 3), 5)
    lap("convwta1")
    w1[:] = o.convstdp(codes, w1, s1, [(0.004, -0.003, 1, 0, 1)], win, cnt, (1, 1), (2, 2, 2, 2))
    lap("stdp1")
    q = o.pool(s1, (2, 2))
    lap("pool1")
    f2 = torch.from_numpy(q.reshape(b * T, 30, 14, 14).astype(np.float32))
    p2 = torch.nn.functional.conv2d(f2, torch.from_numpy(w2), padding=2).numpy().reshape(b, T, 100, 14, 14)
    lap("conv2")
    inh2 = o.inhibit(o.threshold(p2, 10.0))
    lap("threshold+inhibit2")
    s2 = o.fire(inh2)
    lap("fire2")
    win, cnt = o.convwta(inh2, (1, 1), 8)
    lap("convwta2")
    w2[:] = o.convstdp(q, w2, s2, [(0.004, -0.003, 1, 0, 1)], win, cnt, (1, 1), (2, 2, 2, 2))
    lap("stdp2")
    out = o.pool(s2, (14, 14))
    lap("pool2")
    return out


def load_synth():
    """The synthetic-data module by file path: importing it through the
    package would load the GPU library into the CPU-only reference arm."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("spyker_synth", os.path.join(ROOT, "spyker_b200", "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), recorded beside each CPU
    baseline together with the thread count it ran with."""
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _ref_setup():
    import torch

    import oracle
    from tests.golden.make_golden import dog_kernel

    synth = load_synth()

    kind = "reference" if oracle.available("reference") else "port"
    o = oracle.get(kind)
    torch.set_num_threads(os.cpu_count() or 1)
    return o, kind, torch, synth, dog_kernel(o)


def cpu_baseline(seconds: float) -> dict:
    o, kind, torch, synth, dk = _ref_setup()
    imgs = synth.strokes(64, seed=5)
    w1, w2 = synth.conv_weights(30, 2, 5, seed=1), synth.conv_weights(100, 30, 5, seed=2)
    reference_step(o, torch, imgs, w1, w2, dk)
    n, t0, ops = 0, time.perf_counter(), {}
    while time.perf_counter() - t0 < seconds:
        reference_step(o, torch, imgs, w1, w2, dk, ops)
        n += 64
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "images/s", "cores": torch.get_num_threads(), "kind": kind, "cpu": cpu_model(),
            "sample": f"{n} images in batches of 64 through the same 2-layer pipeline, {dt:.1f} s",
            "ops_us_per_image": {k: round(v / n * 1e6, 2) for k, v in ops.items()}}


def reference_arm(args, rank, world):
    """The reference's own CPU implementation on the host cores: a bounded
    sample of each step's batch (the first `sample` of its 4096 images).  Every
    op of the CPU path loops over the samples and its STDP scan walks the
    winners one by one, so its images/s does not depend on the batch size."""
    if rank != 0:
        return
    o, kind, torch, synth, dk = _ref_setup()
    sample = min(1024, args.batch)
    imgs = synth.strokes(args.batch, seed=100)[:sample]
    w1, w2 = synth.conv_weights(30, 2, 5, seed=1), synth.conv_weights(100, 30, 5, seed=2)
    for _ in range(args.warmup):
        reference_step(o, torch, imgs, w1, w2, dk)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        reference_step(o, torch, imgs, w1, w2, dk)
    dt = (time.perf_counter() - t0) / args.steps
    v = sample / dt
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "images/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded stroke images, MNIST geometry)",
        "config": headline_config(args.batch, world, args.mode),
        "cpu_baseline": {"value": v, "unit": "images/s", "cores": torch.get_num_threads(), "kind": kind, "cpu": cpu_model(),
                         "sample": f"{sample} of each step's {args.batch} images per timed step (the CPU path's "
                                   f"cost is per image), reference CPU backend + oneDNN convolution via torch"},
        "e2e": {"value": v, "unit": "images/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# ----------------------------------------------------------------------------
# One-layer STDP on 64 images (--workload config0)
# ----------------------------------------------------------------------------
CFG0_WORKLOAD = ("one-layer-stdp: 64 x 28x28 strokes, T=15, DoG 2x7x7 -> conv 30x5x5 th15 -> inhibit -> "
                 "convwta r3k5 -> fire -> STDP(0.004, -0.003) -> pool 2")


def config0_codes(o, imgs, dk):
    x = imgs.astype(np.float32) / np.float32(255)
    return o.rank_code(o.filter("dog", x[:, None], dk, (3, 3, 3, 3)), T)


def config0_ref_layer(o, torch, codes, w1):
    """The reference's CPU path of the one-layer pipeline after the rank code
    (the first layer of :func:`reference_step`), weights updated in place;
    returns the spikes and the pooled spikes."""
    b = codes.shape[0]
    f = torch.from_numpy(codes.reshape(b * T, 2, 28, 28).astype(np.float32))
    p1 = torch.nn.functional.conv2d(f, torch.from_numpy(w1), padding=2).numpy().reshape(b, T, 30, 28, 28)
    inh1 = o.inhibit(o.threshold(p1, 15.0))
    s1 = o.fire(inh1)
    win, cnt = o.convwta(inh1, (3, 3), 5)
    w1[:] = o.convstdp(codes, w1, s1, [(0.004, -0.003, 1, 0, 1)], win, cnt, (1, 1), (2, 2, 2, 2))
    return s1, o.pool(s1, (2, 2))


def config0_ref_step(o, torch, imgs, w1, dk):
    """The whole one-layer step on the reference's CPU path."""
    return config0_ref_layer(o, torch, config0_codes(o, imgs, dk), w1)[1]


def config0_arm(args, rank, world):
    """The small one-layer training step: 64 images through DoG, rank code
    and the fused conv1 layer, its STDP update and the pool, as one captured
    CUDA graph (the step is a few dozen microseconds of launches); weights
    carried from step to step.  Spikes, winners and weights after the timed
    steps are compared with the reference's CPU path run on the same images
    for the same number of steps."""
    if rank != 0:
        return
    import torch

    import spyker_b200 as spyker
    from spyker_b200 import synth

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    batch = args.batch if args.batch != BATCH else 64
    imgs = synth.strokes(batch, seed=0)
    host = torch.from_numpy(imgs).pin_memory()
    static_u8 = host.to(dev)
    dog = spyker.DoG(3, [spyker.DoGFilter(1, 2), spyker.DoGFilter(2, 1)], pad=3, device=dev)
    conv = spyker.Conv(2, 30, 5, pad=2, device=dev)
    w0 = synth.conv_weights(30, 2, 5, seed=1)
    conv.kernel.copy_(torch.from_numpy(w0))
    conv.stdpconfig = [spyker.STDPConfig(0.004, -0.003)]
    conv.precision = args.precision

    codes_gpu = spyker.code(dog(static_u8.float().div_(255.0)[:, None]), T).cpu().numpy()

    def step():
        codes = spyker.code(dog(static_u8.float().div_(255.0)[:, None]), T)
        spk, win, pooled = spyker.conv_fire_wta(codes, conv, 15.0, 3, 5, pool=2)
        conv.stdp(codes, win, spk)
        return spk, pooled

    step()
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    l0 = spyker._lib.lib.spk_launch_count()
    with torch.cuda.graph(graph):
        spk_g, pooled_g = step()
    launches = spyker._lib.lib.spk_launch_count() - l0
    # parity run: restart from the initial weights, warm-up + timed steps
    # replay the graph, the reference repeats the same number of steps
    conv.kernel.copy_(torch.from_numpy(w0))
    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(dev.index) as clk:
        a.record()
        for _ in range(args.steps):
            graph.replay()
        b.record()
        torch.cuda.synchronize()
    ms = a.elapsed_time(b) / args.steps
    w_gpu = conv.kernel.cpu().numpy().copy()
    spk_last = spk_g.cpu().numpy().copy()
    # end to end: pinned host images -> graph input, replay, pooled map back
    out = torch.empty(pooled_g.shape, dtype=pooled_g.dtype).pin_memory()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        static_u8.copy_(host, non_blocking=True)
        graph.replay()
        out.copy_(pooled_g, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    del graph
    o, kind, torch_, _, dk = _ref_setup()
    steps = args.warmup + args.steps
    # timed: the reference's whole step (its own rank code included)
    w_ref = w0.copy()
    t0 = time.perf_counter()
    for _ in range(steps):
        config0_ref_step(o, torch_, imgs, w_ref, dk)
    ref_s = (time.perf_counter() - t0) / steps
    # parity: the reference's layer and STDP on the GPU's rank code, the
    # same number of steps (the rank codes differ only where equal filter
    # values straddle a time-bin boundary: the reference sorts unstably)
    codes_ref = config0_codes(o, imgs, dk)
    w_par = w0.copy()
    for _ in range(steps):
        s_ref, _ = config0_ref_layer(o, torch_, codes_gpu, w_par)
    rel = float(np.max(np.abs(w_gpu.astype(np.float64) - w_par) / np.maximum(np.abs(w_par), 1e-30)))
    rel_own = float(np.max(np.abs(w_gpu.astype(np.float64) - w_ref) / np.maximum(np.abs(w_ref), 1e-30)))
    flops = 2 * T * 784 * 30 * 50
    peak, peak_source = bf16_peak()
    layer_ms = ms  # the whole step bounds the fused layer's time from above
    print(json.dumps({
        "metric": "images/s (one-layer STDP train + fwd, 64 images) on 1 B200; spike match %",
        "value": batch / (ms * 1e-3), "unit": "images/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": path_dtype(args.precision)[0], "arithmetic": path_dtype(args.precision)[1],
        "data": "synthetic (seeded stroke images, MNIST geometry)",
        "config": {"workload": CFG0_WORKLOAD.replace("64 x", f"{batch} x"), "global_batch": batch, "seq_len": T,
                   "parallelism": "replicas1", "conv_precision": args.precision,
                   "l2": "inputs smaller than L2 (the reference's small CPU case): the step's tensors stay in L2"},
        "e2e": {"value": batch / (e2e_ms * 1e-3), "unit": "images/s", "h2d_bytes_per_step": int(host.numel()),
                "d2h_bytes_per_step": int(out.numel() * out.element_size())},
        "gpu_launches": int(launches), "cuda_graph": True,
        "roofline": {"bound": "tensor", "kernel": "whole step (launch-latency bound at 64 images); algorithmic conv "
                                                  "FLOPs 35.3 MFLOP/img",
                     "achieved": flops * batch / (layer_ms * 1e-3) / 1e12, "peak": peak, "unit": "TFLOP/s",
                     "frac": flops * batch / (layer_ms * 1e-3) / 1e12 / peak, "traffic": None,
                     "peak_source": peak_source},
        "spike_match_vs_reference_pct": 100.0 * float(np.mean(spk_last == s_ref)),
        "weights_max_rel_diff_vs_reference": rel,
        "parity_note": f"after {steps} training steps; the reference's layer and STDP run on the GPU's rank code",
        "rank_code_match_vs_reference_pct": 100.0 * float(np.mean(codes_gpu == codes_ref)),
        "weights_max_rel_diff_vs_reference_own_code": rel_own,
        "cpu_baseline": {"value": batch / ref_s, "unit": "images/s", "cores": torch_.get_num_threads(), "kind": kind, "cpu": cpu_model(),
                         "sample": f"{steps} steps of the same {batch} images, reference CPU backend + oneDNN "
                                   f"convolution via torch"},
        "clocks": clk.summary(),
    }), flush=True)


# ----------------------------------------------------------------------------
# Large-image forward feature extraction (--workload gabor256)
# ----------------------------------------------------------------------------
GABOR_WORKLOAD = ("gabor256-forward: 256 x 256x256 textures, Gabor 4 orientations x 2 wavelengths 11x11, T=30, "
                  "conv1 64x7x7 th20 + inhibit + pool 2, conv2 256x5x5 th12 + inhibit + pool 2")


class GaborNet:
    def __init__(self, spyker, torch, dev, precision):
        from spyker_b200 import synth

        self.sp = spyker
        filters = [spyker.GaborFilter(2.5, th, 0.5, lam, 0.0) for th in (0, 45, 90, 135) for lam in (5.0, 10.0)]
        self.gabor = spyker.Gabor(5, filters, pad=5, device=dev)
        self.conv1 = spyker.Conv(8, 64, 7, pad=3, device=dev)
        self.conv2 = spyker.Conv(64, 256, 5, pad=2, device=dev)
        self.conv1.kernel.copy_(torch.from_numpy(synth.conv_weights(64, 8, 7, seed=11)))
        self.conv2.kernel.copy_(torch.from_numpy(synth.conv_weights(256, 64, 5, seed=12)))
        self.conv1.precision = self.conv2.precision = precision

    def step(self, images):
        sp = self.sp
        codes = sp.code(self.gabor(images), 30)
        _, _, p1 = sp.conv_fire_wta(codes, self.conv1, 20.0, 0, 0, pool=2)
        _, _, p2 = sp.conv_fire_wta(p1, self.conv2, 12.0, 0, 0, pool=2)
        return p2


def gabor_arm(args, rank, world):
    """Large-image forward pass (no STDP): the fused layers against the FP32
    op-by-op path and against the oracle's FP64 pipeline, conv1 potential
    errors against FP64 on the same GPU, and the reference's CPU path."""
    import torch

    import spyker_b200 as spyker
    from spyker_b200 import synth

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    # several GPUs: replicas, each rank its own images (no exchange)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    batch = args.batch if args.batch != BATCH else 256
    # the fused layers take the exact search path (non-negative weights) at
    # either split precision; the precision names the op-by-op potentials
    prec = args.precision
    host = torch.from_numpy(synth.textures(batch, seed=2 + rank)).pin_memory()
    imgs = host.to(dev)[:, None]
    net = GaborNet(spyker, torch, dev, prec)
    for _ in range(args.warmup):
        net.step(imgs)
    barrier()
    spyker._lib.lib.spk_recheck_count(1)
    spyker._lib.lib.spk_recompute_count(1)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(dev.index) as clk:
        barrier()
        a.record()
        for _ in range(args.steps):
            feats = net.step(imgs)
        b.record()
        barrier()
    ms = a.elapsed_time(b) / args.steps
    rechecks = spyker._lib.lib.spk_recheck_count(1) / args.steps
    recomputes = spyker._lib.lib.spk_recompute_count(1) / args.steps
    del feats
    # end to end: pinned host images -> first-spike maps of the features on the host
    # (the features land in a pinned host buffer: a pageable copy of 268 MB
    # per step would time the host's page faults)
    g = spyker.gather(net.step(host.to(dev, non_blocking=True)[:, None]))
    out = torch.empty(g.shape, dtype=g.dtype).pin_memory()
    del g
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record()
    for _ in range(args.steps):
        out.copy_(spyker.gather(net.step(host.to(dev, non_blocking=True)[:, None])), non_blocking=True)
    e1.record()
    barrier()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    t_max = torch.tensor([ms, e2e_ms], device=dev)
    if dist is not None:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
        dist.destroy_process_group()
    ms, e2e_ms = float(t_max[0]), float(t_max[1])
    if rank != 0:
        return  # the comparisons and the CPU leg run on rank 0 only
    # FP32 op-by-op path and potential errors on a sub-batch
    sub = min(4, batch)
    ref = GaborNet(spyker, torch, dev, "fp32")
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ref.step(imgs[:sub])
    torch.cuda.synchronize()
    f0.record()
    want = ref.step(imgs[:sub])
    f1.record()
    torch.cuda.synchronize()
    fp32_ms = f0.elapsed_time(f1)
    got = net.step(imgs[:sub])
    match = float((got == want).float().mean().item()) * 100
    # against the oracle's FP64 pipeline on a 64x64 texture of the same
    # generator (at 256x256 the oracle's convolutions take minutes)
    oracle_match = gabor_oracle_match(spyker, torch, dev, net, prec)
    codes = spyker.code(net.gabor(imgs[:1]), 30)
    pot = spyker.conv(codes, net.conv1.kernel, 1, 3, prec)
    x64 = codes[0].double()
    pot64 = torch.nn.functional.conv2d(x64, net.conv1.kernel.double(), padding=3)
    rel = float(((pot[0].double() - pot64).abs() / pot64.abs().clamp_min(1e-30)).max().item())
    c1 = 2 * 30 * 256 * 256 * 64 * 8 * 49
    c2 = 2 * 30 * 128 * 128 * 256 * 64 * 25
    peak, peak_source = bf16_peak()
    achieved = (c1 + c2) * batch / (ms * 1e-3) / 1e12
    print(json.dumps({
        "metric": "images/s (forward feature extraction), tensor-core path vs FP32 on 1 B200; spike match %",
        "value": batch * world / (ms * 1e-3), "unit": "images/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": path_dtype(prec)[0], "arithmetic": path_dtype(prec)[1],
        "data": "synthetic (seeded 1/f textures + Gaussian blobs, 256x256)",
        "config": {"workload": GABOR_WORKLOAD.replace("256 x", f"{batch} x"), "global_batch": batch * world,
                   "seq_len": 30, "parallelism": f"replicas{world}", "conv_precision": prec,
                   "l2": "inputs larger than L2: the layer-1 spikes are 128 MB per image"},
        "e2e": {"value": batch * world / (e2e_ms * 1e-3), "unit": "images/s",
                "h2d_bytes_per_step": int(host.numel() * 4) * world,
                "d2h_bytes_per_step": int(out.numel() * out.element_size()) * world},
        "roofline": {"bound": "tensor", "kernel": "both fused layers (algorithmic conv FLOPs)", "achieved": achieved,
                     "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "peak_source": peak_source},
        "fp32_path": {"value": sub / (fp32_ms * 1e-3), "unit": "images/s", "sample": f"{sub} images"},
        "feature_match_vs_fp32_pct": match,
        "spike_match_vs_oracle": oracle_match,
        "conv1_potential_max_rel_error_vs_fp64": rel,
        "rows_redecided_exactly_per_step": rechecks,
        "rows_recomputed_per_step": recomputes,
        "cpu_baseline": gabor_cpu_baseline(args.cpu_seconds, net) if not args.no_cpu_baseline else None,
        "clocks": clk.summary(),
    }), flush=True)


def gabor_oracle_match(spyker, torch, dev, net, prec, size=64):
    """Both layers' spikes and the pooled features of the fused GPU layers
    against the oracle's FP64 pipeline on one seeded texture."""
    import oracle
    from spyker_b200 import synth

    kind = "reference" if oracle.available("reference") else "port"
    o = oracle.get(kind)
    img = synth.textures(1, seed=9, size=size)
    x = torch.from_numpy(img).to(dev)[:, None]
    codes = spyker.code(net.gabor(x), 30)
    s1, _, p1 = spyker.conv_fire_wta(codes, net.conv1, 20.0, 0, 0, pool=2)
    s2, _, p2 = spyker.conv_fire_wta(p1, net.conv2, 12.0, 0, 0, pool=2)
    hc = codes.cpu().numpy()
    w1, w2 = net.conv1.kernel.cpu().numpy(), net.conv2.kernel.cpu().numpy()
    r1 = o.fire(o.inhibit(o.threshold(o.conv(hc, w1, (1, 1), (3, 3, 3, 3)), 20.0)))
    q1 = o.pool(r1, (2, 2))
    r2 = o.fire(o.inhibit(o.threshold(o.conv(q1, w2, (1, 1), (2, 2, 2, 2)), 12.0)))
    q2 = o.pool(r2, (2, 2))
    return {"layer1_pct": 100.0 * float(np.mean(s1.cpu().numpy() == r1)),
            "layer2_pct": 100.0 * float(np.mean(s2.cpu().numpy() == r2)),
            "features_pct": 100.0 * float(np.mean(p2.cpu().numpy() == q2)),
            "sample": f"1 texture {size}x{size}", "oracle": f"{kind} (FP64 convolution)"}


def gabor_cpu_baseline(seconds: float, net) -> dict:
    """The reference's CPU implementation of the large-image forward pass
    (its Gabor filter, rank code, threshold / inhibit / fire / pool; oneDNN
    convolution through torch) on 256x256 textures, one image at a time for
    a bounded time, with the GPU network's kernels."""
    o, kind, torch, synth, _ = _ref_setup()
    gk = net.gabor.kernel.cpu().numpy()
    w1, w2 = net.conv1.kernel.cpu().numpy(), net.conv2.kernel.cpu().numpy()
    imgs = synth.textures(4, seed=3)
    _gabor_ref_step(o, torch, imgs[:1], gk, w1, w2)
    n, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds and n < 64:
        _gabor_ref_step(o, torch, imgs[n % 4:n % 4 + 1], gk, w1, w2)
        n += 1
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "images/s", "cores": torch.get_num_threads(), "kind": kind, "cpu": cpu_model(),
            "sample": f"{n} images of 256x256, one at a time, {dt:.1f} s"}


def _gabor_ref_step(o, torch, img, gk, w1, w2):
    x = o.filter("gabor", img[:, None], gk, (5, 5, 5, 5))
    codes = o.rank_code(x, 30)
    b = codes.shape[0]
    f = torch.from_numpy(codes.reshape(b * 30, 8, 256, 256).astype(np.float32))
    p1 = torch.nn.functional.conv2d(f, torch.from_numpy(w1), padding=3).numpy().reshape(b, 30, 64, 256, 256)
    q1 = o.pool(o.fire(o.inhibit(o.threshold(p1, 20.0))), (2, 2))
    del p1
    f2 = torch.from_numpy(q1.reshape(b * 30, 64, 128, 128).astype(np.float32))
    p2 = torch.nn.functional.conv2d(f2, torch.from_numpy(w2), padding=2).numpy().reshape(b, 30, 256, 128, 128)
    return o.pool(o.fire(o.inhibit(o.threshold(p2, 12.0))), (2, 2))


# ----------------------------------------------------------------------------
# Temporal backprop (--workload backprop)
# ----------------------------------------------------------------------------
BP_WORKLOAD = ("temporal-backprop: 256 x 28x28 labelled strokes (10 classes), T=64, conv 32x5x5 -> pool 2 -> "
               "conv 64x3x3 -> pool 2 -> fc 10, first-spike-time loss, SGD")


def backprop_arm(args, rank, world):
    """One training step = rank code -> 3 first-spike layers -> target-rule
    loss -> hand-written backward kernels (autograd) -> SGD update."""
    if rank != 0:
        return  # a one-GPU workload: under torchrun only rank 0 runs it
    import torch

    import spyker_b200 as spyker
    from spyker_b200 import synth, temporal

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    batch = args.batch if args.batch != BATCH else 256
    imgs, labels = synth.labelled_strokes(batch, seed=20 + rank)
    host = torch.from_numpy(imgs).pin_memory()
    x = host.to(dev).float().div_(255.0)[:, None]
    y = torch.from_numpy(labels).to(dev)
    net = temporal.TemporalNet(time=64, seed=4, device=dev, precision=args.precision)
    for _ in range(args.warmup):
        net.step(x, y)
    torch.cuda.synchronize()
    l0 = spyker._lib.lib.spk_launch_count()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(dev.index) as clk:
        torch.cuda.synchronize()
        a.record()
        for _ in range(args.steps):
            loss, t_out = net.step(x, y)
        b.record()
        torch.cuda.synchronize()
    ms = a.elapsed_time(b) / args.steps
    launches = (spyker._lib.lib.spk_launch_count() - l0) // max(args.steps, 1)
    # forward / backward split of one step
    f0, f1, f2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    f0.record()
    t_fwd = net.forward(net.input_times(x))
    lo = net.loss(t_fwd, y)
    f1.record()
    torch.autograd.grad(lo, net.weights)
    f2.record()
    torch.cuda.synchronize()
    fwd_ms, bwd_ms = f0.elapsed_time(f1), f1.elapsed_time(f2)
    # end to end: pinned host images -> loss in pinned host memory (copied
    # back asynchronously every step; the timed region ends after the last)
    loss_bufs = [torch.empty((), dtype=torch.float64).pin_memory() for _ in range(2)]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for k in range(args.steps):
        xe = host.to(dev, non_blocking=True).float().div_(255.0)[:, None]
        loss_bufs[k % 2].copy_(net.step(xe, y)[0], non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    loss_host = loss_bufs[(args.steps - 1) % 2]
    fp32 = None
    if args.precision != "fp32" and not args.no_fp32_compare:
        ref = temporal.TemporalNet(time=64, seed=4, device=dev, precision="fp32")
        ref.step(x, y)
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record()
        ref.step(x, y)
        g1.record()
        torch.cuda.synchronize()
        fp32 = {"value": batch / (g0.elapsed_time(g1) * 1e-3), "unit": "images/s", "steps": 1}
    fwd_flops = 2 * 64 * (784 * 32 * 25 + 196 * 64 * 288 + 10 * 3136)
    peak, peak_source = bf16_peak()
    fwd_achieved = fwd_flops * batch / (fwd_ms * 1e-3) / 1e12
    line = {
        "metric": "images/s (temporal-backprop training step) on 1 B200",
        "value": batch / (ms * 1e-3), "unit": "images/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"fp32": "f32", "bf16x2": "bf16x2-split/f32-acc", "bf16x3": "bf16x3-split/f32-acc"}[args.precision]
        + " forward, f32/f64 backward",
        "data": "synthetic (seeded labelled stroke images, 10 classes)",
        "config": {"workload": BP_WORKLOAD.replace("256 x", f"{batch} x"), "global_batch": batch, "seq_len": 64,
                   "parallelism": "replicas1", "conv_precision": args.precision,
                   "l2": "inputs larger than L2: the layer-1 potentials are 1.6 GB per step"},
        "e2e": {"value": batch / (e2e_ms * 1e-3), "unit": "images/s", "h2d_bytes_per_step": int(host.numel()),
                "d2h_bytes_per_step": int(loss_host.numel() * loss_host.element_size())},
        "gpu_launches": int(launches),
        "kernels_ms": {"forward_and_loss": fwd_ms, "backward": bwd_ms},
        "roofline": {"bound": "tensor", "kernel": "forward: the 3 fused first-spike layers (dense T-step potentials "
                                                    "as algorithmic FLOPs, 0.54 GFLOP/img)",
                     "achieved": fwd_achieved, "peak": peak, "unit": "TFLOP/s", "frac": fwd_achieved / peak,
                     "traffic": None, "peak_source": peak_source},
        "loss": float(loss_host),
        "outputs_fired_pct": 100.0 * float((t_out < 64).float().mean()),
        "clocks": clk.summary(),
    }
    if fp32 is not None:
        line["fp32_path"] = fp32
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = backprop_cpu_baseline(args.cpu_seconds, net, imgs, labels)
    print(json.dumps(line), flush=True)


def backprop_cpu_baseline(seconds: float, net, imgs, labels) -> dict:
    """The training step on the host cores through the oracle's FP64 NumPy
    restatement (the reference has no conv backward: its temporal rule exists
    for fc layers only, cpu/backprop.cpp:105-160), two images at a time for a
    bounded time, with the GPU network's weights."""
    import torch

    import oracle
    from oracle import temporal as ot

    o = oracle.get("port")
    torch.set_num_threads(os.cpu_count() or 1)
    T, th, gamma = net.time, net.thresholds, net.gamma
    w1, w2, w3 = (w.detach().cpu().numpy().astype(np.float64) for w in net.weights)
    w3c = w3.reshape(w3.shape[0], -1, 1, 1)

    def step(x, y):
        codes = o.rank_code(x[:, None].astype(np.float32) / 255.0, T)
        t0 = (T - codes.astype(np.int64).sum(axis=1)).astype(np.float64)
        a1 = ot.conv_forward(t0, w1, th[0], T, (1, 1), (2, 2, 2, 2))
        p1 = ot.pool_forward(a1, (2, 2), time=T)
        a2 = ot.conv_forward(p1, w2, th[1], T, (1, 1), (1, 1, 1, 1))
        p2 = ot.pool_forward(a2, (2, 2), time=T)
        f = p2.reshape(p2.shape[0], -1, 1, 1)
        a3 = ot.conv_forward(f, w3c, th[2], T)
        g3 = -ot.target_rule(a3[:, :, 0, 0], y, T, gamma)[:, :, None, None]
        gf, _ = ot.conv_backward(f, w3c, a3, g3)
        gp2 = ot.pool_backward(a2, gf.reshape(p2.shape), (2, 2))
        gp1, _ = ot.conv_backward(p1, w2, a2, gp2, (1, 1), (1, 1, 1, 1))
        ga1 = ot.pool_backward(a1, gp1, (2, 2))
        ot.conv_backward(t0, w1, a1, ga1, (1, 1), (2, 2, 2, 2))

    step(imgs[:2], labels[:2])
    n, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds and n < 256:
        i = n % (imgs.shape[0] - 1)
        step(imgs[i:i + 2], labels[i:i + 2])
        n += 2
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "images/s", "cores": torch.get_num_threads(), "kind": "port", "cpu": cpu_model(),
            "sample": f"{n} images, two per step, forward + target rule + backward in FP64 NumPy, {dt:.1f} s"}


# ----------------------------------------------------------------------------
# Hyperparameter sweep (--workload sweep)
# ----------------------------------------------------------------------------
SWEEP_WORKLOAD = ("sweep: 32 independent 2-layer STDP networks x 512 stroke images of side 20/28/40/64, T=15, "
                  "conv1 30x5x5 + conv2 100x5x5, per-network threshold U[8,20] and a+ U[0.001,0.01], a- = -0.75 a+")


def sweep_arm(args, rank, world):
    """All networks' training step: per size and layer each network's
    single-network fused search call (``--sweep-path search``) or one
    multi-network fused launch with autotuned schedules (``dense``), and one
    multi-network STDP scan per layer, captured once as a CUDA graph and
    replayed.  Several
    GPUs: each rank trains its own 32 networks (seeds differ by rank), no
    exchange; time = max over ranks."""
    import torch

    import spyker_b200 as spyker
    from spyker_b200 import sweep

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    nets = 32
    images = 512 if args.batch == BATCH else args.batch
    sw = sweep.Sweep(nets=nets, images=images, seed=10 * rank, device=dev, precision=args.precision, tune=True,
                     path=args.sweep_path)
    sw.capture()
    for _ in range(max(args.warmup - 1, 0)):
        sw.replay()
    barrier()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(dev.index) as clk:
        barrier()
        a.record()
        for _ in range(args.steps):
            sw.replay()
        b.record()
        barrier()
    ms = a.elapsed_time(b) / args.steps
    # launches inside one graph (counted while capturing a second one)
    l1 = spyker._lib.lib.spk_launch_count()
    g2 = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g2):
        sw.step()
    launches = spyker._lib.lib.spk_launch_count() - l1
    del g2
    # eager step (no graph) for comparison
    e_a, e_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_a.record()
    sw.step()
    e_b.record()
    torch.cuda.synchronize()
    eager_ms = e_a.elapsed_time(e_b)
    # end to end: pinned host images into the graph's inputs, features back
    h2d = sum(int(g.host.numel()) for g in sw.groups)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record()
    for _ in range(args.steps):
        for g in sw.groups:
            g.images.copy_(g.host.to(dev, non_blocking=True).float().div_(255.0)[:, None])
        feats = [f.cpu() for f in sw.replay()]
    e1.record()
    barrier()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    t_max = torch.tensor([ms, e2e_ms], device=dev)
    if dist is not None:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
        dist.destroy_process_group()
    ms, e2e_ms = float(t_max[0]), float(t_max[1])
    if rank != 0:
        return
    n_img = sw.images_per_step
    flops = sum(
        sum(len(g.per_net[n][1]) for n in range(nets)) * 2 * 15 * (g.size ** 2 * 30 * 50 + (g.size // 2) ** 2 * 100 * 750)
        for g in sw.groups)
    peak, peak_source = bf16_peak()
    achieved = flops / (ms * 1e-3) / 1e12
    print(json.dumps({
        "metric": "images/s (32-network STDP sweep, train + fwd) on 1 B200",
        "value": n_img * world / (ms * 1e-3), "unit": "images/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"fp32": "f32", "bf16x2": "bf16x2-split/f32-acc", "bf16x3": "bf16x3-split/f32-acc"}[args.precision],
        "data": "synthetic (seeded stroke images of 4 sizes)",
        "config": {"workload": SWEEP_WORKLOAD, "global_batch": n_img * world, "seq_len": 15,
                   "parallelism": f"replicas{world}",
                   "networks": nets, "padded_samples": sw.total, "cuda_graph": True, "path": sw.path,
                   "schedules": {f"{sw.groups[g].size}px/layer{l + 1}": list(v) for (g, l), v in sw.schedules.items()},
                   "l2": "inputs larger than L2: 2.0 GB of layer-1 spikes per step"},
        "e2e": {"value": n_img * world / (e2e_ms * 1e-3), "unit": "images/s", "h2d_bytes_per_step": h2d * world,
                "d2h_bytes_per_step": int(sum(f.numel() for f in feats)) * world},
        "gpu_launches": int(launches),
        "eager_step_ms": eager_ms,
        "roofline": {"bound": "tensor", "kernel": "all fused layers (algorithmic conv FLOPs of the real images"
                               + ("; dense-equivalent: the search evaluates fewer rows)" if sw.path == "search" else ")"),
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "peak_source": peak_source},
        "clocks": clk.summary(),
    }), flush=True)


# ----------------------------------------------------------------------------
# Event-list (sparse) input path (--workload sparse)
# ----------------------------------------------------------------------------
SPARSE_WORKLOAD = ("sparse-2layer-stdp: 4096 x [2, 28, 28] event lists at 1/2/5 % density (seeded first-spike "
                   "times), T=15, conv1 30x5x5 -> inhibit -> convwta(r3,k5) -> STDP -> pool 2 -> conv2 100x5x5 -> "
                   "inhibit -> convwta(r1,k8) -> STDP")
SPARSE_DENSITIES = (0.01, 0.02, 0.05)


def _sparse_thresholds(d):
    # the dense rank code of the stroke images fires about 20 % of its
    # inputs: conv1's threshold follows the input density (at least one
    # weight); conv2 sees the pooled layer-1 events and keeps its 10
    return max(1.0, 15.0 * d / 0.2), 10.0


def _sparse_times(n, d, seed):
    rng = np.random.default_rng(seed)
    t = rng.integers(0, T, size=(n, 2, 28, 28))
    return np.where(rng.random((n, 2, 28, 28)) < d, t, T).astype(np.float32)


def sparse_arm(args, rank, world):
    """The 2-layer STDP step of the Kheradpisheh example on event lists
    (Sparse::conv / inhibit / convwta / STDP / pool) at 1, 2 and 5 % input
    density; the reference's own CPU sparse backend times a sample."""
    if rank != 0:
        return  # a one-GPU workload: under torchrun only rank 0 runs it
    import torch

    import spyker_b200 as spyker
    from spyker_b200 import sparse, synth

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    batch = args.batch
    per_density = {}
    launches = 0
    for d in SPARSE_DENSITIES:
        th1, th2 = _sparse_thresholds(d)
        times = torch.from_numpy(_sparse_times(batch, d, 7 + rank)).to(dev)
        dense = spyker.scatter(times.reshape(batch, -1), T).view(batch, T, 2, 28, 28)
        ev = spyker.SparseTensor(dense, 0.0)
        del dense
        c1, c2 = spyker.Conv(2, 30, 5, pad=2, device=dev), spyker.Conv(30, 100, 5, pad=2, device=dev)
        c1.kernel.copy_(torch.from_numpy(synth.conv_weights(30, 2, 5, seed=1)))
        c2.kernel.copy_(torch.from_numpy(synth.conv_weights(100, 30, 5, seed=2)))
        for c in (c1, c2):
            c.stdpconfig = [spyker.STDPConfig(0.004, -0.003)]

        def step():
            o1 = sparse.inhibit(sparse.conv(ev, c1.kernel, th1, 1, 2))
            w1 = sparse.convwta(o1, 3, 5)
            sparse.stdp(c1, ev, w1)
            q = sparse.pool(o1, 2)
            o2 = sparse.inhibit(sparse.conv(q, c2.kernel, th2, 1, 2))
            w2 = sparse.convwta(o2, 1, 8)
            sparse.stdp(c2, q, w2)
            return o1, o2

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        l0 = spyker._lib.lib.spk_launch_count()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.steps):
            o1, o2 = step()
        b.record()
        torch.cuda.synchronize()
        launches = (spyker._lib.lib.spk_launch_count() - l0) // max(args.steps, 1)
        ms = a.elapsed_time(b) / args.steps
        per_density[f"{int(d * 100)}%"] = {
            "images_per_s": batch / (ms * 1e-3), "ms_per_step": ms, "thresholds": [th1, th2],
            "input_events": int(ev.numel), "layer1_events": int(o1.numel), "layer2_events": int(o2.numel),
            "input_density_measured": float(ev.numel) / (batch * 2 * 28 * 28)}
    head = per_density["2%"]
    line = {
        "metric": "images/s (event-list STDP train + fwd) at 1-5 % input density on 1 B200",
        "value": head["images_per_s"], "unit": "images/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (event lists; F32 STDP rule of sparse/stdp.cpp)",
        "data": "synthetic (seeded first-spike times at the stated density)",
        "config": {"workload": SPARSE_WORKLOAD.replace("4096 x", f"{batch} x"), "global_batch": batch,
                   "seq_len": T, "parallelism": "replicas1", "headline_density": "2%"},
        "per_density": per_density,
        "gpu_launches": int(launches),
    }
    if not args.no_cpu_baseline:
        import oracle

        kind = "reference" if oracle.available("reference") else "port"
        o = oracle.get(kind)
        n = 64
        dense = (np.arange(T)[None, :, None, None, None] >= _sparse_times(n, 0.02, 7)[:, None]).astype(np.uint8)
        ev = o.sparse_from_dense(dense, 0.0)
        w1, w2 = synth.conv_weights(30, 2, 5, seed=1), synth.conv_weights(100, 30, 5, seed=2)
        th1, th2 = _sparse_thresholds(0.02)
        cfg = [(0.004, -0.003, 1.0, 0.0, 1.0)]

        def ref_step(w1, w2):
            o1, s1 = o.sparse_conv(ev, (n, T, 2, 28, 28), w1, th1, (2, 2, 2, 2))
            i1 = o.sparse_inhibit(o1, s1)
            win, cnt = o.sparse_convwta(i1, s1, (3, 3), 5)
            w1 = o.sparse_stdp(ev, (n, T, 2, 28, 28), w1, cfg, win, cnt, (2, 2, 2, 2))
            q, sq = o.sparse_pool(i1, s1, (2, 2))
            o2, s2 = o.sparse_conv(q, sq, w2, th2, (2, 2, 2, 2))
            i2 = o.sparse_inhibit(o2, s2)
            win, cnt = o.sparse_convwta(i2, s2, (1, 1), 8)
            w2 = o.sparse_stdp(q, sq, w2, cfg, win, cnt, (2, 2, 2, 2))
            return w1, w2

        ref_step(w1, w2)
        t0, k = time.perf_counter(), 0
        while time.perf_counter() - t0 < min(args.cpu_seconds, 10.0):
            ref_step(w1, w2)
            k += n
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": k / dt, "unit": "images/s", "cores": os.cpu_count() or 1, "kind": kind, "cpu": cpu_model(),
                                "sample": f"{k} images at 2 % density in batches of {n} (reference sparse backend, "
                                          f"its OpenMP threads), {dt:.1f} s"}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------
# R-STDP (--workload rstdp)
# ----------------------------------------------------------------------------
RSTDP_WORKLOAD = ("rstdp-mozafari: 1024 x 28x28 labelled strokes, DoG 6 filters -> T=15 -> conv1 30x5x5 -> pool 2 -> "
                  "conv2 250x3x3 -> pool 3 -> conv3 200x5x5 infinite readout, reward/punish STDP (layer-3 step)")


def rstdp_arm(args, rank, world):
    """The layer-3 R-STDP training step of the Mozafari network."""
    if rank != 0:
        return  # a one-GPU workload: under torchrun only rank 0 runs it
    import torch

    import spyker_b200 as spyker
    from spyker_b200 import rstdp, synth

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    batch = args.batch if args.batch != BATCH else 1024
    imgs, labels = synth.labelled_strokes(batch, seed=30)
    host = torch.from_numpy(imgs).pin_memory()
    y = torch.from_numpy(labels).to(dev)
    net = rstdp.MozafariNetwork(device=dev, precision=args.precision, seed=1)
    x = net.transform(host.to(dev).float().div_(255.0)[:, None])
    for _ in range(args.warmup):
        net.train_layer3(x, y)
    torch.cuda.synchronize()
    l0 = spyker._lib.lib.spk_launch_count()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(dev.index) as clk:
        torch.cuda.synchronize()
        a.record()
        for _ in range(args.steps):
            pred = net.train_layer3(x, y)
        b.record()
        torch.cuda.synchronize()
    ms = a.elapsed_time(b) / args.steps
    launches = (spyker._lib.lib.spk_launch_count() - l0) // max(args.steps, 1)
    # end to end: pinned images -> transform -> step -> labels read back
    bufs = [torch.empty(batch, dtype=torch.int64).pin_memory() for _ in range(2)]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for k in range(args.steps):
        xe = net.transform(host.to(dev, non_blocking=True).float().div_(255.0)[:, None])
        bufs[k % 2].copy_(net.train_layer3(xe, y), non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    perf = rstdp.accuracy(pred.cpu(), torch.from_numpy(labels))
    print(json.dumps({
        "metric": "images/s (R-STDP layer-3 training step) on 1 B200",
        "value": batch / (ms * 1e-3), "unit": "images/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"fp32": "f32", "bf16x2": "bf16x2-split/f32-acc", "bf16x3": "bf16x3-split/f32-acc"}[args.precision],
        "data": "synthetic (seeded labelled stroke images, 10 classes)",
        "config": {"workload": RSTDP_WORKLOAD.replace("1024 x", f"{batch} x"), "global_batch": batch, "seq_len": 15,
                   "parallelism": "replicas1", "conv_precision": args.precision,
                   "l2": "inputs larger than L2: the conv2 potentials are 1.5 GB per 1024 images"},
        "e2e": {"value": batch / (e2e_ms * 1e-3), "unit": "images/s", "h2d_bytes_per_step": int(host.numel()),
                "d2h_bytes_per_step": batch * 8},
        "gpu_launches": int(launches),
        "labels_right_wrong_silent": [int(v) for v in perf[:3]],
        "clocks": clk.summary(),
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default=os.environ.get("SPYKER_BENCH_PRECISION", "bf16x3"),
                    choices=["fp32", "bf16x2", "bf16x3"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--batch", type=int, default=BATCH, help="images per GPU per step (small cases for profiling)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp32-compare", action="store_true")
    ap.add_argument("--no-spike-match", action="store_true")
    ap.add_argument("--trajectory", type=int, default=0,
                    help="after the warm-up, this many synchronised steps recording each layer's exact re-decisions")
    ap.add_argument("--dump-weights", default="", help="save the trained kernels to this .npz")
    ap.add_argument("--mode", default="replicas", choices=["replicas", "dp"],
                    help="several GPUs: independent networks (replicas, the default) or one network trained data "
                         "parallel (dp: one all-gather of the winners per layer and step)")
    ap.add_argument("--sweep-path", default="search", choices=["dense", "search"],
                    help="sweep workload: one multi-network fused launch per size and layer (dense), or the "
                         "single-network first-crossing search per network (search)")
    ap.add_argument("--graph", action="store_true",
                    help="run the headline step as one captured CUDA graph (measured at the eager step's time: "
                         "the kernels dominate and the eager queue already hides the launches)")
    ap.add_argument("--workload", default="kheradpisheh", choices=["kheradpisheh", "config0", "gabor256", "backprop", "sweep", "sparse",
                                                                   "rstdp"],
                    help="kheradpisheh: the 2-layer STDP training step (the headline); config0: the one-layer "
                         "STDP step on 64 images against the reference's CPU path; gabor256: large-image "
                         "forward; backprop: temporal-backprop training of a 3-layer first-spike network; "
                         "sweep: 32 STDP networks on uneven image sizes in one CUDA graph; sparse: the event-list "
                         "path at 1-5 % input density; rstdp: the reward-modulated layer of the Mozafari network")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", args.gpus if args.impl == "reference" else 1))
    if args.impl == "reference":
        reference_arm(args, rank, world)
    elif args.workload == "config0":
        config0_arm(args, rank, world)
    elif args.workload == "gabor256":
        gabor_arm(args, rank, world)
    elif args.workload == "backprop":
        backprop_arm(args, rank, world)
    elif args.workload == "sweep":
        sweep_arm(args, rank, world)
    elif args.workload == "sparse":
        sparse_arm(args, rank, world)
    elif args.workload == "rstdp":
        rstdp_arm(args, rank, world)
    else:
        gpu_arm(args, rank, world)


if __name__ == "__main__":
    main()
