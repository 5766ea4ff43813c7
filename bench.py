#!/usr/bin/env python
"""Benchmark of the exact d3-force tick on the B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (a "step" = one tick): exact mode, n = 50,000 nodes at d3's
phyllotaxis start, m = 100,000 links drawn from d3's LCG (no self-loops),
forceManyBody(-30, theta 0.9) + forceLink(distance 30, default strength) +
forceCollide(radius 5) + forceCenter(0, 0); 1% of nodes moved onto exact copies
of other nodes' positions, 1% to offsets below 1e-12 from other nodes, 0.5%
pinned (fx, fy). Every tick is bit-identical to the CPU oracle (tests/).

`value` is device milliseconds per tick (CUDA events on the engine's stream),
with L2 flushed between ticks (the working set fits in L2). `e2e` is the same
metric through the public API (`Simulation.tick`), with the host-to-device copy
of the node state and the device-to-host read of the result in every step.
`--impl reference` times the reference algorithm's CPU restatement (the
oracle: the reference compiles only with zig, which this machine lacks) on all
host cores. Under torchrun (N > 1) each rank runs an independent replica
(the exact tick does not shard: ordered link / collide sums and one random
stream); rank 0 prints the line.
"""

import argparse
import hashlib
import importlib
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(n=50000, m=100000, collide_radius=5, coincident=0.01, near=0.01, pinned=0.005)
WORKLOAD_NAME = ("exact n=50000 m=100000 manyBody(-30,theta .9)+link(30)+collide(5)+center; "
                 "1% coincident, 1% offsets<1e-12, 0.5% pinned")
METRIC = "ms/tick: exact 50k bit-exact"
SCHEDULE_TICKS = 300  # the configuration's tick count (d3's default alpha schedule)
CHECK_TICK = 95  # 5 warm-up + 3 x 30 ticks: where the CPU protocol's state is compared
PHASES = ["mb_tree", "mb_accumulate", "mb_traverse", "link", "collide_tree", "collide_loop",
          "center", "integrate"]
SIDE_PHASES = {"center_sum_side_stream": 11}
# What the CPU baseline (the oracle) spreads over the host threads, as the
# reference's worker pool does; link and collide's node loop are serial in both.
THREADED = "tree keys, sort and emission jobs; many-body record pass"
# DRAM bytes (read + write) of one collide launch (k_collide_spec) on this
# workload, from an ncu capture of the 11th pass of a 15-tick schedule
# (profiles/k_collide_spec_exact_50k.md)
COLLIDE_DRAM_BYTES = 64813568 + 9635072


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fast", action="store_true", help="skip the fast-mode 1M measurement")
    ap.add_argument("--schedule", type=int, default=SCHEDULE_TICKS,
                    help="ticks of the exact schedule (300 for the configuration; fewer only "
                         "for profiling runs)")
    ap.add_argument("--only", choices=["fast", "learned", "batched"],
                    help="run only this fast-mode leg (no exact line; for profiling)")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def max_over_ranks(x, world):
    """The largest of x over all ranks of the process group (a replicated
    job's time is its slowest replica's); x itself with one rank."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def schedule_positions(warmup, steps, total=None, schedule=SCHEDULE_TICKS):
    """The K timed ticks, spread evenly over the C2 schedule after the W
    warm-up ticks: ticks W + ceil((k + 1) (T - W) / K), k = 0..K-1, where T
    is the schedule's 300 ticks (longer when W + K exceeds it). Returns
    (positions, T)."""
    total = total or max(schedule, warmup + steps)
    span = total - warmup
    pos = [warmup + -(-(k + 1) * span // steps) for k in range(steps)]
    return pos, total


def state_digest(nodes, lcg):
    """SHA-256 of x, y, vx, vy (f64 little-endian) and the LCG state."""
    import numpy as np

    h = hashlib.sha256()
    for f in ("x", "y", "vx", "vy"):
        h.update(np.ascontiguousarray(getattr(nodes, f), dtype="<f8").tobytes())
    h.update(int(lcg).to_bytes(4, "little"))
    return h.hexdigest()


def oracle_protocol(pkg, sc, threads, warmup=5, rounds=3, ticks=30, count_work=False):
    """The reference's timing protocol (bench/threads.js:24-35): `warmup`
    ticks, then the minimum over `rounds` rounds of `ticks` consecutive ticks,
    on the oracle (the reference algorithm restated in C) with `threads` host
    threads. Returns the ms/tick, the state digest after the last tick (tick
    warmup + rounds * ticks) and, with count_work, the exact many-body work
    (cells visited, accepted approximations, leaf point interactions) per tick
    over the last round."""
    import oracle

    core = oracle.load(pkg)
    nodes, sim = sc.setup_exact(pkg, core, **WORKLOAD)
    core.lib.oracle_set_threads(sim.ctx.h, threads)
    sim.tick(warmup)
    best = float("inf")
    work = None
    for r in range(rounds):
        if count_work and r == rounds - 1:
            core.lib.oracle_mb_stat(3)
        t0 = time.perf_counter()
        sim.tick(ticks)
        best = min(best, (time.perf_counter() - t0) * 1e3 / ticks)
    if count_work:
        work = {k: core.lib.oracle_mb_stat(i) / ticks for i, k in enumerate(("V", "A", "P"))}
    digest = state_digest(nodes, core.sim_get_lcg(sim.ctx.h))
    sim.close()
    return best, digest, work


class Clocks:
    """SM clocks and clock-event reasons sampled during the timed region: NVML
    every 5 ms from a thread (reads only), else nvidia-smi every 200 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown"}

    def __init__(self, device):
        self.proc = None
        self.thread = None
        self.samples, self.reason_bits, self.max_mhz = [], 0, None
        try:
            import threading
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(device)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self.stop_flag = threading.Event()

            def loop():
                while not self.stop_flag.is_set():
                    try:
                        self.samples.append(float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)))
                        self.reason_bits |= int(pynvml.nvmlDeviceGetCurrentClocksEventReasons(h))
                    except Exception:
                        pass
                    self.stop_flag.wait(0.005)
            self.thread = threading.Thread(target=loop, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(device), "--query-gpu=" + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join(timeout=5)
            if not self.samples:
                return None
            reasons = sorted(v for b, v in self.REASONS.items() if self.reason_bits & b)
            return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                    "reasons": reasons, "samples": len(self.samples), "source": "nvml 5 ms"}
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], None, set()
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                                "sw_power_cap"), f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi 200 ms"}


FAST_N = 1000000
FAST_ORDER, FAST_OPENING = 8, 1.5


def fast_layout(n=FAST_N, seed=1):
    """The fast-mode precision configuration: n nodes uniform in [0, 1e4)^2
    and m = 2n uniform random links without self-loops (seeded)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    xs = rng.random(n) * 1e4
    ys = rng.random(n) * 1e4
    src = rng.integers(0, n, 2 * n)
    tgt = (src + 1 + rng.integers(0, n - 1, 2 * n)) % n
    return xs, ys, src, tgt


def fast_sim(pkg, core, xs, ys, src, tgt, form, order=FAST_ORDER, opening=FAST_OPENING):
    nodes = pkg.Nodes(len(xs), x=xs, y=ys)
    sim = pkg.forceSimulation(nodes, core=core)
    sim.force("charge", pkg.forceManyBody())
    sim.force("link", pkg.forceLink(src, tgt))
    sim.force("center", pkg.forceCenter())
    sim.precision("fast", order=order, opening=opening, form=form)
    return nodes, sim


def fast_ticks(pkg, core, layout, form, flush_l2, steps=10, warmup=3):
    """Device ms per fast tick (manyBody + link + center) over `steps` ticks
    after `warmup`, L2 flushed before each; also the state digest after 3
    ticks of a fresh run (the bit-exactness check of the plain form)."""
    xs, ys, src, tgt = layout
    nodes, sim = fast_sim(pkg, core, xs, ys, src, tgt, form)
    sim.device_begin()
    for _ in range(warmup):
        flush_l2()
        sim.device_ticks(1)
    times = []
    for _ in range(steps):
        flush_l2()
        times.append(sim.device_ticks(1))
    sim.device_end()
    # the tensor-core form's last pass: M2L / P2P event times and work counts
    stats = {k: core.sim_stat(sim.ctx.h, 54 + i) for i, k in enumerate(
        ("m2l_ms", "near_ms", "m2l_tiles", "m2l_pairs", "p2p_pairs", "m2p_pairs", "p2l_pairs", "q",
         "prepare_ms", "lists_ms", "upward_ms", "p2l_ms", "down_ms", "network_ms", "many_body_ms",
         "far_ms"))}
    sim.close()
    return sum(times) / len(times), stats


def fast_digest(pkg, core, layout, form, ticks=3):
    xs, ys, src, tgt = layout
    nodes, sim = fast_sim(pkg, core, xs, ys, src, tgt, form)
    sim.tick(ticks)
    d = state_digest(nodes, core.sim_get_lcg(sim.ctx.h))
    sim.close()
    return d


def fast_rms(pkg, core, layout, form, targets=4096):
    """The many-body kick of one tick against the FP64 direct sum on
    `targets` seeded nodes (accuracy.py)."""
    import numpy as np
    acc = importlib.import_module("d3-force-wasm_b200.accuracy")
    xs, ys = layout[0], layout[1]
    kick, alpha = acc.many_body_kick(pkg, core, xs, ys, form=form, order=FAST_ORDER,
                                     opening=FAST_OPENING)
    tg = acc.sample_targets(xs, ys, targets)
    ref = acc.direct_kick(xs, ys, np.full(len(xs), -30.0 * alpha), tg)
    return acc.rms(kick, ref, tg)


def fast_roofline(st, rates):
    """The tensor-core form's two dominant kernels against their pipes.
    M2L: every 128-target tile runs, per vector slot (39 at opening 1.5), six
    tcgen05 MMAs of 128 x 32 x 16 (BF16x3 over K = 32: hi*hi, hi*lo, lo*hi),
    2 * 128 * 32 * 16 flops each; achieved = those flops / the M2L launch's
    event time, against the measured dense BF16 peak. The useful share: each
    real source-target pair needs 3 x (2q)^2 multiply-adds of the 32-wide
    padded rows. Near field: the P2P launch (it runs on a second stream
    beside M2L, P2L and the downward pass), about 10 FP32 flops per point
    pair (differences, the squared distance, one reciprocal square root, two
    multiply-adds), against the measured FP32 FMA rate x 2."""
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    bf16 = peaks.get("bf16_tflops", 1590.0)
    out = {}
    if st["m2l_ms"] > 0 and st["m2l_tiles"] > 0:
        issued = st["m2l_tiles"] * 39 * 6 * 2.0 * 128 * 32 * 16
        ach = issued / (st["m2l_ms"] * 1e-3) / 1e12
        q2 = 2 * st["q"]
        useful = st["m2l_pairs"] * 3 * q2 * q2 * 2.0
        out["m2l"] = {"bound": "tensor", "achieved": round(ach, 2), "peak": bf16,
                      "unit": "TFLOP/s", "frac": round(ach / bf16, 4),
                      "useful_frac_of_issued": round(useful / issued, 4),
                      "timing": "event span; the near field runs beside it on a second stream",
                      "ms": round(st["m2l_ms"], 4), "tiles": int(st["m2l_tiles"]),
                      "pairs": int(st["m2l_pairs"]),
                      "peak_source": "measured" if peaks else "fallback"}
    if rates and st["near_ms"] > 0:
        flops = st["p2p_pairs"] * 10.0
        ach = flops / (st["near_ms"] * 1e-3) / 1e12
        pk = 2 * rates["ffma_per_s"] / 1e12
        out["near"] = {"bound": "fp32", "achieved": round(ach, 2), "peak": round(pk, 1),
                      "unit": "TFLOP/s", "frac": round(ach / pk, 4), "ms": round(st["near_ms"], 4),
                      "timing": "event span; M2L, P2L and the downward pass run beside it",
                      "pairs": int(st["p2p_pairs"]), "peak_source": "measured (d3_device_peaks)"}
    return out


def fast_1m(pkg, core, torch, flush_l2, cpu=True):
    """Fast mode at 1M nodes: the reference's FP64 FMM ("plain", bit for bit)
    and the tensor-core form ("bf16x3": BF16x3 M2L, FP32 near field), both at
    order 8 / opening 1.5 / distanceMin 1, with link and center; ms per tick
    and RMS of the many-body kick against an FP64 direct sum on 4,096
    targets. The CPU leg ticks the oracle's fast mode (one thread) and checks
    the plain form's state after 3 ticks bit for bit."""
    layout = fast_layout()
    out = {"workload": "fast n=1000000 m=2000000 uniform [0,1e4)^2; manyBody FMM order 8, "
                       "opening 1.5, distanceMin 1 + link + center",
           "l2": "flushed before every tick"}
    for form in ("plain", "bf16x3"):
        ms, stats = fast_ticks(pkg, core, layout, form, flush_l2)
        out[form] = {"ms_per_tick": round(ms, 4), "steps": 10, "warmup": 3,
                     "rms_vs_direct_sum": fast_rms(pkg, core, layout, form),
                     "rms_targets": 4096}
        if form == "bf16x3":
            out[form]["last_pass"] = stats
    out["bf16x3"]["speedup_vs_plain"] = round(out["plain"]["ms_per_tick"] /
                                              out["bf16x3"]["ms_per_tick"], 3)
    out["roofline"] = fast_roofline(out["bf16x3"]["last_pass"], device_peaks(pkg))
    if cpu:
        import oracle
        ocore = oracle.load(pkg)
        xs, ys, src, tgt = layout
        nodes, sim = fast_sim(pkg, ocore, xs, ys, src, tgt, "plain")
        sim.tick(1)
        t0 = time.perf_counter()
        sim.tick(2)
        cpu_ms = (time.perf_counter() - t0) * 1e3 / 2
        dig_cpu = state_digest(nodes, ocore.sim_get_lcg(sim.ctx.h))
        sim.close()
        out["plain"]["bit_exact_vs_oracle_3_ticks"] = dig_cpu == fast_digest(pkg, core, layout,
                                                                             "plain")
        out["cpu_baseline"] = {"value": round(cpu_ms, 1), "unit": "ms/tick", "cores": 1,
                               "kind": "port",
                               "sample": "ticks 2-3 of the same workload on the oracle (C "
                                         "restatement of the reference's fast mode), one thread"}
    return out


LEARN_LAYOUTS, LEARN_N = 200, 100000
LEARN_HOLD = 16  # ticks on the fallback after a failed check


def learned_1m(pkg, core, torch, flush_l2):
    """The learned form at 1M nodes on the Gaussian-mixture configuration
    (64 clusters, sigma 50-500, Dirichlet(1) weights; SBM links, mean degree
    4, p_in / p_out 20), beside the plain FP64 order-8 FMM and the order-8
    tensor-core form: the network is trained here, on the GPU, by the
    package's kernels on order-4 / order-12 pairs of 200 seeded layouts of
    the same recipe at 100k nodes; the learned form's ticks include its
    sampled check (64 nodes, FP64 direct sum, tolerance 1e-5) and any
    fallback to the order-8 form."""
    import numpy as np
    learned = importlib.import_module("d3-force-wasm_b200.learned")
    acc = importlib.import_module("d3-force-wasm_b200.accuracy")
    t0 = time.perf_counter()
    layouts = [learned.mixture_layout(LEARN_N, 1000 + k)[:2] for k in range(LEARN_LAYOUTS)]
    X, Y = learned.training_pairs(core, layouts)
    t1 = time.perf_counter()
    params, losses = learned.train(core, X, Y)
    t2 = time.perf_counter()
    xs, ys, lab = learned.mixture_layout(FAST_N, 7)
    src, tgt = learned.sbm_links(lab, 7)
    out = {"workload": "fast n=1000000 Gaussian mixture (64 clusters, sigma 50-500, Dirichlet(1)) "
                       "+ SBM links (m=2n, p_in/p_out 20) + center; manyBody opening 1.5, "
                       "distanceMin 1",
           "training": {"layouts": LEARN_LAYOUTS, "nodes_per_layout": LEARN_N,
                        "samples": int(len(X)), "steps": len(losses), "batch": 8192,
                        "loss_first": float(losses[:10].mean()),
                        "loss_last": float(losses[-50:].mean()),
                        "pairs_s": round(t1 - t0, 2), "train_s": round(t2 - t1, 2)}}
    tg = acc.sample_targets(xs, ys, 4096)
    ref = None
    for form, order in (("plain", 8), ("bf16x3", 8), ("bf16x3", 4), ("learned", 8)):
        nodes, sim = fast_sim(pkg, core, xs, ys, src, tgt, form, order=order)
        if form == "learned":
            sim.learned(params, tolerance=1e-5, samples=64, hold=LEARN_HOLD)
        sim.device_begin()
        for _ in range(3):
            flush_l2()
            sim.device_ticks(1)
        # the learned form: two whole check cycles (a checked tick and the
        # `hold` ticks after a failed check), so the checks' cost is in the mean
        timed = 2 * (LEARN_HOLD + 1) if form == "learned" else 10
        times, checked = [], []
        for _ in range(timed):
            flush_l2()
            c0 = core.sim_stat(sim.ctx.h, 50)
            times.append(sim.device_ticks(1))
            checked.append(core.sim_stat(sim.ctx.h, 50) > c0)
        sim.device_end()
        stats = [core.sim_stat(sim.ctx.h, 50 + k) for k in range(3)]
        sim.close()
        kick, alpha = acc.many_body_kick(pkg, core, xs, ys, form=form, order=order) \
            if form != "learned" else _learned_kick(pkg, core, xs, ys, params)
        if ref is None:
            ref = acc.direct_kick(xs, ys, np.full(len(xs), -30.0 * alpha), tg)
        key = form if form != "bf16x3" else "bf16x3_order%d" % order
        out[key] = {"order": order, "ms_per_tick": round(sum(times) / len(times), 4),
                    "rms_vs_direct_sum": acc.rms(kick, ref, tg), "rms_targets": 4096}
        if form == "learned":
            out[key].update({"checks": stats[0], "fallbacks": stats[1],
                             "last_sampled_rms": stats[2], "hold_ticks": LEARN_HOLD,
                             "ticks_run": 3 + timed, "ticks_timed": timed,
                             "ms_checked_ticks": [round(t, 4) for t, c in zip(times, checked) if c],
                             "ms_other_ticks_mean": round(
                                 sum(t for t, c in zip(times, checked) if not c)
                                 / max(1, sum(1 for c in checked if not c)), 4)})
    out["learned"]["speedup_vs_plain_fp64_order8"] = round(
        out["plain"]["ms_per_tick"] / out["learned"]["ms_per_tick"], 3)
    return out


def batched(pkg, core, ticks=300):
    """Batched fast mode: 2,048 graphs (node counts log-uniform in [64,
    16384], about 6M nodes; half uniform links m = 2n, half SBM with 8
    communities, mean degree 4), manyBody FMM order 8 + link + collide(3) in
    FP32, one persistent launch per tick; the launch shape autotuned (3 ticks
    per candidate from the start layout), then `ticks` ticks captured in one
    CUDA graph and timed with CUDA events; per-graph RMS of the many-body kick
    against an FP64 direct sum on 256 sampled targets, at the start layout."""
    import numpy as np
    B = importlib.import_module("d3-force-wasm_b200.batch")
    graphs = B.batch_workload(2048, seed=1)
    b = B.Batch(core, graphs)
    try:
        kick, alpha = b.kick()
        rms = B.graph_rms(b, kick, alpha, range(len(graphs)))
        choice = b.autotune(ticks=3)
        ms = b.run(ticks, graph=True)
        x, y, vx, vy = b.read()
        finite = bool(np.all(np.isfinite(x)) and np.all(np.isfinite(y)))
    finally:
        b.close()
    return {"workload": "2048 graphs, n log-uniform [64, 16384] (%d nodes), half uniform m=2n, "
                        "half SBM (8 communities, mean degree 4); manyBody FMM order 8 + link + "
                        "collide(3), FP32" % int(sum(g[0] for g in graphs)),
            "ticks": ticks, "ms_total": round(ms, 2), "ms_per_tick": round(ms / ticks, 4),
            "launches_per_tick": 1, "cuda_graph": True, "autotune": choice,
            "rms_vs_direct_sum_per_graph": {"median": float(np.median(rms)),
                                            "p90": float(np.percentile(rms, 90)),
                                            "max": float(rms.max()), "targets": 256},
            "state_finite": finite}


def _learned_kick(pkg, core, xs, ys, params):
    """The learned form's many-body kick of one tick from zero velocity."""
    import numpy as np
    n = len(xs)
    nodes = pkg.Nodes(n, x=xs, y=ys, vx=np.zeros(n), vy=np.zeros(n))
    sim = pkg.forceSimulation(nodes, core=core)
    sim.force("charge", pkg.forceManyBody())
    sim.precision("fast", order=8, opening=1.5, form="learned")
    sim.learned(params, tolerance=1e-5, samples=64)
    sim.tick()
    alpha = sim.alpha()
    kick = np.stack([np.asarray(nodes.vx), np.asarray(nodes.vy)], 1) / 0.6
    sim.close()
    return kick, alpha


def exact_device_run(pkg, sc, core, positions, total, flush_l2, world, profile=False):
    """The exact workload's schedule on the device, one sim_tick per tick,
    L2 flushed before each. Returns per-tick device ms (CUDA events on the
    engine's stream), the launches of the timed ticks, the state digest at
    CHECK_TICK and at the end, and (profile) per-phase ms and engine stats at
    the timed ticks."""
    nodes, sim = sc.setup_exact(pkg, core, **WORKLOAD)
    h = sim.ctx.h
    timed = set(positions)
    per_tick, launches, digests = {}, 0, {}
    phases = {k: 0.0 for k in PHASES}
    side = {k: 0.0 for k in SIDE_PHASES}
    depth, levels = [], []
    sim.device_begin()
    for t in range(1, total + 1):
        flush_l2()
        if profile:
            core.sim_set_profile(h, 1 if t in timed else 0)
        l0 = core.sim_stat(h, 6)
        per_tick[t] = sim.device_ticks(1)
        if t in timed:
            launches += int(core.sim_stat(h, 6) - l0)
            if profile:
                for k, name in enumerate(PHASES):
                    phases[name] += core.sim_stat(h, 100 + k)
                for name, k in SIDE_PHASES.items():
                    side[name] += core.sim_stat(h, 100 + k)
                depth.append(core.sim_stat(h, 0))
                levels.append(core.sim_stat(h, 4))
        if t in (min(CHECK_TICK, total), total):
            sim.device_end()
            digests[t] = state_digest(nodes, core.sim_get_lcg(h))
            if t != total:
                sim.device_begin()
    stats = None
    if profile:
        core.sim_set_profile(h, 0)
        k = len(positions)
        stats = {"phase_ms_per_tick": {n: v / k for n, v in phases.items()},
                 "overlapped_ms_per_tick": {n: v / k for n, v in side.items()},
                 "collide_depth_mean": statistics.mean(depth), "collide_depth_max": max(depth),
                 "link_levels_mean": statistics.mean(levels),
                 "collide_serial_fallback": core.sim_stat(h, 2)}
        stats["collide_phases_us_last"] = {
            "guess": core.sim_stat(h, 12), "access_lists": core.sim_stat(h, 19),
            "turns": core.sim_stat(h, 13), "check": core.sim_stat(h, 14)}
        stats["tree_phases_us_last"] = {name: core.sim_stat(h, 30 + j) for j, name in enumerate(
            ["box", "keys", "sort", "runs", "cell_counts", "scan", "owners", "cells"])}
    sim.close()
    return per_tick, launches, digests, stats


def exact_e2e_run(pkg, sc, core, positions, total, flush_l2):
    """The same schedule through the public API: Simulation.tick(1) per tick,
    which copies the node state host-to-device (x, y, vx, vy, fx, fy from
    pinned memory), ticks, and copies x, y, vx, vy back. Wall-clock ms of the
    timed ticks."""
    nodes, sim = sc.setup_exact(pkg, core, **WORKLOAD)
    timed = set(positions)
    out = []
    for t in range(1, total + 1):
        flush_l2()
        t0 = time.perf_counter()
        sim.tick(1)
        if t in timed:
            out.append((time.perf_counter() - t0) * 1e3)
    sim.close()
    return out


def device_peaks(pkg):
    """d3_device_peaks: FP64 rates and the SM-to-SM handoff latency."""
    import ctypes

    lib = pkg.cuda_core().lib
    fn = lib.d3_device_peaks
    fn.restype = ctypes.c_int32
    fn.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_uint32]
    out = (ctypes.c_double * 9)()
    rc = fn(out, 9)
    if rc != 0:
        return None
    return {"dadd_per_s": out[0], "dmul_per_s": out[1], "dfma_per_s": out[2],
            "ddiv_per_s": out[3], "dsqrt_per_s": out[4], "handoff_us": out[5],
            "sms": int(out[6]), "clock_khz": int(out[7]), "ffma_per_s": out[8]}


def run_ours(args, pkg, sc):
    rank, local_rank, world = dist_env()
    if world > 1:
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local_rank)
    import torch
    import torch.distributed as dist

    if world > 1:
        dist.init_process_group("gloo", timeout=__import__("datetime").timedelta(seconds=300))
    core = pkg.cuda_core()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    def flush_l2():
        flush.zero_()
        torch.cuda.synchronize()

    positions, total = schedule_positions(args.warmup, args.steps, schedule=args.schedule)
    n, m = WORKLOAD["n"], WORKLOAD["m"]
    # the timed run: every tick of the schedule on the device, the K ticks at
    # `positions` timed; the clocks are sampled over the whole schedule
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(0 if world > 1 else int(os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0] or 0))
    per_tick, launches, digests, _ = exact_device_run(pkg, sc, core, positions, total, flush_l2, world)
    torch.cuda.synchronize()
    clk = clocks.stop()
    if world > 1:
        dist.barrier()
    ms = max_over_ranks(statistics.mean(per_tick[t] for t in positions), world)
    schedule_ms = statistics.mean(per_tick[t] for t in range(args.warmup + 1, total + 1))
    early_ms = statistics.mean(per_tick[t] for t in range(6, min(26, total + 1)))
    # the same schedule again with the phase timers on (outside the timed run)
    _, _, digests2, prof = exact_device_run(pkg, sc, core, positions, total, flush_l2, world,
                                            profile=True)
    # end to end through the public API
    e2e = exact_e2e_run(pkg, sc, core, positions, total, flush_l2)
    e2e_ms = max_over_ranks(statistics.mean(e2e), world)
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    rates = device_peaks(pkg)
    phase = prof["phase_ms_per_tick"]
    dom = max(phase, key=phase.get)
    # Algorithmic bytes of the collide pass (one launch per tick): per node
    # x, y, vx, vy, radius read and vx, vy written (56 B); per tree cell its
    # 88-byte record and 4-byte skip link, about 1.7 cells per node here.
    cells = 1.7 * n
    alg = {"collide_loop": n * 56 + cells * 92, "mb_traverse": n * 56 + cells * 92,
           "link": m * 32 + 64 * m}.get(dom, n * 64.0)
    achieved = alg / (phase[dom] * 1e-3) / 1e9
    # DRAM bytes (read + write) per collide launch: ncu capture of the bench
    # workload at tick 13 (the source, commit and command are in
    # profiles/k_collide_spec_exact_50k.md)
    traffic = {"collide_loop": COLLIDE_DRAM_BYTES}.get(dom)
    roof = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 2), "peak": hbm,
            "unit": "GB/s", "frac": round(achieved / hbm, 5), "traffic": traffic,
            "algorithmic_bytes": int(alg),
            "peak_source": "measured" if peaks else "fallback"}
    if rates:
        # The collide pass and the link are chains of dependent turns: a turn
        # starts only when the turns it depends on are seen finished from
        # another SM. Bound: depth x one measured SM-to-SM handoff.
        hand = rates["handoff_us"]
        cp = prof["collide_depth_mean"] * hand * 1e-3
        lp = prof["link_levels_mean"] * hand * 1e-3
        roof["critical_path"] = {
            "handoff_us": round(hand, 3),
            "collide_loop": {"depth_mean": round(prof["collide_depth_mean"], 2),
                             "bound_ms": round(cp, 4), "measured_ms": round(phase["collide_loop"], 4),
                             "frac": round(cp / phase["collide_loop"], 4)},
            "link": {"levels_mean": round(prof["link_levels_mean"], 2), "bound_ms": round(lp, 4),
                     "measured_ms": round(phase["link"], 4), "frac": round(lp / phase["link"], 4)}}
    line = {
        "metric": METRIC, "value": round(ms, 4), "unit": "ms/tick", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generators of the reference's scenarios)",
        "config": {"workload": WORKLOAD_NAME, "n": n, "m": m,
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": "flushed before every tick (256 MB write)",
                   "timed_ticks": "%d ticks spread evenly over ticks %d-%d of the %d-tick schedule"
                                  % (args.steps, args.warmup + 1, total, total)},
        "schedule_ms_per_tick": {"timed_ticks": round(ms, 4),
                                 "all_ticks_%d_%d" % (args.warmup + 1, total): round(schedule_ms, 4),
                                 "ticks_6_25": round(early_ms, 4)},
        "e2e": {"value": round(e2e_ms, 4), "unit": "ms/tick", "h2d_bytes_per_step": 48 * n,
                "d2h_bytes_per_step": 32 * n},
        "gpu_launches": launches,
        "phase_ms_per_tick": {k: round(v, 4) for k, v in phase.items()},
        "overlapped_ms_per_tick": {k: round(v, 4) for k, v in prof["overlapped_ms_per_tick"].items()},
        "roofline": roof,
        "engine_stats": {k: v for k, v in prof.items() if k not in ("phase_ms_per_tick",
                                                                    "overlapped_ms_per_tick")},
        "device_rates": rates,
        "clocks": clk,
    }
    # bit-exactness: the two device runs agree, and (CPU leg) the oracle's
    # state after CHECK_TICK ticks equals the device's
    checks = {"device_runs_agree": digests == digests2}
    if not args.no_cpu_baseline and world == 1:
        threads = os.cpu_count() or 1
        cpu_all, dig_all, work = oracle_protocol(pkg, sc, threads, count_work=True)
        cpu_one, dig_one, _ = oracle_protocol(pkg, sc, 1)
        checks["oracle_all_threads_tick_%d" % CHECK_TICK] = dig_all == digests.get(CHECK_TICK)
        checks["oracle_one_thread_tick_%d" % CHECK_TICK] = dig_one == digests.get(CHECK_TICK)
        line["cpu_baseline"] = {
            "value": round(cpu_all, 3), "unit": "ms/tick", "cores": threads, "kind": "port",
            "single_thread": round(cpu_one, 3),
            "sample": "bench/threads.js protocol: 5 warm-up ticks, then the minimum of 3 rounds "
                      "x 30 ticks (ticks 6-95) of the same workload; the oracle (C restatement "
                      "of the reference core, gcc -O3 -ffp-contract=off) on %d threads (threaded "
                      "where the reference's pool is: %s) and on 1 thread" % (threads, THREADED)}
        if rates and work:
            # FP64 work of the many-body traversal per tick, counted by the
            # oracle over ticks 66-95: per visited cell 8 ops (1 a division),
            # per accepted approximation 8 (2 divisions), per leaf point 6
            # (1 division); no FMA (strict f64). Roofline time: the non-division
            # ops at the DADD rate plus the divisions at the measured IEEE
            # division rate.
            V, A, P = work["V"], work["A"], work["P"]
            ops, divs = 8 * V + 8 * A + 6 * P, V + 2 * A + P
            t_roof = ((ops - divs) / rates["dadd_per_s"] + divs / rates["ddiv_per_s"]) * 1e3
            roof["fp64"] = {"kernel": "mb_traverse", "cells_visited": round(V),
                            "approximations": round(A), "point_interactions": round(P),
                            "fp64_ops": round(ops), "divisions": round(divs),
                            "t_roof_ms": round(t_roof, 4),
                            "measured_ms": round(phase["mb_traverse"], 4),
                            "frac": round(t_roof / phase["mb_traverse"], 4)}
    line["config"]["bit_exact"] = all(checks.values())
    line["bit_exact_checks"] = checks
    if not args.no_fast and world == 1:
        # the fast-mode legs; one that fails reports its error, not the line
        for key, leg in (("fast_1m", lambda: fast_1m(pkg, pkg.cuda_core(), torch, flush_l2,
                                                      cpu=not args.no_cpu_baseline)),
                         ("learned_1m", lambda: learned_1m(pkg, pkg.cuda_core(), torch, flush_l2)),
                         ("batched", lambda: batched(pkg, pkg.cuda_core()))):
            try:
                line[key] = leg()
            except Exception as e:  # noqa: BLE001
                line[key] = {"error": "%s: %s" % (type(e).__name__, e)}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_reference(args, pkg, sc):
    """The reference arm: the oracle (the reference's algorithm restated in C;
    zig, node and a wasm runtime are not on this machine) on all host cores,
    over the same schedule and the same K timed ticks as our arm."""
    rank, _, world = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    import oracle

    core = oracle.load(pkg)
    nodes, sim = sc.setup_exact(pkg, core, **WORKLOAD)
    core.lib.oracle_set_threads(sim.ctx.h, threads)
    positions, total = schedule_positions(args.warmup, args.steps)
    timed = set(positions)
    times = []
    for t in range(1, total + 1):
        t0 = time.perf_counter()
        sim.tick(1)
        if t in timed:
            times.append((time.perf_counter() - t0) * 1e3)
    sim.close()
    ms = statistics.mean(times)
    line = {
        "metric": METRIC, "value": round(ms, 3), "unit": "ms/tick", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generators of the reference's scenarios)",
        "config": {"workload": WORKLOAD_NAME, "n": WORKLOAD["n"], "m": WORKLOAD["m"],
                   "timed_ticks": "%d ticks spread evenly over ticks %d-%d of the %d-tick schedule"
                                  % (args.steps, args.warmup + 1, total, total)},
        "impl": "reference",
        "cpu_baseline": {"value": round(ms, 3), "unit": "ms/tick", "cores": threads,
                         "kind": "port",
                         "sample": "the whole %d-tick schedule, the same %d timed ticks as the "
                                   "GPU arm, each timed alone (C restatement of the reference "
                                   "core, threaded where the reference's pool is: %s; zig is "
                                   "unavailable)" % (total, args.steps, THREADED)},
        "e2e": {"value": round(ms, 3), "unit": "ms/tick", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_only(args, pkg):
    """One fast-mode leg alone, printed as its own JSON line (profiling runs)."""
    import torch
    core = pkg.cuda_core()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def flush_l2():
        flush.zero_()
        torch.cuda.synchronize()

    if args.only == "fast":
        out = fast_1m(pkg, core, torch, flush_l2, cpu=not args.no_cpu_baseline)
    elif args.only == "learned":
        out = learned_1m(pkg, core, torch, flush_l2)
    else:
        out = batched(pkg, core)
    print(json.dumps({args.only: out}), flush=True)


def main():
    args = parse()
    pkg = importlib.import_module("d3-force-wasm_b200")
    sc = importlib.import_module("d3-force-wasm_b200.scenarios")
    if args.only:
        run_only(args, pkg)
        return
    if args.impl == "reference":
        run_reference(args, pkg, sc)
    else:
        run_ours(args, pkg, sc)


if __name__ == "__main__":
    main()
