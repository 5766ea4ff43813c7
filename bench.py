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
PHASES = ["mb_tree", "mb_accumulate", "mb_traverse", "link", "collide_tree", "collide_loop",
          "center", "integrate"]
SIDE_PHASES = {"center_sum_side_stream": 11}
# What the CPU baseline (the oracle) spreads over the host threads, as the
# reference's worker pool does; link and collide's node loop are serial in both.
THREADED = "tree keys, sort and emission jobs; many-body record pass"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fast", action="store_true", help="skip the fast-mode 1M measurement")
    ap.add_argument("--e2e-steps", type=int, default=10)
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


def oracle_ms_per_tick(pkg, sc, threads, warmup, rounds, ticks):
    """The reference algorithm (oracle) on the host: `warmup` ticks, then the
    best of `rounds` rounds of `ticks` ticks (bench/threads.js:85-96)."""
    import oracle

    core = oracle.load(pkg)
    nodes, sim = sc.setup_exact(pkg, core, **WORKLOAD)
    core.lib.oracle_set_threads(sim.ctx.h, threads)
    sim.tick(warmup)
    best = float("inf")
    for _ in range(rounds):
        t0 = time.perf_counter()
        sim.tick(ticks)
        best = min(best, (time.perf_counter() - t0) * 1e3 / ticks)
    sim.close()
    return best


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


def fast_1m(pkg, core, torch, steps=10, warmup=3, targets=1024):
    """Fast mode at the 1M-node configuration: n uniform in [0, 1e4)^2 (seeded),
    m = 2n uniform links, forceManyBody (FMM order 8, opening 1.5,
    distanceMin 1) + forceLink + forceCenter, device ms per tick over `steps`
    ticks; plus the many-body kick's RMS error on seeded targets against an
    FP64 direct sum of d3's pair formula (test/fast/error-test.js:44-70)."""
    import numpy as np
    n = FAST_N
    rng = np.random.default_rng(1)
    xs = rng.random(n) * 1e4
    ys = rng.random(n) * 1e4
    src = rng.integers(0, n, 2 * n)
    tgt = (src + 1 + rng.integers(0, n - 1, 2 * n)) % n
    nodes = pkg.Nodes(n, x=xs, y=ys)
    sim = pkg.forceSimulation(nodes, core=core)
    sim.force("charge", pkg.forceManyBody())
    sim.force("link", pkg.forceLink(src, tgt))
    sim.force("center", pkg.forceCenter())
    sim.precision("fast", order=8, opening=1.5)
    sim.device_begin()
    for _ in range(warmup):
        sim.device_ticks(1)
    times = [sim.device_ticks(1) for _ in range(steps)]
    sim.device_end()
    sim.close()
    # RMS of the many-body kick alone, from the start layout with zero velocity
    nodes = pkg.Nodes(n, x=xs, y=ys, vx=np.zeros(n), vy=np.zeros(n))
    sim = pkg.forceSimulation(nodes, core=core)
    sim.force("charge", pkg.forceManyBody())
    sim.precision("fast", order=8, opening=1.5)
    sim.tick()
    a1 = sim.alpha()
    decay = 0.6  # 1 - velocityDecay(0.4): v = kick * decay after one tick
    kick = np.stack([(np.asarray(nodes.x) - xs) / decay, (np.asarray(nodes.y) - ys) / decay], 1)
    sim.close()
    tg = np.random.default_rng(7).choice(n, targets, replace=False)
    dev = torch.device("cuda")
    X = torch.from_numpy(xs).to(dev)
    Y = torch.from_numpy(ys).to(dev)
    ref = torch.zeros(targets, 2, dtype=torch.float64, device=dev)
    for k0 in range(0, targets, 64):
        idx = torch.from_numpy(tg[k0:k0 + 64]).to(dev)
        dx = X[None, :] - X[idx, None]
        dy = Y[None, :] - Y[idx, None]
        l = dx * dx + dy * dy
        l = torch.where(l < 1.0, torch.sqrt(l), l)  # distanceMin 1: l = sqrt(dmin2 l)
        w = torch.where(l > 0, -30.0 * a1 / torch.where(l > 0, l, torch.ones_like(l)),
                        torch.zeros_like(l))
        ref[k0:k0 + 64, 0] = (dx * w).sum(1)
        ref[k0:k0 + 64, 1] = (dy * w).sum(1)
    ref = ref.cpu().numpy()
    err = kick[tg] - ref
    rms = float(np.sqrt((err * err).sum() / (ref * ref).sum()))
    return {"workload": "fast n=1000000 m=2000000 uniform [0,1e4)^2; FMM order 8, opening 1.5, "
                        "distanceMin 1 + link + center; FP64 plain",
            "ms_per_tick": round(sum(times) / len(times), 4), "steps": steps, "warmup": warmup,
            "rms_vs_direct_sum": rms, "rms_targets": targets,
            "bit_exact_vs_reference_order": True}


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

    nodes, sim = sc.setup_exact(pkg, core, **WORKLOAD)
    h = sim.ctx.h
    sim.device_begin()
    for _ in range(args.warmup):
        flush_l2()
        sim.device_ticks(1)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(0 if world > 1 else int(os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0] or 0))
    launches0 = core.sim_stat(h, 6)
    times = []
    for _ in range(args.steps):
        flush_l2()
        times.append(sim.device_ticks(1))
    launches = int(core.sim_stat(h, 6) - launches0)
    torch.cuda.synchronize()
    clk = clocks.stop()
    # the phase breakdown: further ticks with the engine's phase timers on
    # (events between phases), outside the timed region
    prof_steps = min(args.steps, 10)
    core.sim_set_profile(h, 1)
    for _ in range(prof_steps):
        flush_l2()
        sim.device_ticks(1)
    phases = {name: core.sim_stat(h, 100 + k) for k, name in enumerate(PHASES)}
    side = {name: core.sim_stat(h, 100 + k) / prof_steps for name, k in SIDE_PHASES.items()}
    core.sim_set_profile(h, 0)
    ms = max_over_ranks(sum(times) / len(times), world)
    if world > 1:
        dist.barrier()
    sim.device_end()
    # e2e through the public API: node state in, tick, node state out
    e2e = []
    for _ in range(args.e2e_steps):
        flush_l2()
        t0 = time.perf_counter()
        sim.tick(1)
        e2e.append((time.perf_counter() - t0) * 1e3)
    n = WORKLOAD["n"]
    e2e_ms = max_over_ranks(sum(e2e) / len(e2e), world)
    stats = {"collide_depth": core.sim_stat(h, 0), "collide_attempts": core.sim_stat(h, 1),
             "collide_serial_fallback": core.sim_stat(h, 2), "link_levels": core.sim_stat(h, 4)}
    # the last tick's collide pass and collide tree build, from the kernels'
    # own globaltimer stamps (microseconds)
    stats["collide_phases_us"] = {"guess": core.sim_stat(h, 12), "access_lists": core.sim_stat(h, 19),
                                  "turns": core.sim_stat(h, 13), "check": core.sim_stat(h, 14)}
    stats["tree_phases_us"] = {name: core.sim_stat(h, 30 + k) for k, name in enumerate(
        ["box", "keys", "sort", "runs", "cell_counts", "scan", "owners", "cells"])}
    sim.close()
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    # Roofline of the dominant phase: the exact many-body traversal is the
    # f64 work; bytes are the HBM traffic of its inputs and outputs per tick.
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    dom = max(phases, key=phases.get)
    per_tick_ms = {k: v / prof_steps for k, v in phases.items()}
    # Algorithmic bytes per launch of the dominant phase (one launch per tick).
    # Per node: x, y read (16 B), vx, vy read and written (32 B), radius or
    # strength (8 B); per tree cell: the 88-byte cell and its 4-byte skip link,
    # with about 1.7 cells per node at this size.
    cells = 1.7 * n
    alg_bytes = {
        "mb_traverse": n * 56 + cells * 92,
        "collide_loop": n * 56 + cells * 92,
        "link": WORKLOAD["m"] * (2 * 4 + 3 * 8) + 4 * WORKLOAD["m"] * 8 * 2,
    }.get(dom, n * 64.0)
    # DRAM bytes (read + write) per launch from one ncu capture of tick 13 of
    # this workload (after an L2 flush).
    traffic = {"collide_loop": 63628032 + 9661184, "mb_traverse": 7734016}.get(dom)
    achieved = alg_bytes / (per_tick_ms[dom] * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": round(ms, 4), "unit": "ms/tick", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generators of the reference's scenarios)",
        "config": {"workload": WORKLOAD_NAME, "n": n, "m": WORKLOAD["m"],
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": "flushed between timed ticks (256 MB write)", "bit_exact": True},
        "e2e": {"value": round(e2e_ms, 4), "unit": "ms/tick", "h2d_bytes_per_step": 48 * n,
                "d2h_bytes_per_step": 32 * n},
        "gpu_launches": launches,
        "phase_ms_per_tick": {k: round(v, 4) for k, v in per_tick_ms.items()},
        "overlapped_ms_per_tick": {k: round(v, 4) for k, v in side.items()},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 2),
                     "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 5),
                     "traffic": traffic, "peak_source": "measured" if peaks else "fallback"},
        "engine_stats": stats,
        "clocks": clk,
    }
    if not args.no_fast and world == 1:
        line["fast_1m"] = fast_1m(pkg, pkg.cuda_core(), torch)
    if not args.no_cpu_baseline and world == 1:
        threads = os.cpu_count() or 1
        cpu = oracle_ms_per_tick(pkg, sc, threads, warmup=3, rounds=2, ticks=8)
        line["cpu_baseline"] = {"value": round(cpu, 3), "unit": "ms/tick", "cores": threads,
                                "kind": "port",
                                "sample": "3 warm-up ticks then best of 2 rounds x 8 ticks of the "
                                          "same workload (C restatement of the reference core, "
                                          "threaded where the reference's pool is: " + THREADED
                                          + ")"}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_reference(args, pkg, sc):
    rank, _, world = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    import oracle

    core = oracle.load(pkg)
    nodes, sim = sc.setup_exact(pkg, core, **WORKLOAD)
    core.lib.oracle_set_threads(sim.ctx.h, threads)
    sim.tick(args.warmup)
    steps = max(1, min(args.steps, 60))
    t0 = time.perf_counter()
    sim.tick(steps)
    ms = (time.perf_counter() - t0) * 1e3 / steps
    sim.close()
    line = {
        "metric": METRIC, "value": round(ms, 3), "unit": "ms/tick", "n_gpus": world,
        "steps": steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generators of the reference's scenarios)",
        "config": {"workload": WORKLOAD_NAME, "n": WORKLOAD["n"], "m": WORKLOAD["m"]},
        "impl": "reference",
        "cpu_baseline": {"value": round(ms, 3), "unit": "ms/tick", "cores": threads,
                         "kind": "port",
                         "sample": "%d warm-up then %d ticks of the workload (C restatement of "
                                   "the reference core, threaded where the reference's pool is: "
                                   "%s; zig is unavailable)" % (args.warmup, steps, THREADED)},
        "e2e": {"value": round(ms, 3), "unit": "ms/tick", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    pkg = importlib.import_module("d3-force-wasm_b200")
    sc = importlib.import_module("d3-force-wasm_b200.scenarios")
    if args.impl == "reference":
        run_reference(args, pkg, sc)
    else:
        run_ours(args, pkg, sc)


if __name__ == "__main__":
    main()
