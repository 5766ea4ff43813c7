"""`bench.py --impl reference` on the CPU: the reference arm times the oracle
(the reference core's algorithm restated in C) on the host cores, over the
same schedule and workload as the GPU arm, and prints the same JSON line with
`"impl": "reference"`. Under torchrun only rank 0 runs it; the other ranks
exit 0 without work or output. Both arms time the same ticks of the
300-tick schedule (`schedule_positions`)."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench(extra_env, *args):
    env = dict(os.environ, **extra_env)
    env.pop("CUDA_VISIBLE_DEVICES", None)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                           *args], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_the_contract_line():
    sys.path.insert(0, ROOT)
    import bench

    r = _bench({}, "--steps", "3", "--warmup", "3")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == "ms/tick"
    assert d["higher_is_better"] is False
    assert d["steps"] == 3 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert d["value"] > 0 and d["ms_per_step"] == d["value"]
    assert d["config"]["workload"] == bench.WORKLOAD_NAME
    assert d["config"]["n"] == bench.WORKLOAD["n"] and d["config"]["m"] == bench.WORKLOAD["m"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert cb["unit"] == "ms/tick" and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == "ms/tick"
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_do_no_work():
    r = _bench({"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"}, "--gpus", "2",
               "--steps", "3", "--warmup", "3")
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]


def test_timed_ticks_spread_over_the_schedule():
    """The K timed ticks lie after the W warm-up ticks, strictly increasing,
    the last one the schedule's last tick; a run longer than the schedule
    extends it."""
    sys.path.insert(0, ROOT)
    import bench

    for w, k in [(3, 1), (3, 20), (5, 30), (5, 295), (10, 300)]:
        pos, total = bench.schedule_positions(w, k)
        assert total == max(bench.SCHEDULE_TICKS, w + k)
        assert len(pos) == k and pos[-1] == total and pos[0] > w
        assert all(b > a for a, b in zip(pos, pos[1:]))
