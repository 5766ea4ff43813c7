"""The exact parallel center sum: bit-identical to the serial index-order sum
(simple.zig:14-31) on inputs that force its every path: long same-binade runs,
binade crossings, sums through zero, ties, signed zeros, NaN, huge ranges."""

import numpy as np
import pytest

import helpers as H
import parity as P

pkg = H.pkg
pytestmark = pytest.mark.gpu


def _center_only(xs, ys):
    def setup(core):
        nd = pkg.Nodes(len(xs), x=xs, y=ys, vx=[0.0] * len(xs), vy=[0.0] * len(xs))
        sim = pkg.forceSimulation(nd, core=core).force("center", pkg.forceCenter(3.5, -2.25))
        return nd, sim
    return setup


@pytest.mark.parametrize("case", ["walk", "offset", "ties", "tiny_huge", "zeros_nan", "large",
                                  "centered_1m", "one", "odd_tail", "serial_max", "records_min"])
def test_gpu_center_sum_bitwise(ocore, gcore, case):
    """Up to 65,536 nodes the sums run serially on one warp (bulk-copied
    tiles of 1,024 values, an odd last value loaded on its own); above that,
    the parallel record pipeline."""
    rng = np.random.default_rng(5)
    n = 50000
    if case in ("one", "odd_tail", "serial_max", "records_min"):
        n = {"one": 1, "odd_tail": 3073, "serial_max": 65536, "records_min": 65537}[case]
        xs = rng.normal(0, 2500, n)
        ys = 1e3 + rng.normal(0, 1, n)
    elif case == "walk":
        xs = rng.normal(0, 2500, n)
        ys = rng.normal(0, 2500, n)
    elif case == "offset":
        xs = 1e5 + rng.normal(0, 10, n)
        ys = -3e6 + rng.normal(0, 1000, n)
    elif case == "ties":
        xs = np.round(rng.normal(0, 1e6, n)) + 0.5
        ys = np.round(rng.normal(0, 4, n)) * 0.25
    elif case == "tiny_huge":
        xs = rng.normal(0, 1, n) * 10.0 ** rng.integers(-12, 12, n)
        ys = rng.normal(0, 1, n) * 10.0 ** rng.integers(-300, 300, n)
    elif case == "zeros_nan":
        xs = np.where(rng.random(n) < 0.5, -0.0, 0.0)
        ys = rng.normal(0, 1, n)
        ys[n // 2] = np.nan
    elif case == "large":
        n = 300000
        xs = rng.normal(0, 1e4, n)
        ys = rng.uniform(-1, 1, n) * 2.0 ** 40
    else:  # a laid-out graph after centring: the running sum wanders through zero
        n = 1000000
        xs = rng.uniform(-5000, 5000, n)
        xs -= xs.mean()
        ys = rng.uniform(0, 1e4, n)
    P.run_pair(_center_only(list(xs), list(ys)), ocore, gcore, 3)
