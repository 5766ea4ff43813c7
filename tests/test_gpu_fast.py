"""Fast mode on the B200: the Jacobi link and the grid collide are per-node
passes with the reference's per-node operation order, so they match the
oracle bit for bit; the FMM is checked by RMS error."""

import numpy as np
import pytest

import helpers as H
import parity as P

pkg, sc = H.pkg, H.scenarios
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["uniform 4000", "grid 2500 with exact zero deltas"])
def test_gpu_fast_link_collide_center_bitwise(ocore, gcore, name):
    def setup(core):
        nodes, src, tgt = sc.fast_scenario(name)
        sim = pkg.forceSimulation(nodes, core=core)
        sim.force("link", pkg.forceLink(src, tgt))
        sim.force("collide", pkg.forceCollide(3))
        sim.force("center", pkg.forceCenter())
        sim.precision("fast")
        return nodes, sim
    P.run_pair(setup, ocore, gcore, 100)
