"""Batched fast mode on the B200 (no reference counterpart): the per-graph
many-body kick against an FP64 direct sum (the fast mode's judge,
test/fast/error-test.js:44-70) on 256 sampled targets per graph; results
independent of the launch shape and of the CUDA-graph capture (the
reference's determinism contract: results do not depend on how the work is
split, src/core/pool.zig:7-10); and the ticks move the layout."""

import importlib

import numpy as np
import pytest

import helpers as H

B = importlib.import_module("d3-force-wasm_b200.batch")
pytestmark = pytest.mark.gpu


def _graphs(k=48, seed=2, nmax=4096):
    return B.batch_workload(k, seed=seed, nmax=nmax)


def test_gpu_batch_many_body_rms_per_graph(gcore):
    graphs = _graphs()
    b = B.Batch(gcore, graphs)
    try:
        kick, alpha = b.kick()
        rms = B.graph_rms(b, kick, alpha, range(len(graphs)))
        print("per-graph RMS: median %.3g max %.3g" % (np.median(rms), rms.max()))
        assert rms.max() < 1e-4
    finally:
        b.close()


def _state(b):
    return np.concatenate([a.view(np.uint32) for a in b.read()])


def test_gpu_batch_results_independent_of_launch_shape_and_graph(gcore):
    graphs = _graphs(24, seed=5)
    out = []
    for shape, graph in (((256, 1, 16), False), ((1024, 1, 16), True), ((512, 2, 16), True)):
        b = B.Batch(gcore, graphs)
        try:
            b.set_shape(*shape)
            b.run(4, graph=graph)
            b.run(6, graph=graph)
            out.append(_state(b))
        finally:
            b.close()
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[0], out[2])


def test_gpu_batch_ticks_move_and_autotune_picks_a_shape(gcore):
    graphs = _graphs(32, seed=7)
    b = B.Batch(gcore, graphs)
    try:
        choice = b.autotune(ticks=2)
        assert choice["threads"] in (256, 512, 1024) and choice["ms_per_tick"] > 0
        x0 = b.x0.copy()
        ms = b.run(20, graph=True)
        x, y, vx, vy = b.read()
        assert ms > 0 and np.all(np.isfinite(x)) and np.all(np.isfinite(vx))
        assert np.abs(x - x0).max() > 1e-3
    finally:
        b.close()
