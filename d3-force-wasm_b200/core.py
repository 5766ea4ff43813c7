"""ctypes binding of the engine's C ABI (include/d3force_b200.h).

`Core` wraps any shared library exporting that ABI. The product library is the
CUDA engine (``_lib/libd3force_b200.so``, built by ``build.py``); the function
set mirrors the exports of d3-force-wasm's core (``src/core/root.zig``), so the
facade in ``simulation.py`` drives it exactly as ``src/core.js`` drives the
wasm core.
"""

import ctypes
import os

import numpy as np

# Status codes (root.zig:16-25).
OK, GROWN, ARENA_FULL, RNG_EXHAUSTED = 0, 1, 2, 3
BAD_HANDLE, OUT_OF_MEMORY, BAD_ARGUMENT, WORKER_FAILED = -1, -2, -3, -4
STATUS_NAMES = {-1: "BAD_HANDLE", -2: "OUT_OF_MEMORY", -3: "BAD_ARGUMENT", -4: "WORKER_FAILED"}

# Force kinds, scalar slots, array slots (src/core.js:33-42, force.zig:8-21).
CENTER, COLLIDE, LINK, MANY_BODY, RADIAL, X, Y = range(7)
(STRENGTH, CX, CY, THETA2, DISTANCE_MIN2, DISTANCE_MAX2, ITERATIONS, PRECISION, ORDER,
 OPENING, SEED) = range(11)
F0, F1, F2, SOURCE, TARGET = range(5)
PTR_X, PTR_Y, PTR_VX, PTR_VY, PTR_FX, PTR_FY, PTR_FIXED, PTR_PERM, PTR_RNG_BUF, PTR_SNAP = range(10)
# Float parameter arrays per kind (src/core.js:45, force.zig:49-56).
FLOATS = [0, 1, 3, 1, 2, 2, 2]

SYNC_EXPLICIT, SYNC_PER_CALL = 0, 1

RANDOM_FN = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.c_void_p)

CELL_DTYPE = np.dtype([
    ("child", "<u4", (4,)), ("first", "<u4"), ("count", "<u4"),
    ("x0", "<f8"), ("y0", "<f8"), ("x1", "<f8"), ("y1", "<f8"),
    ("x", "<f8"), ("y", "<f8"), ("value", "<f8"), ("r", "<f8"),
])
assert CELL_DTYPE.itemsize == 88


class CoreError(RuntimeError):
    """A negative status from the core (src/core.js:45-48 `check`)."""

    def __init__(self, status):
        super().__init__(STATUS_NAMES.get(status, "core status %d" % status))
        self.status = status


def check(status):
    if status < 0:
        raise CoreError(status)
    return status


_U32, _I32, _F64, _PTR = ctypes.c_uint32, ctypes.c_int32, ctypes.c_double, ctypes.c_size_t

_SIGNATURES = {
    "sim_create": (_U32, []),
    "sim_destroy": (_I32, [_U32]),
    "sim_set_node_count": (_I32, [_U32, _U32]),
    "sim_ptr": (_PTR, [_U32, _U32]),
    "force_create": (_U32, [_U32, _U32]),
    "force_destroy": (_I32, [_U32, _U32]),
    "force_set_count": (_I32, [_U32, _U32, _U32]),
    "force_ptr": (_PTR, [_U32, _U32, _U32]),
    "force_set_scalar": (_I32, [_U32, _U32, _U32, _F64]),
    "force_get_scalar": (_F64, [_U32, _U32, _U32]),
    "force_run": (_I32, [_U32, _U32, _F64]),
    "sim_integrate": (_I32, [_U32, _F64]),
    "sim_snapshot": (_I32, [_U32, _U32]),
    "tree_build": (_I32, [_U32, _U32]),
    "tree_info": (_PTR, [_U32, _U32]),
    "tree_order": (_I32, [_U32, _U32, ctypes.c_void_p]),
    "sim_set_random": (_I32, [_U32, RANDOM_FN, ctypes.c_void_p]),
    "sim_set_lcg": (_I32, [_U32, _U32]),
    "sim_get_lcg": (_U32, [_U32]),
    "sim_set_sync": (_I32, [_U32, _U32]),
    "sim_sync_in": (_I32, [_U32]),
    "sim_set_fixed_source": (_I32, [_U32, _U32]),
    "sim_sync_out": (_I32, [_U32]),
    "sim_tick": (_I32, [_U32, _U32, ctypes.POINTER(_F64), _F64, _F64, _F64,
                        ctypes.POINTER(_U32), _U32]),
    "sim_tick_sync": (_I32, [_U32, _U32, ctypes.POINTER(_F64), _F64, _F64, _F64,
                             ctypes.POINTER(_U32), _U32]),
    "sim_last_tick_ms": (_F64, [_U32]),
    "sim_find": (_I32, [_U32, _F64, _F64, _F64, ctypes.POINTER(_U32)]),
    "sim_stat": (_F64, [_U32, _U32]),
    "sim_set_profile": (_I32, [_U32, _U32]),
    "sim_selftest_wait": (_I32, [_U32, _U32]),
}

# Engine-only entry points bound with signatures (the oracle has none of them).
_ENGINE_SIGNATURES = {
    "sim_set_learned": (_I32, [_U32, ctypes.c_void_p, _U32, _F64, _U32, _U32]),
    "sim_fmm_leaves": (_I32, [_U32, ctypes.c_void_p, _U32]),
}

# Every symbol the header declares; the no-GPU tests check the CUDA library
# exports all of them.
ABI_SYMBOLS = tuple(_SIGNATURES)

# Entry points of the CUDA library alone (the oracle has no counterpart):
# declared in the header and exported by the engine, bound where they are used.
ENGINE_SYMBOLS = ("d3_device_peaks", "d3_many_body_exact_noalloc", "sim_set_learned",
                  "sim_fmm_leaves", "d3_mlp_grad", "d3_mlp_train", "d3_mlp_infer", "batch_create",
                  "batch_destroy", "batch_set_shape", "batch_run", "batch_kick", "batch_read",
                  "batch_autotune")


class Core:
    """One loaded library implementing the C ABI."""

    def __init__(self, path, name=None):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.path = path
        self.name = name or os.path.basename(path)
        self.lib = ctypes.CDLL(path)
        for sym, (res, args) in _SIGNATURES.items():
            fn = getattr(self.lib, sym)
            fn.restype = res
            fn.argtypes = args
            setattr(self, sym, fn)
        for sym, (res, args) in _ENGINE_SIGNATURES.items():
            fn = getattr(self.lib, sym, None)
            if fn is not None:
                fn.restype = res
                fn.argtypes = args
                setattr(self, sym, fn)

    # Typed views of mirrors (valid until the next GROWN / resize).
    @staticmethod
    def f64_view(addr, n):
        if not addr or n == 0:
            return np.zeros(0, np.float64)
        return np.ctypeslib.as_array((ctypes.c_double * n).from_address(addr))

    @staticmethod
    def u32_view(addr, n):
        if not addr or n == 0:
            return np.zeros(0, np.uint32)
        return np.ctypeslib.as_array((ctypes.c_uint32 * n).from_address(addr))

    @staticmethod
    def u8_view(addr, n):
        if not addr or n == 0:
            return np.zeros(0, np.uint8)
        return np.ctypeslib.as_array((ctypes.c_uint8 * n).from_address(addr))

    def tree(self, h):
        """The last tree built on simulation h: extent, cells, perm (copies)."""
        n_cells = self.tree_info(h, 0)
        m = self.tree_info(h, 6)
        extent = self.f64_view(self.tree_info(h, 3), 4).copy()
        if n_cells:
            buf = (ctypes.c_uint8 * (88 * n_cells)).from_address(self.tree_info(h, 2))
            cells = np.frombuffer(bytes(buf), dtype=CELL_DTYPE).copy()
        else:
            cells = np.zeros(0, CELL_DTYPE)
        perm = self.u32_view(self.tree_info(h, 4), m).copy()
        return {"extent": extent, "cells": cells, "perm": perm, "root": self.tree_info(h, 1)}

    def order(self, h, after):
        n_cells = self.tree_info(h, 0)
        out = np.zeros(max(n_cells, 1), np.uint32)
        check(self.tree_order(h, after, out.ctypes.data))
        return out[:n_cells]
