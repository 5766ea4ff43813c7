"""CPU oracle (test infrastructure only).

`load()` builds (if needed) and loads ``_build/libd3oracle.so``, the C
restatement of d3-force-wasm's Zig core, as a `Core` with the engine's ABI.
Only tests/, the smoke check and bench.py's CPU-baseline leg use it; it is the
checker, never the thing measured on the GPU path.
"""

import ctypes
import os
import subprocess

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(ORACLE_DIR, "_build", "libd3oracle.so")


def build():
    src = os.path.join(ORACLE_DIR, "d3force_oracle.c")
    mk = os.path.join(ORACLE_DIR, "Makefile")
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(src),
                                                              os.path.getmtime(mk)):
        subprocess.check_call(["make", "-s", "-C", ORACLE_DIR])
    return LIB


def load(pkg):
    """The oracle as a `pkg.Core` (pkg = the engine package module)."""
    build()
    c = pkg.Core(LIB, "oracle")
    c.lib.oracle_set_threads.restype = ctypes.c_int32
    c.lib.oracle_set_threads.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
    c.lib.oracle_fmm_stat.restype = ctypes.c_uint64
    c.lib.oracle_fmm_stat.argtypes = [ctypes.c_uint32]
    c.lib.oracle_mb_stat.restype = ctypes.c_uint64
    c.lib.oracle_mb_stat.argtypes = [ctypes.c_uint32]
    return c
