"""The CUDA library (no GPU needed): it loads and exports the whole C ABI."""

import ctypes
import os

import pytest

import helpers as H


def test_header_declares_the_bound_symbols():
    with open(os.path.join(H.ROOT, "include", "d3force_b200.h")) as f:
        text = f.read()
    for sym in H.C.ABI_SYMBOLS:
        assert sym + "(" in text, sym


def test_library_exports_every_symbol():
    if not os.path.exists(H.pkg.LIB_PATH):
        pytest.skip("engine not built")
    lib = ctypes.CDLL(H.pkg.LIB_PATH)
    for sym in H.C.ABI_SYMBOLS:
        assert hasattr(lib, sym), sym


def test_engine_only_symbols_declared_and_exported():
    with open(os.path.join(H.ROOT, "include", "d3force_b200.h")) as f:
        text = f.read()
    for sym in H.C.ENGINE_SYMBOLS:
        assert sym + "(" in text, sym
    if not os.path.exists(H.pkg.LIB_PATH):
        pytest.skip("engine not built")
    lib = ctypes.CDLL(H.pkg.LIB_PATH)
    for sym in H.C.ENGINE_SYMBOLS:
        assert hasattr(lib, sym), sym


def test_oracle_exports_every_symbol(ocore):
    for sym in H.C.ABI_SYMBOLS:
        assert hasattr(ocore.lib, sym), sym


def test_status_check_raises():
    with pytest.raises(H.pkg.CoreError):
        H.C.check(-3)
    assert H.C.check(1) == 1
