"""The C-ABI library loads and exports every symbol include/aspher_b200.h
declares (no compute call: this runs without a GPU)."""

import ctypes
import os
import re

import pytest

from aspher_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "include", "aspher_b200.h")

STENCIL_GOLDEN = {(0, 0): 1.0, (1, 0): -0.180875, (1, 1): -0.032860, (2, 0): 0.021189,
                  (2, 1): -0.003912, (2, 2): -0.003198}  # tests/test_stencil.cpp:21-33


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(aspher_[a-z0-9_]+)\s*\(", src)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = _lib.lib()
    names = declared_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n
        assert n in _lib.SIGNATURES, "ctypes signature missing for " + n
    assert lib.aspher_abi_version() == 3


def test_status_strings_match_reference_taxonomy():
    lib = _lib.lib()
    for i, name in enumerate(_lib.STATUS_NAMES):
        assert lib.aspher_status_string(i).decode() == name


def test_stencil_taps_golden():
    """Tap weights computed by the library (host code) vs test_stencil.cpp:21-33."""
    from aspher_b200.api import stencil_taps
    for Ns in (512, 1024, 2048):
        dx, dy, w = stencil_taps(Ns, 2)
        assert len(w) == 13
        for a, b, v in zip(dx, dy, w):
            key = (max(abs(a), abs(b)), min(abs(a), abs(b)))
            assert abs(v - STENCIL_GOLDEN[key]) <= 5e-6
            if a == 0 and b == 0:
                assert v == 1.0


def test_stencil_taps_match_oracle_small_grids():
    from aspher_b200.api import stencil_taps
    from oracle.precond import StencilPreconditioner
    for Ns, R in ((16, 2), (64, 1), (64, 4), (256, 2)):
        dx, dy, w = stencil_taps(Ns, R)
        sp = StencilPreconditioner(Ns, R)
        assert dx == sp.tap_dx and dy == sp.tap_dy
        assert max(abs(a - b) for a, b in zip(w, sp.tap_w)) < 1e-13


def test_invalid_arguments_raise_before_any_device_work():
    from aspher_b200.api import stencil_taps
    with pytest.raises(ValueError):
        stencil_taps(4, 2)  # 2R+1 > Ns
    with pytest.raises(ValueError):
        stencil_taps(64, 0)


def test_stencil_for_level_decision_table():
    """tests/test_precond.cpp:68-101 (exhaustive table)."""
    from aspher_b200.nested import stencil_for_level as f
    omax = 0.4
    assert not f("stencil", False, -1.0, omax)
    assert not f("fft", False, 0.1, omax)
    assert not f("auto", False, 0.9, omax)
    assert f("stencil", True, -1.0, omax) and f("stencil", True, 0.0, omax)
    assert f("stencil", True, 0.9, omax)
    assert not f("fft", True, -1.0, omax) and not f("fft", True, 0.0, omax)
    assert not f("fft", True, 0.9, omax)
    assert f("auto", True, -1.0, omax) and f("auto", True, 0.0, omax)
    assert f("auto", True, 0.39, omax)
    assert not f("auto", True, 0.4, omax) and not f("auto", True, 0.41, omax)
    assert not f("auto", True, 1.0, omax)
    assert f("auto", True, 0.55, 0.6) and not f("auto", True, 0.65, 0.6)
