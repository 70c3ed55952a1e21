"""The C-ABI library loads and exports every entry point that
include/fastlpr_b200.h declares; argument errors are reported without
touching a GPU."""
import ctypes
import os
import re

import pytest

from fastlpr_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "fastlpr_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(flpr_[a-z0-9_]+)\s*\(",
                       src, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), f"missing export {n}"
    bound = {s[0] for s in _lib.SIGNATURES}
    assert set(names) <= bound | {"flpr_version"}, set(names) - bound


def test_argument_errors_need_no_gpu():
    lib = _lib.load()
    L = _lib.ivec([64])
    st = lib.flpr_spread(5, 10, None, _lib.dvec([0] * 9), L, 4, _lib.dvec([1.0]), 1, 1,
                         _lib.pvec([]), None, 0, None, 0, None)
    assert st == -1
    assert b"d=5" in lib.flpr_last_error()
    st = lib.flpr_solve(3, 2, 1, 1, 10, 1, None, None, 0.0, None, None, 0, None)
    assert st == -1
    assert b"order" in lib.flpr_last_error()
    st = lib.flpr_spread(1, 10, None, _lib.dvec([0] * 9), L, 13, _lib.dvec([1.0]), 1, 1,
                         _lib.pvec([]), None, 0, None, 0, None)
    assert st == -1
    assert b"[0,12]" in lib.flpr_last_error()


def test_workspace_queries_are_consistent():
    lib = _lib.load()
    small = lib.flpr_spread_ws(2, 1000, _lib.ivec([64, 64]), 4, 12, 0)
    big = lib.flpr_spread_ws(2, 100000, _lib.ivec([64, 64]), 4, 12, 0)
    assert 0 < small < big
    assert lib.flpr_point_stats_ws(2, 10 ** 6) > 0
    assert lib.flpr_kde_ws(100, 16, 4096) >= 16 * 8


def test_device_knot_map_argument_errors_need_no_gpu():
    lib = _lib.load()
    v = _lib.dvec([0.0, 0.0, 0.0])
    assert lib.flpr_knot_map(5, 10, None, v, v, v, None, None) == -1
    assert b"d=5" in lib.flpr_last_error()
    assert lib.flpr_knot_map(2, 10, None, v, v, v, None, None) == -1
    assert b"null" in lib.flpr_last_error()
    L = _lib.ivec([64, 64])
    st = lib.flpr_spread_dkmap(2, 10, None, None, v, L, 4, v, 1, 1, _lib.pvec([]), None, 0,
                               None, 0, None)
    assert st == -1
    assert b"null knot map" in lib.flpr_last_error()
