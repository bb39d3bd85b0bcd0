"""mdff_gpu_verlet_half_list_noalloc: the half Verlet list for callers that
cannot allocate device memory (its scratch is one static device array).

Its output must equal the existing mdff_gpu_verlet_half_list (which runs on
a handle with allocated buffers) exactly, on two calls in a row, and a call
on a different system in between must leave no trace (the shared array keeps
the previous call's contents).  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from mdff_b200 import _abi, systems
from mdff_b200.engine import ForceEngine
from mdff_b200.params import params_copy

pytestmark = pytest.mark.gpu


def _noalloc(lib, s, which, capacity=None):
    n = s.natm
    cap = capacity if capacity is not None else n * 2000
    point = np.zeros(n + 1, dtype=np.int32)
    lst = np.zeros(max(cap, 1), dtype=np.int32)
    nout = ctypes.c_int(0)
    rx, ry, rz = s.soa()
    A = np.ascontiguousarray(s.cell, dtype=np.float64).reshape(9)
    st = lib.mdff_gpu_verlet_half_list_noalloc(
        ctypes.byref(s.params), _abi.dptr(A), which, _abi.dptr(rx), _abi.dptr(ry), _abi.dptr(rz),
        _abi.iptr(point), _abi.iptr(lst), cap, ctypes.byref(nout))
    return st, point, lst[: min(nout.value, cap)].copy(), nout.value


def _cases():
    return [systems.sio2(nsio2=400, seed=12),
            systems.random_ionic((90, 110), L=19.0, seed=13, triclinic=True)]


def test_noalloc_list_matches_existing_entry_point_twice():
    lib = _abi.load_library()
    cases = _cases()
    expected = {}
    for ci, s in enumerate(cases):
        with ForceEngine(params_copy(s.params), s.cell) as eng:
            for which in (0, 1):
                expected[ci, which] = eng.verlet_half_list(*s.soa(), which=which)
    for rep in range(2):                      # two calls in a row ...
        for ci, s in enumerate(cases):        # ... with another system in between
            for which in (0, 1):
                st, point, lst, n = _noalloc(lib, s, which)
                est, epoint, elst, en = expected[ci, which]
                assert st == 0 and est == 0
                assert n == en
                assert np.array_equal(point, epoint)
                assert np.array_equal(lst, elst)


def test_noalloc_reports_short_capacity_and_size_limit():
    lib = _abi.load_library()
    s = _cases()[1]
    st, point, lst, n = _noalloc(lib, s, 1, capacity=100)
    assert st == _abi.MDFF_ERR_LIST_OVERFLOW and n > 100 and len(lst) == 100
    big = params_copy(s.params)
    big.natm = 40000                          # beyond the static scratch limit
    big.natmi[0] = 40000 - big.natmi[1]
    z = np.zeros(40000)
    A = np.ascontiguousarray(s.cell, dtype=np.float64).reshape(9)
    point = np.zeros(40001, dtype=np.int32)
    nout = ctypes.c_int(0)
    st = lib.mdff_gpu_verlet_half_list_noalloc(ctypes.byref(big), _abi.dptr(A), 1, _abi.dptr(z),
                                               _abi.dptr(z), _abi.dptr(z), _abi.iptr(point), None,
                                               0, ctypes.byref(nout))
    assert st == _abi.MDFF_ERR_BAD_ARGS
