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

from .gpu_util import cells_per_axis, sio2_prepared

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
    """Boxes with 2 cells per axis (every cell scanned) and with 4 and 5 cells
    per axis (the periodic 3x3x3 stencil of the device build)."""
    return [systems.sio2(nsio2=400, seed=12),
            systems.random_ionic((90, 110), L=19.0, seed=13, triclinic=True),
            systems.random_ionic((600, 600), L=30.0, seed=14, triclinic=True),
            sio2_prepared()]


def test_noalloc_list_matches_existing_entry_point_twice():
    lib = _abi.load_library()
    cases = _cases()
    assert [min(cells_per_axis(s, 1)) for s in cases] == [2, 2, 4, 5]
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


def test_noalloc_static_entry_limit_is_not_a_capacity_overflow():
    """More half-list entries than the static array holds (4,194,304) is a
    hard limit with its own status, not the grow-and-retry overflow."""
    lib = _abi.load_library()
    rng = np.random.default_rng(15)
    n, L = 20000, 60.0                        # about 8.5e6 entries within 13 A
    s = systems.random_ionic((4, 4), L=L, seed=15)
    p = params_copy(s.params)
    p.natm = n
    p.natmi[0] = n // 2
    p.natmi[1] = n - n // 2
    p.cutlongrange = 12.3
    p.skindiff = 0.7
    pos = rng.uniform(0.0, L, (n, 3))
    A = np.ascontiguousarray(np.eye(3) * L).reshape(9)
    point = np.zeros(n + 1, dtype=np.int32)
    nout = ctypes.c_int(0)
    rx, ry, rz = (np.ascontiguousarray(pos[:, a]) for a in range(3))
    st = lib.mdff_gpu_verlet_half_list_noalloc(ctypes.byref(p), _abi.dptr(A), 1, _abi.dptr(rx),
                                               _abi.dptr(ry), _abi.dptr(rz), _abi.iptr(point), None,
                                               0, ctypes.byref(nout))
    assert st == _abi.MDFF_ERR_BAD_ARGS
    assert nout.value > 4 * 1024 * 1024
