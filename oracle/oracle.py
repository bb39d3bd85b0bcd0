"""ctypes wrapper of the CPU oracle (liboracle: mdff_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import this module;
the product package (mdff_b200) never does.
"""
import ctypes
import os
import subprocess

import numpy as np

from mdff_b200 import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "libmdff_oracle.so")
_lib = None


class SetupInfo(ctypes.Structure):
    _fields_ = [("alphaES", ctypes.c_double), ("kES", ctypes.c_int * 3), ("nk", ctypes.c_int),
                ("cutlongrange", ctypes.c_double), ("B", ctypes.c_double * 9),
                ("omega", ctypes.c_double), ("WA", ctypes.c_double), ("WB", ctypes.c_double),
                ("WC", ctypes.c_double), ("task", ctypes.c_int * 6)]


class Extra(ctypes.Structure):
    _fields_ = [("efg", ctypes.POINTER(ctypes.c_double)), ("do_efg", ctypes.c_int),
                ("n_scf", ctypes.c_int), ("rmsd", ctypes.c_double),
                ("u_dir", ctypes.c_double), ("u_rec", ctypes.c_double),
                ("u_self", ctypes.c_double), ("u_surf", ctypes.c_double),
                ("n_kardir", ctypes.c_int)]


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        P = ctypes.c_void_p
        DP = ctypes.POINTER(ctypes.c_double)
        IP = ctypes.POINTER(ctypes.c_int)
        L.or_create.restype = P
        L.or_create.argtypes = [ctypes.POINTER(_abi.MdffParams), DP, IP]
        L.or_destroy.argtypes = [P]
        L.or_set_threads.argtypes = [ctypes.c_int]
        L.or_get_threads.restype = ctypes.c_int
        L.or_engforce.restype = ctypes.c_int
        L.or_engforce.argtypes = [P, DP, DP, DP, ctypes.c_int, ctypes.POINTER(_abi.MdffResult),
                                  ctypes.POINTER(Extra)]
        L.or_vnlist.restype = ctypes.c_int
        L.or_vnlist.argtypes = [P, DP, DP, DP, ctypes.c_int, IP, IP, ctypes.c_int, IP]
        L.or_vnlistcheck.restype = ctypes.c_int
        L.or_vnlistcheck.argtypes = [P, DP, DP, DP, DP, IP]
        L.or_kardir_roundtrips.argtypes = [P, DP, DP, DP, ctypes.c_int]
        L.or_kardir_roundtrips.restype = None
        L.or_get_aspc.argtypes = [P, DP]
        L.or_set_aspc.argtypes = [P, DP]
        L.or_get_setup.argtypes = [P, ctypes.POINTER(SetupInfo)]
        L.or_get_kmesh.argtypes = [P, DP, DP, DP, DP, DP, DP]
        L.or_errfc.restype = ctypes.c_double
        L.or_polint.restype = ctypes.c_double
        L.or_polint.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), ctypes.c_int]
        L.or_errfc.argtypes = [ctypes.c_double]
        L.or_tt_damp.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                 DP, DP]
        _lib = L
    return _lib


def set_threads(n):
    lib().or_set_threads(int(n))


def errfc(x):
    return lib().or_errfc(float(x))


def polint(xa, ya):
    """polint of the reference at x = 1 through the points (xa, ya)."""
    xa = np.ascontiguousarray(xa, dtype=np.int32)
    ya = np.ascontiguousarray(ya, dtype=np.float64)
    assert xa.size == ya.size <= 10
    return lib().or_polint(xa.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                           ya.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(xa.size))


def tt_damp(b, c, r, order):
    f = ctypes.c_double()
    fd = ctypes.c_double()
    lib().or_tt_damp(b, c, r, order, ctypes.byref(f), ctypes.byref(fd))
    return f.value, fd.value


class Oracle:
    """CPU FP64 engforce over the same mdff_params as the GPU engine."""

    def __init__(self, params, cell_A):
        self.params = params
        self.natm = params.natm
        st = ctypes.c_int(0)
        A = np.ascontiguousarray(cell_A, dtype=np.float64).reshape(9)
        self._h = lib().or_create(ctypes.byref(params), _abi.dptr(A), ctypes.byref(st))
        if not self._h:
            raise _abi.MdffError(st.value, "oracle create failed")

    def close(self):
        if self._h:
            lib().or_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def setup(self):
        s = SetupInfo()
        lib().or_get_setup(self._h, ctypes.byref(s))
        return s

    def kmesh(self):
        nk = self.setup().nk
        arrs = [np.zeros(nk) for _ in range(6)]
        lib().or_get_kmesh(self._h, *[_abi.dptr(a) for a in arrs])
        return dict(zip(("kx", "ky", "kz", "kk", "Ak", "kcoe"), arrs))

    def engforce(self, rx, ry, rz, itime=0, efg=False, check=True):
        n = self.natm
        rx, ry, rz = (np.ascontiguousarray(a, dtype=np.float64) for a in (rx, ry, rz))
        out = {k: np.zeros(n) for k in ("fx", "fy", "fz")}
        out["mu"] = np.zeros((n, 3))
        out["ef"] = np.zeros((n, 3))
        r = _abi.MdffResult()
        r.fx, r.fy, r.fz = (_abi.dptr(out[k]) for k in ("fx", "fy", "fz"))
        r.mu = _abi.dptr(out["mu"])
        r.ef = _abi.dptr(out["ef"])
        ex = Extra()
        if efg:
            out["efg"] = np.zeros((n, 3, 3))
            ex.efg = _abi.dptr(out["efg"])
            ex.do_efg = 1
        st = lib().or_engforce(self._h, _abi.dptr(rx), _abi.dptr(ry), _abi.dptr(rz), int(itime),
                               ctypes.byref(r), ctypes.byref(ex))
        if check and st != 0:
            raise _abi.MdffError(st, "oracle engforce")
        out["status"] = st
        for k in ("u_lj", "vir_lj", "u_bmhft", "vir_bmhft", "u_coul", "u_pol", "pvirial_coul"):
            out[k] = getattr(r, k)
        for k in ("tau_nonb", "tau_coul", "tau"):
            out[k] = np.array([[getattr(r, k)[a][b] for b in range(3)] for a in range(3)])
        out["n_scf"] = ex.n_scf
        out["n_kardir"] = ex.n_kardir
        out["rmsd"] = ex.rmsd
        out["u_parts"] = dict(dir=ex.u_dir, rec=ex.u_rec, self=ex.u_self, surf=ex.u_surf)
        return out

    def kardir_roundtrips(self, rx, ry, rz, count):
        """The positions after ``count`` in-place kardir/dirkar round trips
        (lattice.f90:183-270), as new arrays."""
        rx, ry, rz = (np.array(a, dtype=np.float64) for a in (rx, ry, rz))
        lib().or_kardir_roundtrips(self._h, _abi.dptr(rx), _abi.dptr(ry), _abi.dptr(rz), int(count))
        return rx, ry, rz

    def vnlist(self, rx, ry, rz, which, capacity=None):
        n = self.natm
        cap = capacity if capacity is not None else n * 2000
        point = np.zeros(n + 1, dtype=np.int32)
        lst = np.zeros(max(cap, 1), dtype=np.int32)
        nout = ctypes.c_int(0)
        rx, ry, rz = (np.ascontiguousarray(a, dtype=np.float64) for a in (rx, ry, rz))
        st = lib().or_vnlist(self._h, _abi.dptr(rx), _abi.dptr(ry), _abi.dptr(rz), int(which),
                             _abi.iptr(point), _abi.iptr(lst), int(cap), ctypes.byref(nout))
        return st, point, lst[: min(nout.value, cap)].copy(), nout.value

    def vnlistcheck(self, rx, ry, rz):
        """vnlistcheck (tools.f90:444-537) against the direct coordinates of
        the last rebuild (zero before the first): returns (rebuilt, disp)
        with disp = largest + second largest displacement."""
        rx, ry, rz = (np.ascontiguousarray(a, dtype=np.float64) for a in (rx, ry, rz))
        d = ctypes.c_double(0.0)
        r = ctypes.c_int(0)
        lib().or_vnlistcheck(self._h, _abi.dptr(rx), _abi.dptr(ry), _abi.dptr(rz), ctypes.byref(d),
                             ctypes.byref(r))
        return bool(r.value), d.value

    def get_aspc(self):
        b = np.zeros((_abi.ASPC_DEPTH, self.natm, 3))
        lib().or_get_aspc(self._h, _abi.dptr(b))
        return b

    def set_aspc(self, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        lib().or_set_aspc(self._h, _abi.dptr(b))
