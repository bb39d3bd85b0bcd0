"""Python host mirror of the engforce boundary (include/mdff_gpu.h).

``ForceEngine(params, cell)`` is what the reference's Fortran ``engforce``
(engforce_driver.f90:102-190) becomes behind the C ABI: create once with the
force field and cell, then call :meth:`engforce` every step with positions.
Errors surface as :class:`MdffError` with the library's status code, the
equivalents of the reference's STOPs (polarisation catastrophe,
moment_from_pola.f90:176-216; list overflow, tools.f90:337-350).
"""
import ctypes

import numpy as np

from . import _abi
from ._abi import MdffError, dptr, iptr


def _mat(m):
    return np.array([[m[a][b] for b in range(3)] for a in range(3)])


class ForceEngine:
    def __init__(self, params, cell):
        self._lib = _abi.load_library()
        self.params = params
        self.natm = params.natm
        A = np.ascontiguousarray(cell, dtype=np.float64).reshape(9)
        h = ctypes.c_void_p()
        st = self._lib.mdff_gpu_create(ctypes.byref(params), dptr(A), ctypes.byref(h))
        if st != 0:
            msg = self._lib.mdff_gpu_last_error(None).decode()
            raise MdffError(st, f"create: {self._lib.mdff_gpu_strerror(st).decode()} ({msg})")
        self._h = h

    # -- lifetime -------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.mdff_gpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st, what, allow=()):
        if st != 0 and st not in allow:
            msg = self._lib.mdff_gpu_last_error(self._h).decode()
            raise MdffError(st, f"{what}: {self._lib.mdff_gpu_strerror(st).decode()} {msg}")
        return st

    # -- the boundary -----------------------------------------------------------
    def set_cell(self, cell):
        A = np.ascontiguousarray(cell, dtype=np.float64).reshape(9)
        self._check(self._lib.mdff_gpu_set_cell(self._h, dptr(A)), "set_cell")

    def engforce(self, rx, ry, rz, itime=0, want_mu=True, want_ef=True, allow_status=()):
        """One engforce call on host arrays.  Returns a dict with fx, fy, fz,
        mu (natm,3), ef (natm,3), the thermodynamic scalars and 3x3 tensors."""
        n = self.natm
        rx, ry, rz = (np.ascontiguousarray(a, dtype=np.float64) for a in (rx, ry, rz))
        out = {k: np.zeros(n) for k in ("fx", "fy", "fz")}
        r = _abi.MdffResult()
        r.fx, r.fy, r.fz = (dptr(out[k]) for k in ("fx", "fy", "fz"))
        if want_mu:
            out["mu"] = np.zeros((n, 3))
            r.mu = dptr(out["mu"])
        if want_ef:
            out["ef"] = np.zeros((n, 3))
            r.ef = dptr(out["ef"])
        st = self._lib.mdff_gpu_engforce(self._h, dptr(rx), dptr(ry), dptr(rz), int(itime),
                                         ctypes.byref(r))
        out["status"] = self._check(st, "engforce", allow_status)
        for k in ("u_lj", "vir_lj", "u_bmhft", "vir_bmhft", "u_coul", "u_pol", "pvirial_coul"):
            out[k] = getattr(r, k)
        for k in ("tau_nonb", "tau_coul", "tau"):
            out[k] = _mat(getattr(r, k))
        return out

    def engforce_device(self, d_pos, d_force, d_mu=0, d_ef=0, itime=0):
        """engforce on device pointers (ints, e.g. torch ``data_ptr()``)."""
        r = _abi.MdffResult()
        st = self._lib.mdff_gpu_engforce_device(self._h, ctypes.c_void_p(d_pos), int(itime),
                                                ctypes.c_void_p(d_force), ctypes.c_void_p(d_mu or None),
                                                ctypes.c_void_p(d_ef or None), ctypes.byref(r))
        self._check(st, "engforce_device")
        out = {k: getattr(r, k) for k in ("u_lj", "vir_lj", "u_bmhft", "vir_bmhft", "u_coul",
                                         "u_pol", "pvirial_coul")}
        for k in ("tau_nonb", "tau_coul", "tau"):
            out[k] = _mat(getattr(r, k))
        return out

    def md_nve(self, d_pos, d_vel, d_invmass, dt, nsteps, itime0=0, energies=True):
        e = np.zeros((max(nsteps, 1), 2)) if energies else None
        st = self._lib.mdff_gpu_md_nve(self._h, ctypes.c_void_p(d_pos), ctypes.c_void_p(d_vel),
                                       ctypes.c_void_p(d_invmass), float(dt), int(nsteps),
                                       int(itime0), dptr(e) if energies else None)
        self._check(st, "md_nve")
        return e

    def stats(self):
        s = _abi.MdffStats()
        self._check(self._lib.mdff_gpu_get_stats(self._h, ctypes.byref(s)), "stats")
        return {f: (list(getattr(s, f)) if f == "kES" else getattr(s, f)) for f, _ in s._fields_}

    def aspc_history(self):
        b = np.zeros((_abi.ASPC_DEPTH, self.natm, 3))
        self._check(self._lib.mdff_gpu_get_aspc_history(self._h, dptr(b)), "get_aspc_history")
        return b

    def set_aspc_history(self, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        self._check(self._lib.mdff_gpu_set_aspc_history(self._h, dptr(b)), "set_aspc_history")

    def verlet_half_list(self, rx, ry, rz, which, capacity=None):
        n = self.natm
        cap = capacity if capacity is not None else n * 2000
        point = np.zeros(n + 1, dtype=np.int32)
        lst = np.zeros(max(cap, 1), dtype=np.int32)
        nout = ctypes.c_int(0)
        rx, ry, rz = (np.ascontiguousarray(a, dtype=np.float64) for a in (rx, ry, rz))
        st = self._lib.mdff_gpu_verlet_half_list(self._h, int(which), dptr(rx), dptr(ry), dptr(rz),
                                                 iptr(point), iptr(lst), int(cap), ctypes.byref(nout))
        return st, point, lst[: min(nout.value, cap)].copy(), nout.value
