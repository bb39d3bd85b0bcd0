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

    def efg(self):
        """Electric field gradient [natm, 3, 3] for the state of the last
        engforce (the reference's efg_t)."""
        e = np.zeros((self.natm, 3, 3))
        self._check(self._lib.mdff_gpu_efg(self._h, dptr(e)), "efg")
        return e

    def set_tc_wait_limit(self, polls):
        """Test hook of the timeout path (mdff_gpu_set_tc_wait_limit): polls of
        the tensor-core structure factor's operand-stage wait; < 0 = default."""
        self._check(self._lib.mdff_gpu_set_tc_wait_limit(self._h, int(polls)), "set_tc_wait_limit")

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

    def kardir_roundtrips(self, rx, ry, rz, count=None):
        """The positions after the reference's in-place kardir/dirkar round
        trips (lattice.f90:183-270), as new arrays: ``count`` of them, by
        default the number the reference's engforce made for the last call
        (``stats()["n_kardir"]``)."""
        if count is None:
            count = self.stats()["n_kardir"]
            if count < 0:
                raise ValueError("the last call's solve is not the reference's SCF")
        rx, ry, rz = (np.array(a, dtype=np.float64) for a in (rx, ry, rz))
        self._check(self._lib.mdff_gpu_kardir_roundtrips(self._h, dptr(rx), dptr(ry), dptr(rz),
                                                         int(count)), "kardir_roundtrips")
        return rx, ry, rz

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


class BatchEngine:
    """Many independent configurations per call (include/mdff_gpu.h batched
    entry points): ``BatchEngine(psets, configs)`` with ``configs`` a list of
    (pset index, natmi per type, cell 3x3); :meth:`engforce` takes the
    concatenated positions and returns per-ion arrays plus one dict of
    scalars per configuration.  Each configuration is one engforce with
    calc = 'other'."""

    def __init__(self, psets, configs):
        self._lib = _abi.load_library()
        self.nconf = len(configs)
        np_ = len(psets)
        arr = (_abi.MdffParams * np_)(*psets)
        self._psets = arr
        pset = np.array([c[0] for c in configs], dtype=np.int32)
        natmi = np.zeros((self.nconf, _abi.NT), dtype=np.int32)
        cells = np.zeros((self.nconf, 9))
        for k, (_, ni, cell) in enumerate(configs):
            natmi[k, : len(ni)] = ni
            cells[k] = np.asarray(cell, dtype=np.float64).reshape(9)
        self.natm = natmi.sum(1)
        self.offsets = np.concatenate([[0], np.cumsum(self.natm)])
        self.ntot = int(self.offsets[-1])
        self._keep = (pset, natmi, cells)
        d = _abi.MdffBatchDesc(self.nconf, pset.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                               natmi.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), dptr(cells))
        h = ctypes.c_void_p()
        st = self._lib.mdff_gpu_batch_create(arr, np_, ctypes.byref(d), ctypes.byref(h))
        if st != 0:
            msg = self._lib.mdff_gpu_batch_last_error(None).decode()
            raise MdffError(st, f"batch_create: {self._lib.mdff_gpu_strerror(st).decode()} ({msg})")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mdff_gpu_batch_destroy(self._h)
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
            msg = self._lib.mdff_gpu_batch_last_error(self._h).decode()
            raise MdffError(st, f"{what}: {self._lib.mdff_gpu_strerror(st).decode()} {msg}")
        return st

    @staticmethod
    def _conf_dicts(confs):
        out = []
        for c in confs:
            d = {k: getattr(c, k) for k in ("u_lj", "vir_lj", "u_bmhft", "vir_bmhft", "u_coul",
                                            "u_pol", "pvirial_coul", "rmsd", "n_pol_iter",
                                            "converged", "catastrophe", "nk", "alphaES",
                                            "cutlongrange")}
            d["kES"] = list(c.kES)
            for k in ("tau_nonb", "tau_coul", "tau"):
                d[k] = _mat(getattr(c, k))
            out.append(d)
        return out

    def engforce(self, rx, ry, rz, allow_status=()):
        n = self.ntot
        rx, ry, rz = (np.ascontiguousarray(a, dtype=np.float64) for a in (rx, ry, rz))
        out = {k: np.zeros(n) for k in ("fx", "fy", "fz")}
        out["mu"] = np.zeros((n, 3))
        out["ef"] = np.zeros((n, 3))
        confs = (_abi.MdffBatchConf * self.nconf)()
        st = self._lib.mdff_gpu_batch_engforce(self._h, dptr(rx), dptr(ry), dptr(rz),
                                               dptr(out["fx"]), dptr(out["fy"]), dptr(out["fz"]),
                                               dptr(out["mu"]), dptr(out["ef"]), confs)
        out["status"] = self._check(st, "batch_engforce", allow_status)
        out["conf"] = self._conf_dicts(confs)
        return out

    def engforce_device(self, d_pos, d_force, d_mu=0, d_ef=0):
        confs = (_abi.MdffBatchConf * self.nconf)()
        st = self._lib.mdff_gpu_batch_engforce_device(self._h, ctypes.c_void_p(d_pos),
                                                      ctypes.c_void_p(d_force),
                                                      ctypes.c_void_p(d_mu or None),
                                                      ctypes.c_void_p(d_ef or None), confs)
        self._check(st, "batch_engforce_device")
        return self._conf_dicts(confs)

    def tune(self):
        c, t, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        self._check(self._lib.mdff_gpu_batch_tune(self._h, ctypes.byref(c), ctypes.byref(t),
                                                  ctypes.byref(ms)), "batch_tune")
        return c.value, t.value, ms.value

    def set_shape(self, cluster, threads):
        self._check(self._lib.mdff_gpu_batch_set_shape(self._h, int(cluster), int(threads)),
                    "batch_set_shape")

    def info(self):
        v = [ctypes.c_int() for _ in range(4)]
        ms = ctypes.c_double()
        self._check(self._lib.mdff_gpu_batch_info(self._h, *[ctypes.byref(x) for x in v],
                                                  ctypes.byref(ms)), "batch_info")
        return dict(ntot=v[0].value, nconf=v[1].value, cluster=v[2].value, threads=v[3].value,
                    ms_last=ms.value)

    # -- force-field gradients ---------------------------------------------
    def fit_define(self, params):
        """params: list of (kind, t1, t2) with kinds _abi.FIT_*; returns the
        current values (theta) of those parameters."""
        k = np.array([p[0] for p in params], dtype=np.int32)
        t1 = np.array([p[1] for p in params], dtype=np.int32)
        t2 = np.array([p[2] for p in params], dtype=np.int32)
        self.nparam = len(params)
        self._check(self._lib.mdff_gpu_batch_fit_define(self._h, self.nparam, iptr(k), iptr(t1),
                                                        iptr(t2)), "batch_fit_define")
        return self.fit_get()

    def fit_set(self, theta):
        th = np.ascontiguousarray(theta, dtype=np.float64)
        self._check(self._lib.mdff_gpu_batch_fit_set(self._h, dptr(th)), "batch_fit_set")

    def fit_get(self):
        th = np.zeros(self.nparam)
        self._check(self._lib.mdff_gpu_batch_fit_get(self._h, dptr(th)), "batch_fit_get")
        return th

    def adjoint(self, gE, gF, gmu=None, per_conf=False):
        """dJ/dtheta for host arrays gE [nconf], gF [ntot, 3] (or SoA [3, ntot]),
        gmu [ntot, 3] (optional), at the positions of the last engforce."""
        gE = np.ascontiguousarray(gE, dtype=np.float64)
        gF = np.asarray(gF, dtype=np.float64)
        if gF.shape == (self.ntot, 3):
            gF = gF.T
        gF = np.ascontiguousarray(gF)
        gm = None if gmu is None else np.ascontiguousarray(gmu, dtype=np.float64)
        grad = np.zeros(self.nparam)
        gc = np.zeros((self.nconf, self.nparam)) if per_conf else None
        st = self._lib.mdff_gpu_batch_adjoint(self._h, gE.ctypes.data, gF.ctypes.data,
                                              None if gm is None else gm.ctypes.data, 0,
                                              dptr(grad), dptr(gc) if per_conf else None)
        self._check(st, "batch_adjoint")
        return (grad, gc) if per_conf else grad

    def adjoint_device(self, d_gE, d_gF, d_gmu=0):
        grad = np.zeros(self.nparam)
        st = self._lib.mdff_gpu_batch_adjoint(self._h, ctypes.c_void_p(d_gE), ctypes.c_void_p(d_gF),
                                              ctypes.c_void_p(d_gmu or None), 1, dptr(grad), None)
        self._check(st, "batch_adjoint")
        return grad
