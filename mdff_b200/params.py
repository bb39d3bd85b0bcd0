"""Force-field parameters with the reference's namelist defaults.

``make_params(natmi, **keywords)`` fills an :class:`MdffParams` the way the
reference's ``*_default_tag`` routines followed by a namelist read would:

* control_default_tag (control.f90:201-245)
* non_bonded_default_tag (non_bonded.f90:169-201)
* coulomb_default_tag (coulomb.f90:152-181)
* pim_default_tag (pim.f90:107-140)

Keyword names are the namelist names.  Per-type tables are given as dicts
keyed by 0-based type tuples, e.g. ``Abmhftd={(0, 1): 1312.9}``, or as
numpy arrays.  New ``&gputag`` keywords: precision, solver, cg_tol,
cg_max_iter, fail_on_nonconvergence, device, wall24.  Thole functions:
thole_type (MDFF_THOLE_*) and thole_param (per ordered type pair).  Dipole
algorithms: algo_moment_from_pola (MDFF_ALGO_*), algo_ext_dipole (MDFF_EXT_*)
and omegakO.  Wannier centres: lwfc (per type), ldip_wfc, rcut_wfc.
"""
import numpy as np

from . import _abi

NT = _abi.NT

_DEFAULTS = dict(
    # &controltag
    lcoulomb=0, lbmhft=0, lbmhftd=0, lnmlj=0, lsurf=0, lreduced=0,
    calc=_abi.CALC_MD, cutshortrange=0.0, cutlongrange=0.0, skindiff=0.15,
    # &non_bondedtag
    trunc=_abi.TRUNC_NONE, symmetric_pot_nb=1,
    # &coulombtag
    alphaES=1.0, kES=(10, 10, 10), lautoES=0, epsw=1e-6, thole_type=_abi.THOLE_NONE,
    # &pimtag
    conv_tol_ind=1e-6, min_scf_pol_iter=3, max_scf_pol_iter=100,
    extrapolate_order=0, symmetric_pot_pim=1, algo_moment_from_pola=_abi.ALGO_SCF,
    algo_ext_dipole=_abi.EXT_ASPC, omegakO=0.7, ldip_wfc=1, rcut_wfc=0.5,
    # &gputag
    precision=_abi.PREC_FP64, solver=_abi.SOLVER_SCF, cg_tol=0.0, cg_max_iter=200,
    fail_on_nonconvergence=0, device=0,
)

_TABLE2 = ("epslj", "sigmalj", "plj", "qlj", "Abmhftd", "Bbmhftd", "Cbmhftd",
           "Dbmhftd", "BDbmhftd", "wall24", "thole_param")
_TABLE3 = ("ldip_damping", "pol_damp_b", "pol_damp_c", "pol_damp_k")


def _fill(arr_field, value, shape, dtype):
    a = np.zeros(shape, dtype=dtype)
    if isinstance(value, dict):
        for k, v in value.items():
            a[k] = v
    elif value is not None:
        v = np.asarray(value, dtype=dtype)
        a[tuple(slice(0, s) for s in v.shape)] = v
    flat = a.ravel()
    dst = np.ctypeslib.as_array(arr_field).reshape(-1)
    dst[:] = flat
    return a


def make_params(natmi, **kw):
    """Build an MdffParams.  ``natmi`` = ions per type in POSFF order."""
    p = _abi.MdffParams()
    natmi = list(natmi)
    p.ntype = len(natmi)
    p.natm = int(sum(natmi))
    for i, n in enumerate(natmi):
        p.natmi[i] = n
    # LJ defaults qlj = 12, plj = 6 (non_bonded.f90:180-181)
    kw.setdefault("qlj", np.full((NT, NT), 12.0))
    kw.setdefault("plj", np.full((NT, NT), 6.0))
    # thole_param = 1.662 (coulomb.f90:175)
    kw.setdefault("thole_param", np.full((NT, NT), 1.662))
    unknown = set(kw) - set(_DEFAULTS) - set(_TABLE2) - set(_TABLE3) - {
        "qch", "dip", "ldip_polar", "poldip", "poldip_iso", "lwfc"}
    if unknown:
        raise KeyError(f"unknown keywords: {sorted(unknown)}")
    for k, v in _DEFAULTS.items():
        val = kw.get(k, v)
        if k == "kES":
            for i in range(3):
                p.kES[i] = int(val[i])
        else:
            setattr(p, k, val)
    _fill(p.qch, kw.get("qch"), (NT,), np.float64)
    _fill(p.dip, kw.get("dip"), (NT, 3), np.float64)
    for name in _TABLE2:
        _fill(getattr(p, name), kw.get(name), (NT, NT), np.float64)
    for name in _TABLE3:
        dt = np.int32 if name in ("ldip_damping", "pol_damp_k") else np.float64
        _fill(getattr(p, name), kw.get(name), (NT, NT, NT), dt)
    _fill(p.ldip_polar, kw.get("ldip_polar"), (NT,), np.int32)
    _fill(p.lwfc, kw.get("lwfc"), (NT,), np.int32)
    pol = np.zeros((NT, 3, 3))
    if kw.get("poldip") is not None:
        src = kw["poldip"]
        if isinstance(src, dict):
            for k, v in src.items():
                pol[k] = v
        else:
            src = np.asarray(src, dtype=np.float64)
            pol[: src.shape[0]] = src
    # poldip_iso (pim.f90:219-231): isotropic tensor from a scalar
    if kw.get("poldip_iso") is not None:
        for it, a in dict(kw["poldip_iso"]).items():
            if a != 0.0:
                pol[it] = np.eye(3) * a
    _fill(p.poldip, pol, (NT, 3, 3), np.float64)
    return p


def params_copy(p):
    q = _abi.MdffParams()
    import ctypes
    ctypes.memmove(ctypes.byref(q), ctypes.byref(p), ctypes.sizeof(p))
    return q


def itype_of(p):
    """Per-ion 0-based type array (read_pos.f90:187-199: grouped by type)."""
    return np.repeat(np.arange(p.ntype), [p.natmi[i] for i in range(p.ntype)]).astype(np.int32)


def charges_of(p):
    return np.array([p.qch[t] for t in itype_of(p)], dtype=np.float64)
