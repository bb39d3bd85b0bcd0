"""Shared helpers of the GPU parity tests: compare the CUDA engine with the
CPU oracle on the same seeded inputs."""
import numpy as np

from mdff_b200 import params as P, systems


def rel(a, b):
    """max |a-b| / max |b| (0 if both vanish)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).max() if b.size else 0.0
    num = np.abs(a - b).max() if b.size else 0.0
    if den == 0.0:
        return num
    return num / den


def rms_rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def forces(r):
    return np.stack([r["fx"], r["fy"], r["fz"]], 1)


def compare(g, o, tol, keys_scalar=("u_bmhft", "u_lj", "u_coul", "u_pol", "vir_bmhft"),
            check_ef=True, check_mu=True):
    """Assert GPU result g agrees with oracle result o to relative tol."""
    errs = {}
    errs["f"] = rel(forces(g), forces(o))
    for k in keys_scalar:
        if abs(o[k]) > 0:
            errs[k] = abs(g[k] - o[k]) / abs(o[k])
        else:
            errs[k] = abs(g[k])
    for k in ("tau_nonb", "tau_coul"):
        errs[k] = rel(g[k], o[k])
    if check_mu and "mu" in g:
        errs["mu"] = rel(g["mu"], o["mu"])
    if check_ef and "ef" in g:
        errs["ef"] = rel(g["ef"], o["ef"])
    bad = {k: v for k, v in errs.items() if not (v <= tol)}
    assert not bad, f"errors above {tol}: {bad}"
    return errs


def small_systems():
    """Parity cases at sizes the oracle finishes in seconds."""
    out = []
    for tag in ("twocharges", "twodipoles", "twocharges_twopola"):
        out.append(systems.ex04(tag))
    dampkw = dict(ldip_damping={(1, 0, 1): 1, (1, 1, 1): 1},
                  pol_damp_b={(1, 0, 1): 3.0, (1, 1, 1): 4.1},
                  pol_damp_c={(1, 0, 1): 1.0, (1, 1, 1): 1.7},
                  pol_damp_k={(1, 0, 1): 4, (1, 1, 1): 3})
    out.append(systems.random_ionic((24, 24), L=13.0, seed=21, calc=P._abi.CALC_OTHER, **dampkw))
    out.append(systems.random_ionic((20, 28), L=13.5, seed=22, triclinic=True,
                                    q=(1.2, -0.857142857142857), calc=P._abi.CALC_OTHER, **dampkw))
    out.append(systems.nacl(ncell=2, rcut=12.0, kmax=6))
    out.append(systems.nacl(ncell=2, rcut=12.0, kmax=6, lbmhft=0, lbmhftd=1,
                            BDbmhftd={(0, 0): 3.1, (0, 1): 2.9, (1, 1): 2.7}))
    ljkw = dict(lbmhft=0, lnmlj=1, trunc=2, epslj={(0, 0): 0.01, (0, 1): 0.02, (1, 1): 0.015},
                sigmalj={(0, 0): 2.0, (0, 1): 2.2, (1, 1): 2.6},
                qlj={(0, 0): 12.0, (0, 1): 10.0, (1, 1): 12.0}, plj={(0, 0): 6.0, (0, 1): 5.0, (1, 1): 6.0})
    out.append(systems.random_ionic((16, 16), L=12.0, seed=23, pol=(0.0, 0.0), **ljkw))
    both = dict(ljkw, lbmhft=1, trunc=1)
    out.append(systems.random_ionic((16, 16), L=12.0, seed=24, pol=(0.0, 0.0), **both))
    out.append(systems.mgo(ncell=2, calc=P._abi.CALC_OTHER, conv_tol_ind=1e-12))
    out.append(systems.sio2(nsio2=120, seed=8, calc=P._abi.CALC_OTHER, conv_tol_ind=1e-12))
    return out


def sio2_prepared():
    """The 12,000-ion SiO2-like glass at its prepared state
    (tests/golden/sio2_state.npz, written by make_bench_states.py)."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "sio2_state.npz"))
    s = systems.sio2(place=False)
    assert int(z["natm"]) == s.natm and np.allclose(z["cell"], s.cell)
    s.pos = np.array(z["pos"])
    s.vel = np.array(z["vel"])
    return s


def config_systems(**extra):
    """The three single-box workloads at their full sizes: SiO2-like glass
    12,000 ions (PIM + TT, kmax 12), MgO 8,000 ions (PIM + TT, kmax from
    ewald_param at epsw 1e-7), molten NaCl 1,728 ions (BMH + Ewald)."""
    kw = dict(calc=P._abi.CALC_OTHER)
    kw.update(extra)
    s = sio2_prepared()
    for k, v in kw.items():
        setattr(s.params, k, v)
    return {"sio2_12000": s, "mgo_8000": systems.mgo(**kw), "nacl_1728": systems.nacl(**kw)}


def cells_per_axis(s, which):
    """Cells per axis of the device list build for system s: the face widths
    over the build cutoff (the larger of the two lists' cut + skin)."""
    A = np.asarray(s.cell, dtype=np.float64)
    B = np.linalg.inv(A).T * np.linalg.det(A)
    om = abs(np.linalg.det(A))
    W = om / np.linalg.norm(B, axis=0)
    p = s.params
    rc = p.cutlongrange
    if p.lcoulomb:
        rc = min(rc, 0.5 * W.min())
    rs = max(rc if p.lcoulomb else 0.0, p.cutshortrange if (p.lbmhft or p.lbmhftd or p.lnmlj) else 0.0)
    rs += p.skindiff
    return [int(np.floor(w / (rs * (1 + 1e-9) + 1e-9))) for w in W]
