"""GPU: the CG dipole solve (FP64 and mixed) and the mixed-precision engine
against the FP64 oracle run to a tight SCF tolerance."""
import numpy as np
import pytest

from mdff_b200 import _abi, systems
from mdff_b200.engine import ForceEngine
from mdff_b200.params import params_copy

from .gpu_util import compare, forces, rel, rms_rel

pytestmark = pytest.mark.gpu


def _pim_cases():
    return [
        systems.random_ionic((24, 24), L=13.0, seed=51, calc=_abi.CALC_OTHER, conv_tol_ind=1e-13,
                             max_scf_pol_iter=500,
                             ldip_damping={(1, 0, 1): 1}, pol_damp_b={(1, 0, 1): 3.0},
                             pol_damp_c={(1, 0, 1): 1.0}, pol_damp_k={(1, 0, 1): 4}),
        systems.mgo(ncell=2, calc=_abi.CALC_OTHER, conv_tol_ind=1e-13, max_scf_pol_iter=500),
        systems.sio2(nsio2=150, seed=9, calc=_abi.CALC_OTHER, conv_tol_ind=1e-13,
                     max_scf_pol_iter=500),
    ]


@pytest.mark.parametrize("case", range(3))
def test_cg_fp64_matches_converged_scf(oracle, case):
    s = _pim_cases()[case]
    o = oracle.Oracle(s.params, s.cell).engforce(*s.soa())
    p = params_copy(s.params)
    p.solver = _abi.SOLVER_CG
    p.cg_tol = 1e-12
    with ForceEngine(p, s.cell) as eng:
        g = eng.engforce(*s.soa())
        st = eng.stats()
    assert st["converged"] and st["n_pol_iter"] < o["n_scf"]
    compare(g, o, 1e-9)


@pytest.mark.parametrize("case", range(3))
def test_mixed_precision_force_error(oracle, case):
    """The mixed engine's bar: force error <= 1e-5 relative RMS vs the FP64 oracle."""
    s = _pim_cases()[case]
    o = oracle.Oracle(s.params, s.cell).engforce(*s.soa())
    p = params_copy(s.params)
    p.solver = _abi.SOLVER_CG
    p.cg_tol = 1e-10
    p.precision = _abi.PREC_MIXED
    with ForceEngine(p, s.cell) as eng:
        g = eng.engforce(*s.soa())
    e_f = rms_rel(forces(g), forces(o))
    e_mu = rms_rel(g["mu"], o["mu"])
    e_u = abs(g["u_coul"] - o["u_coul"]) / abs(o["u_coul"])
    assert e_f <= 1e-5, e_f
    assert e_mu <= 1e-5, e_mu
    assert e_u <= 1e-6, e_u


def test_mixed_precision_nacl(oracle):
    s = systems.nacl(ncell=2, kmax=6)
    o = oracle.Oracle(s.params, s.cell).engforce(*s.soa())
    p = params_copy(s.params)
    p.precision = _abi.PREC_MIXED
    with ForceEngine(p, s.cell) as eng:
        g = eng.engforce(*s.soa())
    assert rms_rel(forces(g), forces(o)) <= 1e-5
    assert abs(g["u_coul"] - o["u_coul"]) / abs(o["u_coul"]) <= 1e-6


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_cg_md_sequence_matches_oracle(oracle, prec):
    """An MD sequence with the CG solver and the ASPC predictor (calc md): the
    static pass merged into the first FP64 residual, the order ramp on the
    launch-by-launch path and the whole-step graph after it.  Every step
    against the oracle's SCF on the same positions and history: FP64 to
    1e-9, mixed within the 1e-5 force bar; the ASPC history at the end."""
    s = systems.sio2(nsio2=150, seed=9, calc=_abi.CALC_MD, conv_tol_ind=1e-12,
                     max_scf_pol_iter=500, extrapolate_order=2)
    orc = oracle.Oracle(params_copy(s.params), s.cell)
    p = params_copy(s.params)
    p.solver = _abi.SOLVER_CG
    p.cg_tol = 1e-12
    p.cg_max_iter = 500
    if prec == "mixed":
        p.precision = _abi.PREC_MIXED
    rng = np.random.default_rng(5)
    pos = s.pos.copy()
    with ForceEngine(p, s.cell) as eng:
        for itime in range(8):
            soa = tuple(np.ascontiguousarray(pos[:, a]) for a in range(3))
            g = eng.engforce(*soa, itime=itime)
            o = orc.engforce(*soa, itime=itime)
            if prec == "fp64":
                compare(g, o, 1e-9)
            else:
                assert rms_rel(forces(g), forces(o)) <= 1e-5, itime
                assert rms_rel(g["mu"], o["mu"]) <= 1e-5, itime
            pos = pos + rng.uniform(-0.01, 0.01, pos.shape)
        h = eng.aspc_history()
    ho = orc.get_aspc()
    assert rel(h, ho) <= (1e-9 if prec == "fp64" else 1e-5)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_split_polarisable_blocks_md_sequence(oracle, prec):
    """Polarisable ions in two type blocks with a non-polarisable block between
    them (types: polarisable anion, cation, polarisable anion), so the ion map
    of the dipole solve's fields and the ion slots of the tensor-core structure
    factor are not one index range; an MD sequence with the CG solver and the
    ASPC predictor (merged first residual, force-pass structure factor from
    the solve's accumulation) against the oracle at every step: FP64 to 1e-9,
    mixed within the 1e-5 force bar."""
    s = systems.random_ionic((20, 30, 20), L=13.0, seed=17, q=(-1.5, 2.0, -1.5), pol=(1.1, 0.0, 1.1),
                             calc=_abi.CALC_MD, conv_tol_ind=1e-12, max_scf_pol_iter=500,
                             extrapolate_order=2)
    orc = oracle.Oracle(params_copy(s.params), s.cell)
    p = params_copy(s.params)
    p.solver = _abi.SOLVER_CG
    p.cg_tol = 1e-12
    p.cg_max_iter = 500
    if prec == "mixed":
        p.precision = _abi.PREC_MIXED
    rng = np.random.default_rng(23)
    pos = s.pos.copy()
    with ForceEngine(p, s.cell) as eng:
        for itime in range(6):
            soa = tuple(np.ascontiguousarray(pos[:, a]) for a in range(3))
            g = eng.engforce(*soa, itime=itime)
            o = orc.engforce(*soa, itime=itime)
            if prec == "fp64":
                compare(g, o, 1e-9)
            else:
                assert rms_rel(forces(g), forces(o)) <= 1e-5, itime
                assert rms_rel(g["mu"], o["mu"]) <= 1e-5, itime
                assert abs(g["u_coul"] - o["u_coul"]) <= 1e-6 * abs(o["u_coul"]), itime
            pos = pos + rng.uniform(-0.01, 0.01, pos.shape)
