"""Thole functions on the dipole-dipole field and energy (ewald_dir.f90:305-430):
the four variants (linear, expon1, expon2, gauss) of the FP64 engine against
the CPU oracle (the reference's SCF to a tight tolerance) to 1e-9, the mixed
engine (CG) to the 1e-5 force bar, and Thole visibly active; the batched
engine with Thole against the same oracle (its fit gradient rejects Thole)."""
import numpy as np
import pytest

from mdff_b200 import _abi, systems
from mdff_b200._abi import MdffError
from mdff_b200.engine import BatchEngine, ForceEngine
from mdff_b200.params import params_copy

from .gpu_util import compare, forces, rms_rel

pytestmark = pytest.mark.gpu

# both types polarisable; linear with s = a A ~ 2.4 A, inside the shortest pairs
CASES = [(_abi.THOLE_LINEAR, 2.5), (_abi.THOLE_EXPON1, 0.572), (_abi.THOLE_EXPON2, 1.9088),
         (_abi.THOLE_GAUSS, 0.957)]


def _system(ttype, a):
    return systems.random_ionic((20, 20), L=12.5, seed=61, pol=(0.8, 1.1), calc=_abi.CALC_OTHER,
                                conv_tol_ind=1e-12, max_scf_pol_iter=800, thole_type=ttype,
                                thole_param=np.full((_abi.NT, _abi.NT), a))


@pytest.mark.parametrize("case", range(4))
def test_thole_fp64_matches_oracle(oracle, case):
    s = _system(*CASES[case])
    o = oracle.Oracle(s.params, s.cell).engforce(*s.soa())
    p = params_copy(s.params)
    p.solver = _abi.SOLVER_SCF
    with ForceEngine(p, s.cell) as eng:
        g = eng.engforce(*s.soa())
    compare(g, o, 1e-9)
    # Thole changes the answer
    q = params_copy(s.params)
    q.thole_type = _abi.THOLE_NONE
    o0 = oracle.Oracle(q, s.cell).engforce(*s.soa())
    assert rms_rel(forces(o0), forces(o)) > 1e-6


@pytest.mark.parametrize("case", range(4))
def test_thole_mixed_cg(oracle, case):
    s = _system(*CASES[case])
    o = oracle.Oracle(s.params, s.cell).engforce(*s.soa())
    p = params_copy(s.params)
    p.solver = _abi.SOLVER_CG
    p.cg_tol = 1e-10
    p.precision = _abi.PREC_MIXED
    with ForceEngine(p, s.cell) as eng:
        g = eng.engforce(*s.soa())
    assert rms_rel(forces(g), forces(o)) <= 1e-5
    assert rms_rel(g["mu"], o["mu"]) <= 1e-5


def test_batch_thole_matches_oracle(oracle):
    """The batched engine with the four Thole functions in one batch (one
    parameter set each), FP64: every box equals the oracle to 1e-9; mixed:
    within the 1e-5 force bar."""
    systs = [_system(*c) for c in CASES]
    for prec, tol in ((_abi.PREC_FP64, None), (_abi.PREC_MIXED, 1e-5)):
        psets, configs = [], []
        for k, s in enumerate(systs):
            p = params_copy(s.params)
            p.precision = prec
            p.solver = _abi.SOLVER_CG
            p.cg_tol = 1e-12
            p.cg_max_iter = 2000
            psets.append(p)
            configs.append((k, [p.natmi[0], p.natmi[1]], s.cell))
        P = np.concatenate([s.pos for s in systs])
        with BatchEngine(psets, configs) as eng:
            out = eng.engforce(P[:, 0], P[:, 1], P[:, 2])
            offs = eng.offsets
        for k, s in enumerate(systs):
            o = oracle.Oracle(s.params, s.cell).engforce(*s.soa())
            a, b = offs[k], offs[k + 1]
            g = {key: out[key][a:b] for key in ("fx", "fy", "fz", "mu", "ef")}
            g.update(out["conf"][k])
            if tol is None:
                compare(g, o, 1e-9)
            else:
                assert rms_rel(forces(g), forces(o)) <= tol


def test_batch_fit_rejects_thole():
    """The fit gradient does not cover Thole functions."""
    s = _system(*CASES[0])
    p = params_copy(s.params)
    p.solver = _abi.SOLVER_CG
    with BatchEngine([p], [(0, [p.natmi[0], p.natmi[1]], s.cell)]) as eng:
        with pytest.raises(MdffError) as e:
            eng.fit_define([(_abi.FIT_A, 0, 1)])
        assert e.value.status == _abi.MDFF_ERR_UNSUPPORTED
