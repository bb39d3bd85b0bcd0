"""Wannier-centre dipoles (moment_from_pola.f90:136-147, 632-807) on the GPU
against the CPU oracle: forces, dipoles and energies to 1e-9 with the
centres' dipoles on and off (ldip_wfc), in the FP64 SCF and CG and the
mixed engine (1e-5 force bar); a missing centre and a centre type placed
before another type are errors; the batched engine rejects centres."""
import pytest

from mdff_b200 import _abi, systems
from mdff_b200._abi import MdffError
from mdff_b200.engine import BatchEngine, ForceEngine
from mdff_b200.params import params_copy

from .gpu_util import compare, forces, rms_rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ldip", [1, 0])
def test_wfc_fp64_matches_oracle(oracle, ldip):
    s = systems.wannier_box(calc=_abi.CALC_OTHER)
    p = params_copy(s.params)
    p.ldip_wfc = ldip
    o = oracle.Oracle(p, s.cell).engforce(*s.soa())
    with ForceEngine(p, s.cell) as eng:
        g = eng.engforce(*s.soa())
    compare(g, o, 1e-9)


@pytest.mark.parametrize("prec", [_abi.PREC_FP64, _abi.PREC_MIXED])
def test_wfc_cg(oracle, prec):
    s = systems.wannier_box(calc=_abi.CALC_OTHER, seed=32)
    o = oracle.Oracle(s.params, s.cell).engforce(*s.soa())
    p = params_copy(s.params)
    p.solver = _abi.SOLVER_CG
    p.cg_tol = 1e-10
    p.precision = prec
    with ForceEngine(p, s.cell) as eng:
        g = eng.engforce(*s.soa())
    if prec == _abi.PREC_FP64:
        compare(g, o, 1e-8)
    else:
        assert rms_rel(forces(g), forces(o)) <= 1e-5


def test_wfc_errors():
    s = systems.wannier_box(calc=_abi.CALC_OTHER)
    p = params_copy(s.params)
    p.lwfc[1] = 5
    with ForceEngine(p, s.cell) as eng:
        with pytest.raises(MdffError) as e:
            eng.engforce(*s.soa())
        assert e.value.status == _abi.MDFF_ERR_BAD_ARGS
    q = params_copy(s.params)
    q.lwfc[0], q.lwfc[2] = -1, 0
    with pytest.raises(MdffError) as e:
        ForceEngine(q, s.cell)
    assert e.value.status == _abi.MDFF_ERR_BAD_ARGS
    with pytest.raises(MdffError):
        BatchEngine([s.params], [(0, [s.params.natmi[t] for t in range(3)], s.cell)])
