"""Wannier-centre dipoles (moment_from_pola.f90:136-147, 632-807) on the GPU
against the CPU oracle: forces, dipoles and energies to 1e-9 with the
centres' dipoles on and off (ldip_wfc), in the FP64 SCF and CG and the
mixed engine (1e-5 force bar) and in the batched engine; a missing centre
and a centre type placed before another type are errors."""
import pytest

from mdff_b200 import _abi, systems
from mdff_b200._abi import MdffError
from mdff_b200.engine import BatchEngine, ForceEngine
from mdff_b200.params import params_copy

import numpy as np

from .gpu_util import compare, forces, rel, rms_rel

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
    # the batched engine reports a missing centre the same way
    with BatchEngine([p], [(0, [p.natmi[t] for t in range(3)], s.cell)]) as b:
        with pytest.raises(MdffError) as e:
            b.engforce(*s.soa())
        assert e.value.status == _abi.MDFF_ERR_BAD_ARGS


@pytest.mark.parametrize("ldip", [1, 0])
def test_wfc_batch_matches_oracle(oracle, ldip):
    """Wannier-centre boxes in one batch with a box without centres: each
    configuration against the oracle (FP64 PCG to 1e-11: 1e-8 relative)."""
    boxes = [systems.wannier_box(calc=_abi.CALC_OTHER, conv_tol_ind=1e-12, ldip_wfc=ldip),
             systems.wannier_box(calc=_abi.CALC_OTHER, conv_tol_ind=1e-12, ldip_wfc=ldip, seed=32,
                                 L=9.3),
             systems.random_ionic((20, 20), L=11.0, seed=33, calc=_abi.CALC_OTHER)]
    psets = []
    for b in boxes:
        p = params_copy(b.params)
        p.solver = _abi.SOLVER_CG
        p.cg_tol = 1e-11
        psets.append(p)
    desc = [(k, [b.params.natmi[t] for t in range(b.params.ntype)], b.cell) for k, b in enumerate(boxes)]
    pos = [np.concatenate([b.soa()[a] for b in boxes]) for a in range(3)]
    with BatchEngine(psets, desc) as be:
        g = be.engforce(*pos)
    off = 0
    for b in boxes:
        n = b.params.natm
        o = oracle.Oracle(b.params, b.cell).engforce(*b.soa())
        fg = np.stack([g["fx"][off:off + n], g["fy"][off:off + n], g["fz"][off:off + n]], 1)
        assert rel(fg, forces(o)) < 1e-8
        assert rel(g["mu"][off:off + n], o["mu"]) < 1e-8
        off += n
