"""Tensor-core reciprocal kernels of the mixed engine: the structure factor of
the FP32 CG operator (k_rec_rho_tc) and the FP32 field / force partials
(k_rec_field_tc).

The mixed engine on the tensor cores (default) must agree with the same
engine on the CUDA-core kernels (MDFF_REC_TC=0, MDFF_FIELD_TC=0) to the CG
tolerance, on boxes that reach both B-tile widths (kz 7 -> 32 rows, kz 16
-> 64 rows), a triclinic cell, a box with fewer ions than one K block and an
odd ion count, a box whose polarisable ions sit in two type blocks with a
non-polarisable block between them (the structure factor's ion slots and the
fields' ion map are not one index range); both must meet the 1e-5 force bar
against the CPU oracle."""
import numpy as np
import pytest

from mdff_b200 import _abi, systems
from mdff_b200.engine import ForceEngine
from mdff_b200.params import params_copy

from .gpu_util import forces, rms_rel

pytestmark = pytest.mark.gpu


def _cases():
    return [
        systems.random_ionic((24, 24), L=13.0, seed=51, calc=_abi.CALC_OTHER),
        systems.random_ionic((10, 10), L=10.0, seed=3, triclinic=True, calc=_abi.CALC_OTHER),
        systems.random_ionic((8, 8), L=9.0, seed=4, calc=_abi.CALC_OTHER),
        # odd ion count: table rows of odd stride, a partial last K block
        systems.random_ionic((19, 18), L=12.0, seed=8, q=(1.2, -1.2), calc=_abi.CALC_OTHER),
        systems.mgo(ncell=2, kmax=16, calc=_abi.CALC_OTHER),
        systems.sio2(nsio2=150, seed=9, calc=_abi.CALC_OTHER),
        systems.random_ionic((20, 30, 20), L=13.0, seed=17, q=(-1.5, 2.0, -1.5), pol=(1.1, 0.0, 1.1),
                             calc=_abi.CALC_OTHER),
    ]


def _run(s, tc, monkeypatch):
    monkeypatch.setenv("MDFF_REC_TC", "1" if tc else "0")
    monkeypatch.setenv("MDFF_FIELD_TC", "1" if tc else "0")
    p = params_copy(s.params)
    p.solver = _abi.SOLVER_CG
    p.cg_tol = 1e-10
    p.precision = _abi.PREC_MIXED
    with ForceEngine(p, s.cell) as eng:
        r = eng.engforce(*s.soa())
        st = eng.stats()
    assert st["converged"]
    return r


@pytest.mark.parametrize("case", range(7))
def test_tensor_core_operator_matches_cuda_core(oracle, case, monkeypatch):
    s = _cases()[case]
    a = _run(s, True, monkeypatch)
    b = _run(s, False, monkeypatch)
    assert rms_rel(forces(a), forces(b)) <= 2e-6
    assert rms_rel(a["mu"], b["mu"]) <= 2e-6
    assert abs(a["u_coul"] - b["u_coul"]) <= 1e-7 * abs(b["u_coul"])
    o = oracle.Oracle(s.params, s.cell).engforce(*s.soa())
    assert rms_rel(forces(a), forces(o)) <= 1e-5
