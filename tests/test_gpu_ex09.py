"""The reference's own ex09 decks (examples/ex09/config: 200 ions O / Si / B,
BMH / BMHFTD / Ewald / PIM / damped PIM in the 11 combinations of its
test.config), read through mdff_b200.mdffio into tests/golden/ex09_decks.npz:
the GPU engine in FP64 + SCF must equal the oracle to 1e-10, and the mixed
engine must stay within 1e-5 RMS force error."""
import os

import numpy as np
import pytest

from mdff_b200 import _abi
from mdff_b200.engine import ForceEngine
from mdff_b200.params import params_copy

from .gpu_util import compare, forces, rms_rel

pytestmark = pytest.mark.gpu
FX = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ex09_decks.npz"))
TESTS = [int(t[0]) for t in FX["tests"]]


def _params(t):
    return _abi.MdffParams.from_buffer_copy(FX[f"params_{t}"].tobytes())


@pytest.mark.parametrize("t", TESTS)
def test_ex09_fp64_vs_oracle(oracle, t):
    p = _params(t)
    P = FX["pos"]
    soa = [np.ascontiguousarray(P[:, a]) for a in range(3)]
    o = oracle.Oracle(params_copy(p), FX["cell"]).engforce(*soa)
    with ForceEngine(params_copy(p), FX["cell"]) as eng:
        g = eng.engforce(*soa)
        st = eng.stats()
    if o["n_scf"]:
        assert st["n_pol_iter"] == o["n_scf"]
    compare(g, o, 1e-10)


@pytest.mark.parametrize("t", [t for t in TESTS if _params(t).ldip_polar[0]])
def test_ex09_mixed_error(t):
    p64 = _params(t)
    pm = params_copy(p64)
    pm.precision = _abi.PREC_MIXED
    pm.solver = _abi.SOLVER_CG
    pm.cg_tol = 1e-8
    P = FX["pos"]
    soa = [np.ascontiguousarray(P[:, a]) for a in range(3)]
    with ForceEngine(params_copy(p64), FX["cell"]) as e64, ForceEngine(pm, FX["cell"]) as emx:
        a = e64.engforce(*soa)
        b = emx.engforce(*soa)
    assert rms_rel(forces(b), forces(a)) <= 1e-5
