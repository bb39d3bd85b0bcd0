"""Electric field gradients (mdff_gpu_efg) against the oracle's restatement of
the reference's doefg terms (ewald_dir.f90:543-582, ewald_rec.f90:209-217,
the self term): FP64 to 1e-10 relative on the small parity systems and the
reference's ex09 decks with Coulomb."""
import os

import numpy as np
import pytest

from mdff_b200 import _abi
from mdff_b200.engine import ForceEngine
from mdff_b200.params import params_copy

from .gpu_util import rel, small_systems

pytestmark = pytest.mark.gpu
CASES = [s for s in small_systems() if s.params.lcoulomb]
FX = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ex09_decks.npz"))


def _check(oracle, p, cell, pos):
    soa = [np.ascontiguousarray(pos[:, a]) for a in range(3)]
    o = oracle.Oracle(params_copy(p), cell).engforce(*soa, efg=True)
    with ForceEngine(params_copy(p), cell) as eng:
        eng.engforce(*soa)
        g = eng.efg()
    assert rel(g, o["efg"]) <= 1e-10
    # the reciprocal part fills the upper triangle only (as the reference)
    return g


@pytest.mark.parametrize("k", range(len(CASES)), ids=[s.name for s in CASES])
def test_efg_small_systems(oracle, k):
    s = CASES[k]
    _check(oracle, s.params, s.cell, s.pos)


@pytest.mark.parametrize("t", [3, 8, 11])
def test_efg_ex09(oracle, t):
    p = _abi.MdffParams.from_buffer_copy(FX[f"params_{t}"].tobytes())
    _check(oracle, p, FX["cell"], FX["pos"])
