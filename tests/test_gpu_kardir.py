"""The reference's in-place kardir/dirkar round trips (lattice.f90:183-270):
the engine counts those of each engforce (stats n_kardir: one per
short-range routine, per multipole_ES_dir and for the Wannier centres) and
mdff_gpu_kardir_roundtrips applies them to the caller's positions.  Both are
compared with the oracle, which makes the round trips where the reference
does (ewald_dir.f90:138,739, non_bonded.f90:716,823,1113,1221,
moment_from_pola.f90:685,803): equal counts and bit-identical positions."""
import numpy as np
import pytest

from mdff_b200 import _abi, systems
from mdff_b200.engine import ForceEngine
from mdff_b200.params import params_copy

from .gpu_util import small_systems

pytestmark = pytest.mark.gpu

CASES = small_systems() + [systems.wannier_box(calc=_abi.CALC_OTHER)]
IDS = [s.name + f"_{i}" for i, s in enumerate(CASES)]


@pytest.mark.parametrize("sysi", range(len(CASES)), ids=IDS)
def test_roundtrip_count_and_positions_match_oracle(oracle, sysi):
    s = CASES[sysi]
    orc = oracle.Oracle(s.params, s.cell)
    o = orc.engforce(*s.soa())
    with ForceEngine(params_copy(s.params), s.cell) as eng:
        eng.engforce(*s.soa())
        n = eng.stats()["n_kardir"]
        assert n == o["n_kardir"] > 0
        g = eng.kardir_roundtrips(*s.soa())
    r = orc.kardir_roundtrips(*s.soa(), n)
    for a, b in zip(g, r):
        assert np.array_equal(a, b)


def test_roundtrips_move_positions_of_a_triclinic_cell(oracle):
    """On a triclinic cell the round trips change some positions (by an ulp or
    so): the comparison above is not comparing unchanged arrays."""
    s = systems.random_ionic((20, 28), L=13.5, seed=22, triclinic=True, calc=_abi.CALC_OTHER)
    x = s.soa()
    with ForceEngine(params_copy(s.params), s.cell) as eng:
        g = eng.kardir_roundtrips(*x, 25)
    moved = sum(int((a != b).sum()) for a, b in zip(g, x))
    assert moved > 0
    assert max(float(np.abs(a - b).max()) for a, b in zip(g, x)) < 1e-12
    r = oracle.Oracle(s.params, s.cell).kardir_roundtrips(*x, 25)
    for a, b in zip(g, r):
        assert np.array_equal(a, b)


def test_count_limit_is_refused():
    s = systems.nacl(ncell=2, rcut=12.0, kmax=6)
    with ForceEngine(params_copy(s.params), s.cell) as eng:
        with pytest.raises(_abi.MdffError) as e:
            eng.kardir_roundtrips(*s.soa(), (1 << 20) + 1)
        assert e.value.status == _abi.MDFF_ERR_BAD_ARGS
        x = s.soa()
        assert all(np.array_equal(a, b) for a, b in zip(eng.kardir_roundtrips(*x, 0), x))


def test_count_is_undefined_for_other_solvers():
    s = systems.mgo(ncell=2, calc=_abi.CALC_OTHER)
    p = params_copy(s.params)
    p.solver = _abi.SOLVER_CG
    with ForceEngine(p, s.cell) as eng:
        eng.engforce(*s.soa())
        assert eng.stats()["n_kardir"] == -1
        with pytest.raises(ValueError):
            eng.kardir_roundtrips(*s.soa())
