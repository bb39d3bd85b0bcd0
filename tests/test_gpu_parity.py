"""GPU parity: the CUDA engine through the C ABI against the CPU oracle.

FP64 + the reference's SCF solver must reproduce energies, forces, stress,
dipoles and fields to 1e-10 relative; the neighbour lists must be identical
(the reference's 1-based CSR half lists, tools.f90:273-368)."""
import numpy as np
import pytest

from mdff_b200 import _abi, systems
from mdff_b200.engine import ForceEngine
from mdff_b200.params import params_copy

from .gpu_util import compare, rel, small_systems, forces

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10
CASES = small_systems()
IDS = [s.name + f"_{i}" for i, s in enumerate(CASES)]


@pytest.mark.parametrize("sysi", range(len(CASES)), ids=IDS)
def test_engforce_fp64_scf(oracle, sysi):
    s = CASES[sysi]
    o = oracle.Oracle(s.params, s.cell).engforce(*s.soa())
    with ForceEngine(params_copy(s.params), s.cell) as eng:
        g = eng.engforce(*s.soa())
        st = eng.stats()
    if o["n_scf"]:
        assert st["n_pol_iter"] == o["n_scf"]
    compare(g, o, TOL_FP64)


@pytest.mark.parametrize("sysi", range(len(CASES)), ids=IDS)
def test_verlet_lists_bit_exact(oracle, sysi):
    s = CASES[sysi]
    orc = oracle.Oracle(s.params, s.cell)
    with ForceEngine(params_copy(s.params), s.cell) as eng:
        for which in (0, 1):
            p = s.params
            if which == 0 and not (p.lbmhft or p.lbmhftd or p.lnmlj):
                continue
            if which == 1 and not p.lcoulomb:
                continue
            so, po, lo, no = orc.vnlist(*s.soa(), which=which)
            sg, pg, lg, ng = eng.verlet_half_list(*s.soa(), which=which)
            assert so == 0 and sg == 0
            assert no == ng
            assert np.array_equal(po, pg)
            assert np.array_equal(lo, lg)


def test_repeat_calls_are_deterministic():
    # calc other than md/opt: no ASPC predictor, so both calls take the same path
    s = systems.random_ionic((24, 24), L=13.0, seed=31, calc=_abi.CALC_OTHER)
    with ForceEngine(params_copy(s.params), s.cell) as eng:
        a = eng.engforce(*s.soa())
        b = eng.engforce(*s.soa())
    for k in ("fx", "fy", "fz", "mu", "ef"):
        assert np.array_equal(a[k], b[k]), k
    assert a["u_coul"] == b["u_coul"]


@pytest.mark.parametrize("order", [2, 4])
def test_aspc_md_sequence_matches_oracle(oracle, order):
    """calc='md' with ASPC orders 2 and 4 (the MD workloads' order) over
    moving steps past the order ramp: the predictor, corrector and history
    rotation (moment_from_pola.f90:493-598)."""
    s = systems.random_ionic((20, 20), L=12.5, seed=41, calc=_abi.CALC_MD,
                             extrapolate_order=order, conv_tol_ind=1e-9)
    orc = oracle.Oracle(s.params, s.cell)
    rng = np.random.default_rng(1)
    pos = s.pos.copy()
    with ForceEngine(params_copy(s.params), s.cell) as eng:
        for itime in range(0, order + 4):
            soa = tuple(np.ascontiguousarray(pos[:, a]) for a in range(3))
            o = orc.engforce(*soa, itime=itime)
            g = eng.engforce(*soa, itime=itime)
            compare(g, o, 1e-9)
            pos = pos + rng.uniform(-0.02, 0.02, pos.shape)
        h = eng.aspc_history()
    assert rel(h, orc.get_aspc()) < 1e-9


def test_aspc_history_roundtrip():
    s = systems.random_ionic((10, 10), L=11.0, seed=4)
    with ForceEngine(params_copy(s.params), s.cell) as eng:
        b = np.random.default_rng(0).normal(size=(_abi.ASPC_DEPTH, s.natm, 3))
        eng.set_aspc_history(b)
        assert np.array_equal(eng.aspc_history(), b)


def test_set_cell_and_list_rebuild(oracle):
    s = systems.random_ionic((20, 20), L=12.5, seed=42)
    with ForceEngine(params_copy(s.params), s.cell) as eng:
        eng.engforce(*s.soa())
        cell2 = s.cell * 1.03
        pos2 = s.pos * 1.03
        eng.set_cell(cell2)
        soa = tuple(np.ascontiguousarray(pos2[:, a]) for a in range(3))
        g = eng.engforce(*soa)
    p2 = params_copy(s.params)
    o = oracle.Oracle(p2, cell2).engforce(*soa)
    # the clamp of cutlongrange happens at creation only (coulomb.f90:377-383),
    # both sides keep the original cutoff
    compare(g, o, 1e-10)
