"""GPU failure detection without any GPU fault: every failure is a status
code returned by the host side after a normal kernel run."""
import numpy as np
import pytest

from mdff_b200 import _abi, systems
from mdff_b200.engine import ForceEngine, MdffError
from mdff_b200.params import params_copy

pytestmark = pytest.mark.gpu


def test_polarisation_catastrophe_status():
    # alpha large enough that the induced dipoles exceed 10 eA
    s = systems.random_ionic((10, 10), L=10.0, seed=61, pol=(0.0, 40.0), max_scf_pol_iter=5,
                             calc=_abi.CALC_OTHER)
    with ForceEngine(params_copy(s.params), s.cell) as eng:
        with pytest.raises(MdffError) as e:
            eng.engforce(*s.soa())
        assert e.value.status == _abi.MDFF_ERR_CATASTROPHE
        # the handle stays usable
        s2 = systems.random_ionic((10, 10), L=10.0, seed=61, pol=(0.0, 0.0))
    with ForceEngine(params_copy(s2.params), s2.cell) as eng2:
        eng2.engforce(*s2.soa())


def test_not_converged_status():
    s = systems.random_ionic((12, 12), L=11.0, seed=62, conv_tol_ind=1e-14, max_scf_pol_iter=2,
                             min_scf_pol_iter=1, calc=_abi.CALC_OTHER)
    p = params_copy(s.params)
    p.fail_on_nonconvergence = 1
    with ForceEngine(p, s.cell) as eng:
        with pytest.raises(MdffError) as e:
            eng.engforce(*s.soa())
        assert e.value.status == _abi.MDFF_ERR_NOT_CONVERGED
        assert eng.stats()["n_pol_iter"] == 2


def test_list_overflow_recovers(oracle):
    """Positions compressed after the first call overflow the rows sized for
    the first density: the engine grows them and redoes the call."""
    s = systems.random_ionic((150, 150), L=28.0, seed=63, skindiff=0.3, pol=(0.0, 0.0))
    with ForceEngine(params_copy(s.params), s.cell) as eng:
        eng.engforce(*s.soa())
        cap0 = eng.stats()["list_capacity"]
        assert cap0 < s.natm * s.natm
        # cluster a third of the ions into a small region
        pos = s.pos.copy()
        rng = np.random.default_rng(2)
        pos[: s.natm // 3] = 2.0 + rng.uniform(0, 5.0, (s.natm // 3, 3))
        soa = tuple(np.ascontiguousarray(pos[:, a]) for a in range(3))
        g = eng.engforce(*soa)
        assert eng.stats()["list_capacity"] > cap0
    o = oracle.Oracle(s.params, s.cell).engforce(*soa)
    assert np.abs(g["fx"] - o["fx"]).max() <= 1e-9 * np.abs(o["fx"]).max()


def test_bad_parameters_rejected():
    s = systems.random_ionic((4, 4), L=10.0, extrapolate_order=7)
    with pytest.raises(MdffError) as e:
        ForceEngine(params_copy(s.params), s.cell)
    assert e.value.status == _abi.MDFF_ERR_BAD_ARGS


def test_tensor_core_wait_timeout_is_reported_and_recovers(oracle):
    """A bounded device wait that runs out: with the operand-stage wait of the
    tensor-core structure factor (the mixed engine's CG operator) limited to
    zero polls, every CTA with more than two K blocks gives up at its first
    such wait, drains the products it issued and frees its tensor memory; the
    call returns MDFF_ERR_TIMEOUT.  With the default limit restored the same
    handle computes the forces again, equal to a fresh handle's and within the
    mixed engine's bar of the oracle."""
    s = systems.sio2(nsio2=1000, seed=64, calc=_abi.CALC_OTHER)   # 3000 ions: 4 K blocks per chunk
    p = params_copy(s.params)
    p.precision = _abi.PREC_MIXED
    p.solver = _abi.SOLVER_CG
    p.cg_tol = 1e-8
    with ForceEngine(p, s.cell) as eng:
        eng.set_tc_wait_limit(0)
        with pytest.raises(MdffError) as e:
            eng.engforce(*s.soa())
        assert e.value.status == _abi.MDFF_ERR_TIMEOUT
        eng.set_tc_wait_limit(-1)
        g = eng.engforce(*s.soa())
    with ForceEngine(params_copy(p), s.cell) as eng2:
        g2 = eng2.engforce(*s.soa())
    for k in ("fx", "fy", "fz", "mu"):
        assert np.array_equal(g[k], g2[k]), k
    o = oracle.Oracle(params_copy(s.params), s.cell).engforce(*s.soa())
    f = np.stack([g["fx"], g["fy"], g["fz"]], 1)
    fo = np.stack([o["fx"], o["fy"], o["fz"]], 1)
    assert np.sqrt(((f - fo) ** 2).sum() / (fo ** 2).sum()) <= 1e-5
