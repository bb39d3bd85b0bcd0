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


def _patch_system():
    """300 ions (150 +1.5 cations, 150 -1.5 polarisable anions) in a 28 A box
    and two arrangements: A, the seeded sparse one (1.9 A apart at least),
    and B, where 60 cations and 60 anions sit on a 2.1 A rock-salt patch at
    the box centre (about 110 neighbours within rc + skin, well over the
    rows sized at creation for A's density).  Ions of A within 11 A of the
    centre that are not on the patch move to places the patch ions left
    more than 11 A from it."""
    L, c = 28.0, 14.0
    s = systems.random_ionic((150, 150), L=L, seed=72, skindiff=0.3, q=(1.5, -1.5), pol=(0.0, 1.1),
                             calc=_abi.CALC_MD, extrapolate_order=2, conv_tol_ind=1e-10,
                             max_scf_pol_iter=400)
    g = np.array([(i, j, k) for i in range(-3, 4) for j in range(-3, 4) for k in range(-3, 4)])
    g = g[np.argsort((g * g).sum(1), kind="stable")]
    cat = np.array([p for p in g if p.sum() % 2 == 0][:60], dtype=float)
    ani = np.array([p for p in g if p.sum() % 2 != 0][:60], dtype=float)
    posA = s.pos.copy()
    patch = list(range(60)) + list(range(150, 210))
    dist = lambda P: np.linalg.norm(P - c, axis=1)
    free = [posA[i] for i in patch if dist(posA[i:i + 1])[0] > 11.0]
    posB = posA.copy()
    posB[:60] = c + 2.1 * cat
    posB[150:210] = c + 2.1 * ani
    near = [i for i in range(300) if i not in patch and dist(posA[i:i + 1])[0] <= 11.0]
    assert len(near) <= len(free)
    for k, i in enumerate(near):
        posB[i] = free[k]
    return s, posA, posB


def test_list_overflow_retry_keeps_the_aspc_history(oracle):
    """A list overflow in an MD step with polarisable ions: the call grows the
    rows and redoes itself; the ASPC predictor shifts the dipole history in
    place, so the redo must start from the history as the call found it.
    Forces at every step and the history at the end equal the oracle's."""
    s, posA, posB = _patch_system()
    orc = oracle.Oracle(params_copy(s.params), s.cell)
    rng = np.random.default_rng(3)
    seq = [posA, posA + rng.uniform(-0.02, 0.02, posA.shape), posB,
           posB + rng.uniform(-0.02, 0.02, posB.shape), posB + rng.uniform(-0.02, 0.02, posB.shape)]
    with ForceEngine(params_copy(s.params), s.cell) as eng:
        cap0 = eng.stats()["list_capacity"]
        for itime, pos in enumerate(seq):
            soa = tuple(np.ascontiguousarray(pos[:, a]) for a in range(3))
            g = eng.engforce(*soa, itime=itime)
            o = orc.engforce(*soa, itime=itime)
            f = np.stack([g["fx"], g["fy"], g["fz"]], 1)
            fo = np.stack([o["fx"], o["fy"], o["fz"]], 1)
            assert np.abs(f - fo).max() <= 1e-9 * np.abs(fo).max(), itime
        assert eng.stats()["list_capacity"] > cap0        # the rows grew at step 2
        h = eng.aspc_history()
    ho = orc.get_aspc()
    assert np.abs(h - ho).max() <= 1e-9 * np.abs(ho).max()
