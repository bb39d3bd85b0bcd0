"""The oracle's kO dipole algorithms (moment_from_pola.f90:822-2529) and the
polynomial predictor (:2276-2412), on the CPU.

polint is pinned by known answers worked by hand from the reference's
recurrence: with abscissae xa(t) = 1 - t it takes hp from xa(i+1) where
Neville's scheme has xa(i+m), so through three points it returns
4 y0 - 5 y1 + 2 y2 (not the quadratic 3 y0 - 3 y1 + y2); through two points
it is the linear 2 y0 - y1.  The kO algorithms must converge to the same
dipoles as the plain SCF (they solve the same linear system)."""
import numpy as np
import pytest

from mdff_b200 import _abi, systems
from mdff_b200.params import params_copy


def test_polint_known_answers(oracle):
    y = np.array([1.3, -0.7, 2.9, 0.4, -1.1])
    assert oracle.polint([0, -1], y[:2]) == 2 * y[0] - y[1]
    assert abs(oracle.polint([0, -1, -2], y[:3]) - (4 * y[0] - 5 * y[1] + 2 * y[2])) < 1e-14
    # constants are reproduced at every order
    for n in range(1, 6):
        assert abs(oracle.polint([1 - t for t in range(1, n + 1)], np.full(n, 0.37)) - 0.37) < 1e-13


def _system(calc=_abi.CALC_OTHER, **kw):
    return systems.random_ionic((16, 16), L=11.5, seed=71, calc=calc, **kw)


@pytest.mark.parametrize("algo,tol,bar", [(_abi.ALGO_KO_V1, 1e-10, 1e-8), (_abi.ALGO_KO_V2, 1e-10, 1e-8),
                                          (_abi.ALGO_KO_V4_1, 1e-6, 1e-4)])
def test_ko_converges_to_scf_solution(oracle, algo, tol, bar):
    s = _system(conv_tol_ind=1e-12, max_scf_pol_iter=400)
    ref = oracle.Oracle(s.params, s.cell).engforce(*s.soa())
    p = params_copy(s.params)
    p.algo_moment_from_pola = algo
    p.conv_tol_ind = tol
    p.max_scf_pol_iter = 100
    o = oracle.Oracle(p, s.cell).engforce(*s.soa())
    assert o["rmsd"] <= tol and o["n_scf"] < p.max_scf_pol_iter
    mu, mr = o["mu"], ref["mu"]
    assert np.abs(mu - mr).max() <= bar * np.abs(mr).max()
    # the inner relaxation takes fewer outer passes than the plain SCF
    if algo != _abi.ALGO_KO_V4_1:
        assert o["n_scf"] < ref["n_scf"]


def test_ko_rejections(oracle):
    s = _system()
    for algo in (_abi.ALGO_KO_V3, _abi.ALGO_KO_V4_2):
        p = params_copy(s.params)
        p.algo_moment_from_pola = algo
        with pytest.raises(_abi.MdffError) as e:
            oracle.Oracle(p, s.cell).engforce(*s.soa())
        assert e.value.status == _abi.MDFF_ERR_UNSUPPORTED
    p = params_copy(s.params)
    p.algo_moment_from_pola = _abi.ALGO_KO_V4_1
    p.max_scf_pol_iter = 101
    with pytest.raises(_abi.MdffError) as e:
        oracle.Oracle(p, s.cell).engforce(*s.soa())
    assert e.value.status == _abi.MDFF_ERR_BAD_ARGS
