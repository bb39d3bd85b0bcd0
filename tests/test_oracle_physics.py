"""Size-independent physical checks of the CPU oracle (its restatement of the
reference algorithm): forces are minus the gradient of the total energy
(including the PIM energy at the converged dipoles), the Ewald energy does not
depend on alpha, Newton's third law, and NR erfc / Tang-Toennies accuracy."""
import math

import numpy as np
import pytest

from mdff_b200 import systems


def _etot(r):
    return r["u_bmhft"] + r["u_lj"] + r["u_coul"]


@pytest.mark.parametrize("triclinic", [False, True])
def test_forces_are_energy_gradient(oracle, triclinic):
    s = systems.random_ionic((12, 12), L=12.0, seed=3, triclinic=triclinic, conv_tol_ind=1e-13,
                             calc=2,
                             ldip_damping={(1, 0, 1): 1}, pol_damp_b={(1, 0, 1): 3.0},
                             pol_damp_c={(1, 0, 1): 1.0}, pol_damp_k={(1, 0, 1): 4})
    o = oracle.Oracle(s.params, s.cell)
    r0 = o.engforce(*s.soa())
    f = np.stack([r0["fx"], r0["fy"], r0["fz"]], 1)
    h = 1e-5
    rng = np.random.default_rng(0)
    for ia in rng.choice(s.natm, 4, replace=False):
        for a in range(3):
            p = s.pos.copy()
            p[ia, a] += h
            ep = _etot(o.engforce(*(np.ascontiguousarray(p[:, k]) for k in range(3))))
            p[ia, a] -= 2 * h
            em = _etot(o.engforce(*(np.ascontiguousarray(p[:, k]) for k in range(3))))
            fd = -(ep - em) / (2 * h)
            assert abs(fd - f[ia, a]) < 2e-5 * max(1.0, abs(f[ia, a])), (ia, a, fd, f[ia, a])


def test_newton_third_law(oracle):
    s = systems.random_ionic((15, 15), L=13.0, seed=5)
    r = oracle.Oracle(s.params, s.cell).engforce(*s.soa())
    tot = np.array([r["fx"].sum(), r["fy"].sum(), r["fz"].sum()])
    assert np.abs(tot).max() < 1e-9 * np.abs(r["fx"]).max()


def test_ewald_alpha_invariance(oracle):
    s = systems.random_ionic((10, 10), L=11.0, seed=9, pol=(0.0, 0.0))
    us = []
    for alpha, k in ((0.55, 12), (0.75, 16)):
        s2 = systems.random_ionic((10, 10), L=11.0, seed=9, pol=(0.0, 0.0), alphaES=alpha,
                                  kES=(k, k, k), cutlongrange=5.5)
        us.append(oracle.Oracle(s2.params, s2.cell).engforce(*s2.soa())["u_coul"])
    assert abs(us[0] - us[1]) < 1e-5 * abs(us[0])


def test_nr_erfc_accuracy(oracle):
    for x in np.linspace(0.0, 4.0, 41):
        e = oracle.errfc(x)
        assert abs(e - math.erfc(x)) <= 1.3e-7 * max(math.erfc(x), 1e-300) + 1e-16


def test_tang_toennies_closed_form(oracle):
    for order in (1, 4, 6, 8):
        for r in (0.5, 1.7, 3.2):
            b, c = 2.3, 1.4
            f, fd = oracle.tt_damp(b, c, r, order)
            br = b * r
            s = sum(br ** k / math.factorial(k) for k in range(order + 1))
            assert abs(f - (1 - c * math.exp(-br) * s)) < 1e-14
            assert abs(fd - c * b * math.exp(-br) * br ** order / math.factorial(order)) < 1e-14
    # the reference's order-0 quirk (tt_damp.f90:85-93): f = 1 - c(1+br)e^{-br}
    f, fd = oracle.tt_damp(2.0, 1.0, 1.0, 0)
    assert abs(f - (1 - 3.0 * math.exp(-2.0))) < 1e-14
