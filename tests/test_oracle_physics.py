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


def test_oracle_kardir_roundtrips_match_numpy(oracle):
    """The oracle's in-place round trip (kardir then dirkar, lattice.f90:183-270)
    restated in numpy with the same left-to-right sums: bit for bit."""
    from mdff_b200 import _abi, systems
    s = systems.random_ionic((20, 28), L=13.5, seed=22, triclinic=True, calc=_abi.CALC_OTHER)
    orc = oracle.Oracle(s.params, s.cell)
    A = np.asarray(s.cell, dtype=np.float64).reshape(3, 3)
    B = np.array(orc.setup().B[:], dtype=np.float64).reshape(3, 3)
    x, y, z = (np.array(a, dtype=np.float64) for a in s.soa())
    for _ in range(7):
        v1 = x * B[0, 0] + y * B[1, 0] + z * B[2, 0]
        v2 = x * B[0, 1] + y * B[1, 1] + z * B[2, 1]
        v3 = x * B[0, 2] + y * B[1, 2] + z * B[2, 2]
        x = v1 * A[0, 0] + v2 * A[0, 1] + v3 * A[0, 2]
        y = v1 * A[1, 0] + v2 * A[1, 1] + v3 * A[1, 2]
        z = v1 * A[2, 0] + v2 * A[2, 1] + v3 * A[2, 2]
    r = orc.kardir_roundtrips(*s.soa(), 7)
    for a, b in zip(r, (x, y, z)):
        assert np.array_equal(a, b)


def test_oracle_counts_the_reference_roundtrips(oracle):
    """One round trip per short-range routine, per multipole_ES_dir (static
    field, each SCF iteration, final pass) and for the Wannier centres."""
    from mdff_b200 import _abi, systems
    s = systems.mgo(ncell=2, calc=_abi.CALC_OTHER)
    o = oracle.Oracle(s.params, s.cell).engforce(*s.soa())
    assert o["n_scf"] > 0
    assert o["n_kardir"] == 1 + (1 + o["n_scf"] + 1)
    s = systems.nacl(ncell=2, rcut=12.0, kmax=6)
    o = oracle.Oracle(s.params, s.cell).engforce(*s.soa())
    assert o["n_kardir"] == 1 + 1
