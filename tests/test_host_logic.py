"""Host-side set-up logic (no GPU): parameter defaults, symmetrisation, k
mesh, Ewald parameter rule, Verlet-list properties, synthetic systems."""
import math

import numpy as np
import pytest

from mdff_b200 import _abi, make_params, systems


def test_defaults_follow_reference():
    p = make_params([2])
    assert p.skindiff == 0.15 and p.conv_tol_ind == 1e-6       # control.f90:230, pim.f90:120
    assert p.min_scf_pol_iter == 3 and p.max_scf_pol_iter == 100
    assert list(p.kES) == [10, 10, 10] and p.alphaES == 1.0     # coulomb.f90:167-171
    assert p.qlj[0][0] == 12.0 and p.plj[0][0] == 6.0           # non_bonded.f90:180-181
    assert p.symmetric_pot_nb == 1 and p.symmetric_pot_pim == 1


def test_kmesh_half_space_count(oracle):
    s = systems.nacl(ncell=2, kmax=5)
    o = oracle.Oracle(s.params, s.cell)
    k = 5
    # coulomb.f90:472: nk = kz + ky(2kz+1) + kx(2ky+1)(2kz+1)
    assert o.setup().nk == k + k * (2 * k + 1) + k * (2 * k + 1) ** 2
    km = o.kmesh()
    assert np.all(np.diff(km["kk"]) >= 0)      # sorted by |k|^2 (kspace.f90:286-342)
    assert np.allclose(km["Ak"], np.exp(-km["kk"] / (4 * s.params.alphaES ** 2)) / km["kk"])


def test_ewald_param_rule(oracle):
    s = systems.mgo(ncell=2, lautoES=1, epsw=1e-7, rcut=50.0)
    o = oracle.Oracle(s.params, s.cell)
    info = o.setup()
    L = s.info["L"]
    assert abs(info.cutlongrange - 0.5 * L) < 1e-12        # clamp to half the cell
    cut = 0.5 * L
    tol = math.sqrt(abs(math.log(1e-7 * cut)))
    alpha = math.sqrt(abs(math.log(1e-7 * cut * tol))) / cut
    assert abs(info.alphaES - alpha) < 1e-14
    assert list(info.kES) == [systems.ewald_kmax(alpha, cut, 1e-7, L)] * 3


def test_mgo_kmax_stated():
    s = systems.mgo(ncell=10)
    assert s.info["kmax"] == 16 and abs(s.info["L"] - 42.13) < 0.01


def test_box_sizes_match_configs():
    assert abs(systems.nacl(ncell=6).info["L"] - 37.82) < 0.01
    assert abs(systems.box_length(4000, 28.0855 + 2 * 15.9994, 2.2) - 56.61) < 0.01


def test_symmetrisation_upper_triangle_wins(oracle):
    # non_bonded.f90:287-301: X(:,it) = X(it,:) sequentially -> (i<j) entries win
    s = systems.random_ionic((4, 4), L=10.0, Abmhftd={(0, 1): 100.0, (1, 0): 5.0, (1, 1): 50.0})
    o = oracle.Oracle(s.params, s.cell)
    s2 = systems.random_ionic((4, 4), L=10.0, Abmhftd={(0, 1): 100.0, (1, 0): 100.0, (1, 1): 50.0})
    o2 = oracle.Oracle(s2.params, s2.cell)
    assert o.engforce(*s.soa())["u_bmhft"] == o2.engforce(*s2.soa())["u_bmhft"]


def test_half_list_is_parity_masked_full_list(oracle):
    s = systems.random_ionic((30, 30), L=13.0, seed=11, triclinic=True)
    o = oracle.Oracle(s.params, s.cell)
    st, point, lst, n = o.vnlist(*s.soa(), which=1)
    assert st == 0 and point[0] == 1 and point[-1] == n + 1
    pairs = set()
    for i in range(s.natm):
        row = lst[point[i] - 1: point[i + 1] - 1] - 1
        assert np.all(np.diff(row) > 0)            # ascending ja within a row
        for j in row:
            odd = (i + j) % 2
            assert (i > j and odd == 0) or (i < j and odd == 1)
            pairs.add((min(i, j), max(i, j)))
    assert len(pairs) == n                          # each pair exactly once


def test_list_overflow_reported(oracle):
    s = systems.random_ionic((20, 20), L=12.0, seed=2)
    o = oracle.Oracle(s.params, s.cell)
    st, point, lst, n = o.vnlist(*s.soa(), which=1, capacity=10)
    assert st == _abi.MDFF_ERR_LIST_OVERFLOW and n > 10


def test_sio2_rsi_minimum_separations():
    s = systems.sio2(nsio2=300, seed=4)
    L = s.info["L"]
    n_si = 300
    d = s.pos[:, None, :] - s.pos[None, :, :]
    d -= L * np.round(d / L)
    r = np.sqrt((d ** 2).sum(-1)) + np.eye(s.natm) * 99
    assert r[:n_si, n_si:].min() >= 1.4 - 1e-12
    assert r[n_si:, n_si:].min() >= 2.2 - 1e-12
    assert r[:n_si, :n_si].min() >= 2.5 - 1e-12


def test_seeded_systems_are_reproducible():
    a = systems.nacl(ncell=2, seed=5)
    b = systems.nacl(ncell=2, seed=5)
    assert np.array_equal(a.pos, b.pos) and np.array_equal(a.vel, b.vel)
