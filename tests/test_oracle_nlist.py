"""The oracle's Verlet-list routines on the CPU: vnlist_pbc
(tools.f90:273-368) against an independent numpy scan, and vnlistcheck
(tools.f90:444-537): the largest + second largest displacement, ties, the
`.gt.` threshold and the new reference after a rebuild."""
import numpy as np

from mdff_b200 import systems
from mdff_b200.params import params_copy


def _numpy_half_list(s, rs):
    A = np.asarray(s.cell)
    S = s.pos @ np.linalg.inv(A).T                 # direct coordinates
    n = s.natm
    point, lst = [1], []
    for i in range(n):
        j = np.arange(n)
        mask = ((i > j) & ((i + j) % 2 == 0)) | ((i < j) & ((i + j) % 2 == 1))
        d = S[i] - S[j]
        d = d - np.where(d >= 0, np.floor(d + 0.5), np.ceil(d - 0.5))   # Fortran NINT
        r = d @ A.T
        keep = mask & ((r * r).sum(1) <= rs * rs)
        lst.extend((j[keep] + 1).tolist())
        point.append(len(lst) + 1)
    return np.array(point), np.array(lst)


def test_vnlist_matches_numpy_scan(oracle):
    s = systems.random_ionic((70, 80), L=16.0, seed=5, triclinic=True)
    o = oracle.Oracle(params_copy(s.params), s.cell)
    for which, cut in ((0, s.params.cutshortrange), (1, s.params.cutlongrange)):
        st, point, lst, n = o.vnlist(*s.soa(), which=which)
        p2, l2 = _numpy_half_list(s, cut + s.params.skindiff)
        assert st == 0 and n == len(l2)
        assert np.array_equal(point, p2)
        assert np.array_equal(lst, l2)


def _soa(p):
    return tuple(np.ascontiguousarray(p[:, a]) for a in range(3))


def test_vnlistcheck_top_two_threshold_and_reference(oracle):
    s = systems.random_ionic((20, 20), L=13.0, seed=3)
    skin = s.params.skindiff                       # 0.7 A
    o = oracle.Oracle(params_copy(s.params), s.cell)
    r, d = o.vnlistcheck(*s.soa())
    assert r and d > skin                          # stored coordinates start at zero
    r, d = o.vnlistcheck(*s.soa())
    assert not r and d == 0.0
    # largest + second largest: 0.3 + 0.25 (a third, smaller move does not count)
    p = s.pos.copy()
    p[3, 0] += 0.3
    p[7, 1] -= 0.25
    p[11, 2] += 0.1
    r, d = o.vnlistcheck(*_soa(p))
    assert not r and abs(d - 0.55) < 1e-12
    # ties: two moves of 0.36 sum to 0.72 > 0.7
    p[3, 0] = s.pos[3, 0] + 0.36
    p[7, 1] = s.pos[7, 1] - 0.36
    r, d = o.vnlistcheck(*_soa(p))
    assert r and abs(d - 0.72) < 1e-12
    # the rebuild made these positions the reference
    r, d = o.vnlistcheck(*_soa(p))
    assert not r and d == 0.0
    # a move across the periodic boundary counts by its minimum image
    q = p.copy()
    q[5, 0] += 13.0 + 0.2
    r, d = o.vnlistcheck(*_soa(q))
    assert not r and abs(d - 0.2) < 1e-9
