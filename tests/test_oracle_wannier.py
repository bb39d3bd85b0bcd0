"""Wannier-centre dipoles of get_dipole_moments (moment_from_pola.f90:136-147,
632-807) in the oracle, on the CPU: the dipole of each O is -2 times the sum
of its centres' minimum-image offsets (computed here independently with
numpy), the centres themselves carry none, ldip_wfc switches them out of the
Coulomb pass, and a missing centre is an error."""
import numpy as np
import pytest

from mdff_b200 import _abi, mdffio, systems
from mdff_b200.params import params_copy


def test_wfc_dipoles_match_offsets(oracle):
    s = systems.wannier_box(calc=_abi.CALC_OTHER)
    o = oracle.Oracle(s.params, s.cell).engforce(*s.soa())
    n, L = 16, s.info["L"]
    ref = np.zeros((n, 3))
    for k in range(n):
        d = s.pos[2 * n + 4 * k: 2 * n + 4 * k + 4] - s.pos[n + k]
        d -= L * np.round(d / L)
        ref[k] = -2.0 * d.sum(0)
    # O: induced dipoles are zero (not polarisable), so mu is the centres' dipole
    assert np.abs(o["mu"][n:2 * n] - ref).max() <= 1e-13 * np.abs(ref).max()
    assert np.abs(o["mu"][2 * n:]).max() == 0.0
    q = params_copy(s.params)
    q.ldip_wfc = 0
    o2 = oracle.Oracle(q, s.cell).engforce(*s.soa())
    assert np.abs(o2["mu"][n:2 * n]).max() == 0.0
    assert np.abs(o2["fx"] - o["fx"]).max() > 1.0


def test_missing_centre_is_an_error(oracle):
    s = systems.wannier_box(calc=_abi.CALC_OTHER)
    q = params_copy(s.params)
    q.lwfc[1] = 5
    with pytest.raises(_abi.MdffError) as e:
        oracle.Oracle(q, s.cell).engforce(*s.soa())
    assert e.value.status == _abi.MDFF_ERR_BAD_ARGS


def test_wannier_keywords(tmp_path):
    nl = {"pimtag": {"lwfc": [0, 4, -1], "ldip_wfc": False, "rcut_wfc": 0.4}}
    p = mdffio.params_from_namelists(nl, [2, 2, 8])
    assert list(p.lwfc[:3]) == [0, 4, -1] and p.ldip_wfc == 0 and p.rcut_wfc == 0.4
    f = tmp_path / "control.F"
    mdffio.write_control(f, p, ["M", "O", "W"])
    r = mdffio.params_from_namelists(mdffio.read_control(f), [2, 2, 8])
    assert list(r.lwfc[:3]) == [0, 4, -1] and r.ldip_wfc == 0 and r.rcut_wfc == 0.4
    d = mdffio.params_from_namelists({}, [2, 2])
    assert list(d.lwfc[:2]) == [0, 0] and d.ldip_wfc == 1 and d.rcut_wfc == 0.5


def test_dipwfc_layout(tmp_path):
    f = tmp_path / "DIPWFC"
    mdffio.write_dipwfc(f, ["M", "O", "W"], [1, 1, 2], [[0, 0, 0], [0.25, -1.5e-3, 0.0], [0, 0, 0], [0, 0, 0]],
                        [0, 4, -1])
    lines = f.read_text().splitlines()
    # '(a,3e16.8)': a3 label then three E16.8 fields; centres (lwfc < 0) left out
    assert lines == ["M    0.00000000E+00  0.00000000E+00  0.00000000E+00",
                     "O    0.25000000E+00 -0.15000000E-02  0.00000000E+00"]
