"""A C host program (tests/c_abi/engforce_host.c, gcc, linked against the
library) drives create -> engforce -> destroy on the GPU the way the Fortran
shim does; its forces, dipoles and energies equal the Python path's and
match the CPU oracle to 1e-10."""
import subprocess

import numpy as np
import pytest

from mdff_b200 import _abi, systems
from mdff_b200.engine import ForceEngine

from .c_abi.build_host import compile_c
from .gpu_util import forces, rel

pytestmark = pytest.mark.gpu


def test_c_host_matches_python_and_oracle(oracle, tmp_path):
    exe = compile_c("engforce_host", tmp_path)
    if exe is None:
        pytest.skip("no C compiler")
    s = systems.random_ionic((20, 20), L=12.5, seed=61, pol=(0.8, 1.1), calc=_abi.CALC_OTHER,
                             conv_tol_ind=1e-12, max_scf_pol_iter=400)
    n = s.natm
    (tmp_path / "p.bin").write_bytes(bytes(s.params))
    np.ascontiguousarray(s.cell, dtype=np.float64).tofile(str(tmp_path / "c.bin"))
    np.ascontiguousarray(np.concatenate(s.soa())).tofile(str(tmp_path / "x.bin"))
    r = subprocess.run([exe, str(tmp_path / "p.bin"), str(tmp_path / "c.bin"), str(tmp_path / "x.bin"),
                        str(tmp_path / "o.bin"), "2"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = np.fromfile(str(tmp_path / "o.bin"), dtype=np.float64)
    assert out.size == 6 * n + 3
    fc = np.stack([out[:n], out[n:2 * n], out[2 * n:3 * n]], 1)
    muc = out[3 * n:6 * n].reshape(n, 3)
    with ForceEngine(s.params, s.cell) as eng:
        eng.engforce(*s.soa(), itime=0)
        g = eng.engforce(*s.soa(), itime=1)
    assert rel(fc, forces(g)) <= 1e-13 and rel(muc, g["mu"]) <= 1e-13
    assert abs(out[6 * n + 1] - g["u_coul"]) <= 1e-13 * abs(g["u_coul"])
    o = oracle.Oracle(s.params, s.cell).engforce(*s.soa())
    assert rel(fc, forces(o)) <= 1e-10 and rel(muc, o["mu"]) <= 1e-10
    assert abs(out[6 * n + 1] - o["u_coul"]) <= 1e-10 * abs(o["u_coul"])
    assert abs(out[6 * n] - o["u_bmhft"]) <= 1e-10 * abs(o["u_bmhft"])
