"""The device Verlet-list rebuild schedule against the reference's
vnlistcheck (tools.f90:444-537), restated in the oracle.

A velocity-Verlet trajectory of molten NaCl (1,728 ions, 1200 K, rc 8 A and a
0.3 A skin, so 4 cells per axis and a rebuild every few steps) is driven by
the FP64 engine through the C ABI.  At every step the engine checks its list
(largest + second largest minimum-image displacement since the last build,
compared with skindiff by `.gt.`) and rebuilds on the device; the oracle's
vnlistcheck run on the same positions must ask for a rebuild on exactly the
same steps, and the forces computed from the possibly stale device list must
equal the oracle's, whose pair loops scan all ions, at every step.
"""
import numpy as np
import pytest

from mdff_b200 import _abi, systems
from mdff_b200.engine import ForceEngine
from mdff_b200.params import params_copy

from .gpu_util import cells_per_axis, compare, forces

pytestmark = pytest.mark.gpu

NSTEPS = 60


def test_rebuild_steps_match_vnlistcheck(oracle):
    s = systems.nacl(ncell=6, rcut=8.0, skin=0.3, calc=_abi.CALC_OTHER)
    assert min(cells_per_axis(s, 1)) >= 3
    orc = oracle.Oracle(params_copy(s.params), s.cell)
    dt = 1e-3 * systems.TIME_UNIT           # 1 fs
    invm = (1.0 / s.mass)[:, None]
    pos = s.pos.copy()
    vel = s.vel.copy()
    rebuilt_gpu, rebuilt_orc, disp_orc = [], [], []
    with ForceEngine(params_copy(s.params), s.cell) as eng:
        last = 0
        for t in range(NSTEPS + 1):
            soa = tuple(np.ascontiguousarray(pos[:, a]) for a in range(3))
            g = eng.engforce(*soa)
            nreb = eng.stats()["list_rebuilds"]
            rebuilt_gpu.append(nreb - last)
            last = nreb
            r, d = orc.vnlistcheck(*soa)
            rebuilt_orc.append(int(r))
            disp_orc.append(d)
            o = orc.engforce(*soa)
            compare(g, o, 1e-9, check_mu=False)
            f = forces(g)
            if t > 0:
                vel += 0.5 * dt * f * invm   # second kick of the previous step
            if t < NSTEPS:
                vel += 0.5 * dt * f * invm
                pos += dt * vel
    # step 0 builds on both sides (the oracle's stored coordinates start at zero)
    assert rebuilt_gpu[0] == 1 and rebuilt_orc[0] == 1
    assert rebuilt_gpu == rebuilt_orc, (rebuilt_gpu, rebuilt_orc)
    assert sum(rebuilt_gpu[1:]) >= 4, "the trajectory should cross the skin several times"
    # the steps in between stay within the skin
    for t in range(1, NSTEPS + 1):
        if not rebuilt_orc[t]:
            assert disp_orc[t] <= s.params.skindiff
