"""Generates the benchmark starting states (tests/golden/<workload>_state.npz).

The SiO2-like workload is built by seeded random sequential insertion
(mdff_b200.systems.sio2), which leaves ion pairs far from their minima: NVE
from there heats the glass by ~2e4 K in 25 steps.  The starting state is
therefore prepared once, on a GPU, by
  1. FIRE minimisation (displacements capped at 0.05 A, <= 300 iterations),
  2. Maxwell velocities at 300 K (seed 7),
  3. 200 velocity-Verlet steps (1 fs) rescaled to 300 K every step
     (the reference's equilibration rescale, runmd.f90:321-331),
and stored as float64 positions / velocities.  Both benchmark arms (the CUDA
engine and the CPU restatement) start from this file.

    python tests/golden/make_bench_states.py [sio2|mgo|nacl] [out_dir]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def main():
    import torch
    import bench
    from mdff_b200 import systems
    from mdff_b200.engine import ForceEngine

    name = sys.argv[1] if len(sys.argv) > 1 else "sio2"
    out_dir = sys.argv[2] if len(sys.argv) > 2 else os.path.dirname(os.path.abspath(__file__))
    s, wl = bench.make_system(name)
    dev = torch.device("cuda", 0)
    p = bench.engine_params(s, "fp64", "cg")
    eng = ForceEngine(p, s.cell)
    pos = torch.tensor(np.ascontiguousarray(s.pos.T), dtype=torch.float64, device=dev).contiguous()
    vel = torch.zeros_like(pos)
    invm = torch.tensor(1.0 / s.mass, dtype=torch.float64, device=dev)
    n_relax = bench.fire_relax(eng, pos, s.mass, 300)
    vel.copy_(torch.tensor(np.ascontiguousarray(systems.maxwell(np.random.default_rng(7), s.mass,
                                                                300.0).T), device=dev))
    dt = bench.DT_FS * 1e-3 * systems.TIME_UNIT
    bench.equilibrate(eng, pos, vel, invm, s.mass, dt, 200, 300.0, 0)
    eng.close()
    path = os.path.join(out_dir, f"{name}_state.npz")
    np.savez_compressed(path, pos=pos.cpu().numpy().T.copy(), vel=vel.cpu().numpy().T.copy(),
                        cell=s.cell, natm=s.natm, fire_iterations=n_relax,
                        protocol="FIRE<=300 (0.05 A cap), Maxwell 300 K seed 7, 200 VV steps "
                                 "rescaled to 300 K, dt 1 fs, FP64 engine with CG 1e-8")
    print(path, n_relax)


if __name__ == "__main__":
    main()
