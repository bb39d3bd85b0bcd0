"""Benchmark: PIM + Ewald MD steps/s on one B200 (and N replicas).

Workload (default): the 12,000-ion SiO2-like glass (4000 Si +2.4, 8000 O -1.2;
BKS Buckingham + r^-24 wall, O polarisability 1.3 A^3 with Tang-Toennies
damping, Ewald alpha 0.3, rc 10 A, kmax 12), seeded synthetic positions and
Maxwell velocities at 300 K.  One step = one velocity-Verlet MD step (the
engforce call of the engine plus the two kicks), positions / velocities /
forces resident in HBM.  The engine runs mixed precision (FP32 pair,
T-tensor and phase arithmetic, FP64 sums) with the CG dipole solve to the
config's 1e-8 rms tolerance.

Reported beside the headline: the plain FP64 engine (the reference's SCF
algorithm) and FP64 + CG, the RMS force error of the mixed engine vs the FP64
engine on the same configuration, e2e through the C ABI with host buffers,
roofline of the dominant kernel class, the CPU oracle baseline, clocks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from mdff_b200 import replicas  # noqa: E402

DT_FS = 1.0
# the headline metric, printed identically by both arms
METRIC = "PIM+Ewald steps/s @12k ions: mixed vs FP64 GPU (F err\u22641e-5), vs CPU host"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sio2", choices=["sio2", "mgo", "nacl"])
    ap.add_argument("--fp64-steps", type=int, default=10)
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-check", action="store_true", help="skip the mixed-vs-FP64 force check")
    ap.add_argument("--relax", type=int, default=300, help="FIRE iterations before MD")
    ap.add_argument("--equil", type=int, default=50, help="rescaled MD steps before warm-up")
    ap.add_argument("--drift-steps", type=int, default=5000, help="NVE steps for the energy drift")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-evaluation measurement")
    ap.add_argument("--no-fit", action="store_true", help="skip the fitting-gradient measurement")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the MgO 8,000 and NaCl 1,728 records")
    ap.add_argument("--write-decks", metavar="DIR", default=None,
                    help="write each workload's starting state as POSFF + control.F under DIR "
                         "(the reference's input formats) and exit")
    return ap.parse_args()


TYPE_NAMES = {"sio2": ["Si", "O"], "mgo": ["Mg", "O"], "nacl": ["Na", "Cl"]}


def write_decks(outdir):
    """The three workloads as the reference reads them: POSFF (positions and
    velocities of the starting state, types grouped) and control.F (every
    parameter as a namelist entry, calc = 'md').  The SiO2-like workload's
    r^-24 wall has no keyword in the reference: its control file says so in a
    comment, with the wall constants."""
    from mdff_b200 import mdffio
    out = {}
    for name in ("sio2", "mgo", "nacl"):
        s, wl = make_system(name)
        pos, vel = s.pos, s.vel
        st = load_state(name, s)
        if st is not None:
            pos, vel = st[0], st[1]
        p = s.params
        names = TYPE_NAMES[name]
        natmi = [int(p.natmi[t]) for t in range(p.ntype)]
        first = np.concatenate([[0], np.cumsum(natmi)[:-1]]).astype(int)
        masses = [float(s.mass[i]) for i in first]
        d = os.path.join(outdir, wl["workload"])
        os.makedirs(d, exist_ok=True)
        mdffio.write_posff(os.path.join(d, "POSFF"), wl["workload"], s.cell, names, natmi, pos, vel=vel)
        ctl = os.path.join(d, "control.F")
        mdffio.write_control(ctl, p, names, masses=masses, calc="md",
                             extra_md={"dt": DT_FS * 1e-3, "npas": 5000})
        walls = [(i, j, p.wall24[i][j]) for i in range(p.ntype) for j in range(p.ntype)
                 if p.wall24[i][j] != 0.0]
        if walls:
            with open(ctl) as f:
                body = f.read()
            note = ["! extension used by this workload, not a keyword of the reference: a W/r^24",
                    "! wall added to the Buckingham pairs (eV A^24):"]
            note += [f"!   wall24({i + 1},{j + 1}) = {w!r}" for i, j, w in walls]
            with open(ctl, "w") as f:
                f.write("\n".join(note) + "\n" + body)
        out[name] = d
    return out


def make_system(name):
    from mdff_b200 import _abi, systems
    if name == "sio2":
        # the insertion is skipped when the prepared starting state exists
        have = os.path.exists(os.path.join(ROOT, "tests", "golden", "sio2_state.npz"))
        s = systems.sio2(place=not have)
        wl = dict(workload="sio2_pim_ewald_12000", natm=s.natm, box_A=round(s.info["L"], 4),
                  rcut_A=10.0, alpha=0.3, kmax=12, pim="O 1.3 A^3 + TT damping",
                  short_range="BKS Buckingham + r^-24 wall", dt_fs=DT_FS, ensemble="NVE")
    elif name == "mgo":
        s = systems.mgo()
        wl = dict(workload="mgo_pim_ewald_8000", natm=s.natm, box_A=round(s.info["L"], 4),
                  rcut_A=10.0, alpha=0.35, kmax=s.info["kmax"], dt_fs=DT_FS, ensemble="NVE")
    else:
        s = systems.nacl()
        wl = dict(workload="nacl_bmh_ewald_1728", natm=s.natm, box_A=round(s.info["L"], 4),
                  rcut_A=12.0, alpha=0.3, kmax=10, dt_fs=DT_FS, ensemble="NVE")
    s.params.calc = _abi.CALC_MD
    return s, wl


def load_state(name, s):
    """Prepared starting state (tests/golden/make_bench_states.py), or None."""
    path = os.path.join(ROOT, "tests", "golden", f"{name}_state.npz")
    if not os.path.exists(path):
        return None
    z = np.load(path)
    if int(z["natm"]) != s.natm or not np.allclose(z["cell"], s.cell):
        return None
    return z["pos"], z["vel"], str(z["protocol"])


def engine_params(s, precision, solver):
    from mdff_b200 import _abi
    from mdff_b200.params import params_copy
    p = params_copy(s.params)
    p.precision = _abi.PREC_MIXED if precision == "mixed" else _abi.PREC_FP64
    p.solver = _abi.SOLVER_CG if solver == "cg" else _abi.SOLVER_SCF
    p.cg_tol = p.conv_tol_ind
    return p


def _physical_gpu(local_rank):
    """The device index / UUID nvidia-smi and NVML know for this rank's GPU."""
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "").strip()
    if vis:
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        if local_rank < len(ids):
            return ids[local_rank]
    return str(local_rank)


class Clocks:
    """SM clocks and clock-event reasons during the timed region: nvidia-smi
    every 200 ms and, beside it, NVML read in-process every 5 ms (the timed
    region of the default run is ~50 ms).  Reading only; nothing is set."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        gpu = _physical_gpu(gpu_index)
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={gpu}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        self.nv, self.nv_max, self.t = [], None, None
        try:
            import threading
            import pynvml as nv
            nv.nvmlInit()
            h = (nv.nvmlDeviceGetHandleByUUID(gpu) if not gpu.isdigit()
                 else nv.nvmlDeviceGetHandleByIndex(int(gpu)))
            self.nv_max = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self._nvml, self._halt = nv, threading.Event()

            def loop():
                while not self._halt.is_set():
                    try:
                        self.nv.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                        int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))))
                    except Exception:
                        return
                    self._halt.wait(0.005)

            self.t = threading.Thread(target=loop, daemon=True)
            self.t.start()
        except Exception:
            self.t = None

    def _stop_nvml(self):
        if self.t is None:
            return []
        self._halt.set()
        self.t.join(timeout=2.0)
        try:
            self._nvml.nvmlShutdown()
        except Exception:
            pass
        nv, out = self._nvml, []
        bits = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
                ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
                ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
                ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))
        for mhz, mask in list(self.nv):
            out.append((mhz, {nm for nm, c in bits if mask & int(getattr(nv, c, 0))}))
        return out

    def stop(self):
        nvml = self._stop_nvml()
        rows = []
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            self.f.flush()
            rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        try:
            os.unlink(self.f.name)
        except OSError:
            pass
        sm, mx, reasons = [], self.nv_max, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        n_smi = 0
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                n_smi += 1
                for nm, v in zip(names, r[5:9]):
                    if "Active" in v and "Not" not in v:
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        for mhz, rs in nvml:
            sm.append(mhz)
            reasons |= rs
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "samples_nvidia_smi": n_smi, "samples_nvml": len(nvml)}


def fire_relax(eng, pos, mass, iters, fmax_stop=0.5):
    """FIRE minimisation (Bitzek et al., PRL 97, 170201 (2006)) of the seeded
    random-insertion structure on the device, displacements capped at
    0.05 A per iteration: the insertion leaves ion pairs far from their
    minima and NVE from there heats the glass by thousands of K."""
    import torch
    f = torch.zeros_like(pos)
    v = torch.zeros_like(pos)
    m = torch.as_tensor(mass, dtype=torch.float64, device=pos.device)[None, :]
    dt, dtmax, a, npos = 0.02, 0.1, 0.1, 0
    eng.engforce_device(pos.data_ptr(), f.data_ptr())
    for it in range(iters):
        P = float((f * v).sum())
        if P > 0:
            npos += 1
            fn = float(f.norm())
            vn = float(v.norm())
            v = (1 - a) * v + a * vn * f / max(fn, 1e-30)
            if npos > 5:
                dt = min(dt * 1.1, dtmax)
                a *= 0.99
        else:
            npos = 0
            dt *= 0.5
            v.zero_()
            a = 0.1
        v += dt * f / m
        dx = dt * v
        mx = float(dx.abs().max())
        if mx > 0.05:
            dx *= 0.05 / mx
        pos += dx
        eng.engforce_device(pos.data_ptr(), f.data_ptr())
        if float(f.abs().max()) < fmax_stop:
            break
    return it + 1


def equilibrate(eng, pos, vel, invm, mass, dt, steps, temp, itime):
    """Velocity-Verlet with velocity rescaling to temp each step (the
    reference's equilibration rescale, runmd.f90:321-331)."""
    import torch
    from mdff_b200 import systems
    n = mass.size
    m = torch.as_tensor(mass, dtype=torch.float64, device=pos.device)[None, :]
    for _ in range(steps):
        eng.md_nve(pos.data_ptr(), vel.data_ptr(), invm.data_ptr(), dt, 1, itime, energies=False)
        itime += 1
        ek = 0.5 * float((m * vel * vel).sum())
        T = 2 * ek / (3 * n * systems.BOLTZ_UNIT)
        vel *= (temp / T) ** 0.5
    return itime


def flush_l2(buf):
    buf.add_(1.0)  # 256 MiB read + write, larger than the 126 MB L2


def run_ours(args, rank, world, local_rank):
    import torch
    from mdff_b200 import _abi, systems
    from mdff_b200.engine import ForceEngine

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    s, wl = make_system(args.workload)
    n = s.natm
    dt = DT_FS * 1e-3 * systems.TIME_UNIT
    p = engine_params(s, "mixed", "cg")
    p.device = local_rank
    eng = ForceEngine(p, s.cell)
    pos = torch.tensor(np.ascontiguousarray(s.pos.T), dtype=torch.float64, device=dev).contiguous()
    vel = torch.tensor(np.ascontiguousarray(s.vel.T), dtype=torch.float64, device=dev).contiguous()
    invm = torch.tensor(1.0 / s.mass, dtype=torch.float64, device=dev)
    l2buf = torch.zeros(256 * 2 ** 20 // 4, dtype=torch.float32, device=dev)
    itime = 0
    st0 = load_state(args.workload, s)
    if st0 is not None:
        pos.copy_(torch.tensor(np.ascontiguousarray(st0[0].T), device=dev))
        vel.copy_(torch.tensor(np.ascontiguousarray(st0[1].T), device=dev))
        wl["start"] = "tests/golden/%s_state.npz: %s" % (args.workload, st0[2])
    else:
        t_prep = time.perf_counter()
        n_relax = fire_relax(eng, pos, s.mass, args.relax) if args.relax > 0 else 0
        vel.copy_(torch.tensor(np.ascontiguousarray(
            systems.maxwell(np.random.default_rng(7), s.mass, 300.0).T), dtype=torch.float64,
            device=dev))
        itime = equilibrate(eng, pos, vel, invm, s.mass, dt, args.equil, 300.0, itime)
        wl["start"] = (f"prepared in place: FIRE {n_relax} iterations, Maxwell 300 K, {args.equil} "
                       f"rescaled VV steps ({time.perf_counter() - t_prep:.1f} s)")
    for _ in range(args.warmup):
        eng.md_nve(pos.data_ptr(), vel.data_ptr(), invm.data_ptr(), dt, 1, itime, energies=False)
        itime += 1
    torch.cuda.synchronize()
    dist_barrier(world)
    clk = Clocks(local_rank) if rank == 0 else None
    step_ms, launches, iters, rms0, nres = [], 0, [], [], []
    torch.cuda.synchronize()
    dist_barrier(world)
    for _ in range(args.steps):
        flush_l2(l2buf)
        torch.cuda.synchronize()
        eng.md_nve(pos.data_ptr(), vel.data_ptr(), invm.data_ptr(), dt, 1, itime, energies=False)
        itime += 1
        st = eng.stats()
        step_ms.append(st["ms_last"])
        launches += st["n_launches"]
        iters.append(st["n_pol_iter"])
        rms0.append(st["rmsd_initial"])
        nres.append(st["n_fp64_residuals"])
    torch.cuda.synchronize()
    dist_barrier(world)
    clocks = clk.stop() if clk else None
    # per-kernel-class CUDA-event timing: a separate pass of the same MD (the
    # events around every launch would split the CUDA graph of the CG loop)
    assert eng._lib.mdff_gpu_profile(eng._h, 1) == 0
    for _ in range(min(args.steps, 30)):
        flush_l2(l2buf)
        torch.cuda.synchronize()
        eng.md_nve(pos.data_ptr(), vel.data_ptr(), invm.data_ptr(), dt, 1, itime, energies=False)
        itime += 1
    kms = np.zeros(_abi.NKCLASS)
    kl = np.zeros(_abi.NKCLASS, dtype=np.int64)
    kw = np.zeros(_abi.NKCLASS)
    eng._lib.mdff_gpu_kernel_times(eng._h, _abi.dptr(kms), kl.ctypes.data_as(
        __import__("ctypes").POINTER(__import__("ctypes").c_longlong)), _abi.dptr(kw))
    eng._lib.mdff_gpu_profile(eng._h, 0)
    value, total_s = replicas.throughput(world, args.steps, sum(step_ms) / 1e3)
    res = dict(value=value, ms_per_step=1e3 * total_s / args.steps, launches=launches,
               cg_iters_mean=float(np.mean(iters)), clocks=clocks, wl=wl,
               cg_first_residual_rmsd_mean=float(np.mean(rms0)),
               cg_fp64_residuals_mean=float(np.mean(nres)),
               kms=kms, kl=kl, kw=kw, prof_steps=min(args.steps, 30))
    if rank != 0:
        return res, None
    # ---- extras on rank 0 ---------------------------------------------------
    extra = {}
    pos_h = pos.cpu().numpy()
    soa = tuple(np.ascontiguousarray(pos_h[a]) for a in range(3))
    hist = eng.aspc_history()
    # FP64 engines on the same trajectory point (same ASPC history)
    for tag, prec, solver in ((("fp64_scf", "fp64", "scf"), ("fp64_cg", "fp64", "cg"))
                              if args.fp64_steps > 0 else ()):
        pe = engine_params(s, prec, solver)
        pe.device = local_rank
        e2 = ForceEngine(pe, s.cell)
        pos2 = pos.clone()
        vel2 = vel.clone()
        e2.set_aspc_history(hist)
        ms, it2 = [], []
        it = itime
        for k in range(args.fp64_steps + 2):
            flush_l2(l2buf)
            torch.cuda.synchronize()
            e2.md_nve(pos2.data_ptr(), vel2.data_ptr(), invm.data_ptr(), dt, 1, it, energies=False)
            it += 1
            if k >= 2:
                st2 = e2.stats()
                ms.append(st2["ms_last"])
                it2.append(st2["n_pol_iter"])
        extra[tag + "_steps_per_s"] = 1e3 / float(np.mean(ms))
        extra[tag + "_iters_mean"] = float(np.mean(it2))
        e2.close()
    # force error of the mixed engine vs the FP64 engine (tight SCF) on one config
    if not args.no_check:
        check_force_error(extra, s, soa)
    run_e2e = args.e2e_steps is None or args.e2e_steps > 0
    ne = args.e2e_steps or args.steps
    if run_e2e:
        run_e2e_loop(extra, eng, s, soa, vel, itime, ne, l2buf, dt)
    peak32 = __import__("ctypes").c_double(0)
    peak64 = __import__("ctypes").c_double(0)
    eng._lib.mdff_gpu_peak_flops(local_rank, 0, __import__("ctypes").byref(peak32))
    eng._lib.mdff_gpu_peak_flops(local_rank, 1, __import__("ctypes").byref(peak64))
    extra["peak_fp32_tflops"] = peak32.value
    extra["peak_fp64_tflops"] = peak64.value
    # NVE energy drift (SiO2, 5000 steps in the configuration): the mixed engine
    # and the FP64 CG engine continue from the same trajectory point
    if args.drift_steps > 0:
        extra["nve_drift"] = {"steps": args.drift_steps, "dt_fs": DT_FS}
        for tag, prec in (("mixed", "mixed"), ("fp64_cg", "fp64")):
            if tag == "mixed":
                e_d = eng
                p_d, v_d, it_d = pos.clone(), vel.clone(), itime
            else:
                pe = engine_params(s, prec, "cg")
                pe.device = local_rank
                e_d = ForceEngine(pe, s.cell)
                e_d.set_aspc_history(hist)
                p_d, v_d, it_d = pos.clone(), vel.clone(), itime
            en = []
            done = 0
            while done < args.drift_steps:
                nst = min(500, args.drift_steps - done)
                en.append(e_d.md_nve(p_d.data_ptr(), v_d.data_ptr(), invm.data_ptr(), dt, nst, it_d))
                it_d += nst
                done += nst
            en = np.concatenate(en)
            etot = en[:, 0] + en[:, 1]
            t_ps = np.arange(etot.size) * DT_FS * 1e-3
            slope = np.polyfit(t_ps, etot, 1)[0]
            extra["nve_drift"][tag] = {
                "slope_meV_per_atom_per_ps": 1e3 * slope / n,
                "max_dev_meV_per_atom": 1e3 * float(np.abs(etot - etot[0]).max()) / n,
                "temperature_K_mean": float(2 * en[:, 0].mean() / (3 * n * systems.BOLTZ_UNIT)),
            }
            if tag != "mixed":
                e_d.close()
    extra["stats"] = eng.stats()
    extra["_cpu_point"] = (soa, hist, itime)
    eng.close()
    if not args.no_cpu:
        extra["_at_point"] = gpu_at_point(s, hist, itime, soa, local_rank)
    return res, extra


def check_force_error(extra, s, soa):
    from mdff_b200 import _abi
    from mdff_b200.engine import ForceEngine
    pt = engine_params(s, "fp64", "scf")
    pt.conv_tol_ind = 1e-11
    pt.max_scf_pol_iter = 400
    pt.calc = _abi.CALC_OTHER
    e3 = ForceEngine(pt, s.cell)
    ref = e3.engforce(*soa)
    e3.close()
    pm = engine_params(s, "mixed", "cg")
    pm.calc = _abi.CALC_OTHER
    e4 = ForceEngine(pm, s.cell)
    mix = e4.engforce(*soa)
    e4.close()
    fr = np.stack([ref["fx"], ref["fy"], ref["fz"]], 1)
    fm = np.stack([mix["fx"], mix["fy"], mix["fz"]], 1)
    extra["force_err_rms_rel_vs_fp64"] = float(np.sqrt(((fm - fr) ** 2).sum() / (fr ** 2).sum()))
    extra["dipole_err_rms_rel_vs_fp64"] = float(np.sqrt(((mix["mu"] - ref["mu"]) ** 2).sum()
                                                        / (ref["mu"] ** 2).sum()))
    extra["energy_err_rel_vs_fp64"] = abs(mix["u_coul"] + mix["u_bmhft"] - ref["u_coul"]
                                          - ref["u_bmhft"]) / abs(ref["u_coul"] + ref["u_bmhft"])


def run_e2e_loop(extra, eng, s, soa, vel, itime, ne, l2buf, dt):
    """End to end through the C ABI as a host caller (the Fortran shim) runs
    it: positions in, forces and dipoles out, in caller-owned pinned host
    arrays reused every step (one mdff_result), the integrator on the host."""
    import ctypes
    import torch
    from mdff_b200 import _abi
    n = s.natm
    pin = lambda *shape: torch.zeros(*shape, dtype=torch.float64, pin_memory=True).numpy()
    r3 = pin(3, n)
    f3 = pin(3, n)
    mu = pin(n, 3)
    r3[:] = np.stack(soa)
    v_h = np.ascontiguousarray(vel.cpu().numpy())
    kick = (0.5 * dt / s.mass)[None, :]
    res = _abi.MdffResult()
    res.fx, res.fy, res.fz = (_abi.dptr(f3[a]) for a in range(3))
    res.mu = _abi.dptr(mu)
    args = [eng._h] + [_abi.dptr(r3[a]) for a in range(3)]
    call = eng._lib.mdff_gpu_engforce
    tmp = np.empty_like(v_h)

    def engforce(it):
        st = call(*args, int(it), ctypes.byref(res))
        if st != 0:
            raise _abi.MdffError(st, "engforce")

    engforce(itime)
    e_ms, wall = [], []
    for k in range(ne):
        flush_l2(l2buf)
        torch.cuda.synchronize()
        # wall clock of one whole step: kick + drift on the host, the ABI call
        # (positions in, forces and dipoles out), kick
        t0 = time.perf_counter()
        np.multiply(f3, kick, out=tmp)
        v_h += tmp
        np.multiply(v_h, dt, out=tmp)
        r3 += tmp
        itime += 1
        engforce(itime)
        np.multiply(f3, kick, out=tmp)
        v_h += tmp
        wall.append(time.perf_counter() - t0)
        e_ms.append(eng.stats()["ms_last"])
    extra["e2e"] = {"value": ne / float(np.sum(wall)), "unit": "steps/s",
                    "h2d_bytes_per_step": 3 * n * 8, "d2h_bytes_per_step": 3 * n * 8 * 2 + 8 * 7 + 8 * 27,
                    "timing": "host wall clock (perf_counter) per step: host integrator + "
                              "mdff_gpu_engforce with pinned host arrays",
                    "device_span_value": 1e3 / float(np.mean(e_ms))}


def dist_barrier(world):
    replicas.barrier(world)


def host_cores(threads):
    """Threads the CPU leg used and what the host offers."""
    try:
        aff = len(os.sched_getaffinity(0))
    except AttributeError:
        aff = None
    return {"cores": threads, "host_cpus": os.cpu_count(), "host_cpus_usable": aff}


def cpu_baseline_sample(s, hist, itime, pos_soa):
    """Oracle (C restatement of the reference engforce, OpenMP over all host
    threads): one warm-start engforce (SCF, ASPC history from the GPU run) of
    the same workload = one MD step of the reference algorithm.  Its result is
    also the FP64 reference the GPU engines' errors are stated against."""
    from oracle import oracle as O
    from mdff_b200.params import params_copy
    o = O.Oracle(params_copy(s.params), s.cell)
    o.set_aspc(hist)
    t = time.perf_counter()
    r = o.engforce(*pos_soa, itime=itime)
    dt_s = time.perf_counter() - t
    return dt_s, r["n_scf"], O.lib().or_get_threads(), r


def gpu_at_point(s, hist, itime, soa, local_rank):
    """One engforce of the FP64 engine (the reference's SCF) and of the mixed
    engine (CG) at a trajectory point, both with the run's ASPC history: the
    results compared with the oracle's at the same point."""
    from mdff_b200.engine import ForceEngine
    out = {}
    for tag, prec, solver in (("fp64_scf", "fp64", "scf"), ("mixed", "mixed", "cg")):
        p = engine_params(s, prec, solver)
        p.device = local_rank
        with ForceEngine(p, s.cell) as e:
            e.set_aspc_history(hist)
            r = e.engforce(*soa, itime=itime)
            r["n_iter"] = e.stats()["n_pol_iter"]
        out[tag] = r
    return out


def errors_vs_oracle(g, o):
    """Relative errors of a GPU result g against the oracle's o: RMS and max
    over the forces, RMS over the dipoles, total energy."""
    fg = np.stack([g["fx"], g["fy"], g["fz"]], 1)
    fo = np.stack([o["fx"], o["fy"], o["fz"]], 1)
    ug = g["u_coul"] + g["u_bmhft"] + g["u_lj"]
    uo = o["u_coul"] + o["u_bmhft"] + o["u_lj"]
    mo = float((o["mu"] ** 2).sum())
    return {"force_rms_rel": float(np.sqrt(((fg - fo) ** 2).sum() / (fo ** 2).sum())),
            "force_max_rel": float(np.abs(fg - fo).max() / np.abs(fo).max()),
            "dipole_rms_rel": float(np.sqrt(((g["mu"] - o["mu"]) ** 2).sum() / mo)) if mo > 0 else 0.0,
            "energy_rel": float(abs(ug - uo) / abs(uo))}


KCLS = ("list_build", "short_range", "real_space_field", "real_space_force",
        "structure_factor", "reciprocal_field", "other")

# DRAM bytes (read + write) per launch of each class's main kernel on the 12k
# SiO2 workload, from one ncu capture (profiles/k_rec_rho_tc_k_rec_field_tc_sio2_12000.md,
# profiles/realspace_kernels_sio2_12000.md); the working set is L2-resident
TRAFFIC = {
    "structure_factor": {"kernel": "k_rec_rho_tc", "bytes": 4.211e6},
    "reciprocal_field": {"kernel": "k_rec_field_tc<0, 32>", "bytes": 4.118e6},
    "real_space_force": {"kernel": "k_es_force<float>", "bytes": 20.09e6},
    "short_range": {"kernel": "k_shortrange<double, 1>", "bytes": 18.96e6},
    "real_space_field": {"kernel": "k_static_cache", "bytes": 20.27e6},
}


def roofline_block(res, extra):
    kms, kl, kw = res["kms"], res["kl"], res["kw"]
    c = int(np.argmax(kms))
    if kw[c] == 0:
        # dominant class without an algorithmic op count: report the reciprocal one
        c = 4 if kms[4] >= kms[5] else 5
    avg_ms = kms[c] / max(kl[c], 1)
    ops_per_launch = kw[c] / max(kl[c], 1)
    achieved = ops_per_launch / (avg_ms * 1e-3) / 1e12
    peak = extra["peak_fp32_tflops"]
    share = {KCLS[i]: round(float(kms[i] / kms.sum()), 4) for i in range(len(KCLS)) if kms[i] > 0}
    # kernel time per step of each class in the profiling pass (one stream,
    # events around every launch), against the overlapped step's ms_per_step
    per_step = {KCLS[i]: round(float(kms[i] / res["prof_steps"]), 4)
                for i in range(len(KCLS)) if kms[i] > 0}
    tr = TRAFFIC.get(KCLS[c])
    return {"kernel": KCLS[c], "bound": "fp32_fma", "achieved": round(achieved, 3),
            "peak": round(peak, 3), "unit": "TFLOP/s", "frac": round(achieved / peak, 4),
            "traffic": tr["bytes"] if tr else None,
            "traffic_kernel": tr["kernel"] if tr else None,
            "launches": int(kl[c]), "avg_launch_ms": round(avg_ms, 5),
            "peak_source": "measured live: register-resident FP32 FMA loop on all SMs (mdff_gpu_peak_flops); "
                           "MEASURED_PEAKS.json has HBM and bf16 tensor peaks only",
            "note": "achieved counts algorithmic ops of the class (all its launches); the FP32 CG-operator "
                    "launches of the reciprocal classes run on the tcgen05 tensor cores (split TF32), so "
                    "frac compares with the CUDA-core FP32 ceiling",
            "time_share": share, "class_ms_per_step": per_step}


def run_reference(args, rank, world):
    if rank != 0:
        return
    from mdff_b200 import systems
    from oracle import oracle as O
    from mdff_b200.params import params_copy
    s, wl = make_system(args.workload)
    o = O.Oracle(params_copy(s.params), s.cell)
    dt = DT_FS * 1e-3 * systems.TIME_UNIT
    st0 = load_state(args.workload, s)
    pos = (st0[0] if st0 is not None else s.pos).copy()
    vel = (st0[1] if st0 is not None else s.vel).copy()
    wl["start"] = ("tests/golden/%s_state.npz" % args.workload) if st0 is not None else \
        "random-insertion state (no prepared state file)"
    invm = (1.0 / s.mass)[:, None]
    soa = lambda p: tuple(np.ascontiguousarray(p[:, a]) for a in range(3))
    r = o.engforce(*soa(pos), itime=0)
    f = np.stack([r["fx"], r["fy"], r["fz"]], 1)
    times = []
    itime = 0
    for k in range(args.warmup + args.steps):
        vel += 0.5 * dt * f * invm
        pos += dt * vel
        itime += 1
        t = time.perf_counter()
        r = o.engforce(*soa(pos), itime=itime)
        el = time.perf_counter() - t
        f = np.stack([r["fx"], r["fy"], r["fz"]], 1)
        vel += 0.5 * dt * f * invm
        if k >= args.warmup:
            times.append(el)
    tot = sum(times)
    val = args.steps / tot
    cores = O.lib().or_get_threads()
    line = {"metric": METRIC, "impl": "reference", "value": val,
            "unit": "steps/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": dict(wl, solver="scf (reference algorithm)", precision="fp64"),
            "cpu_baseline": dict({"value": val, "unit": "steps/s", "kind": "port",
                                  "sample": f"{args.steps} MD steps (velocity Verlet, warm ASPC) of the "
                                            f"{wl['natm']}-ion workload, C restatement of engforce, "
                                            f"OpenMP {cores} threads"}, **host_cores(cores)),
            "e2e": {"value": val, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_config_record(name, local_rank, l2buf, steps=20, warmup=5, fp64_steps=10, cpu=True):
    """One of the other single-box workloads (MgO 8,000 ions, NaCl 1,728 ions)
    from its seeded lattice start: velocity-Verlet MD steps/s of the mixed
    engine and of the FP64 engine (the reference's SCF; FP64 + CG too when
    the ions are polarisable), device-timed with L2 flushed before each step;
    at the last configuration, one engforce of each engine and, with cpu, one
    warm-start oracle engforce (the CPU figure of this workload) against which
    their errors are stated."""
    import torch
    from mdff_b200 import systems
    from mdff_b200.engine import ForceEngine
    dev = torch.device("cuda", local_rank)
    s, wl = make_system(name)
    pim = bool(s.params.ldip_polar[1])
    dt = DT_FS * 1e-3 * systems.TIME_UNIT
    pos = torch.tensor(np.ascontiguousarray(s.pos.T), dtype=torch.float64, device=dev).contiguous()
    vel = torch.tensor(np.ascontiguousarray(s.vel.T), dtype=torch.float64, device=dev).contiguous()
    invm = torch.tensor(1.0 / s.mass, dtype=torch.float64, device=dev)
    out = {"config": dict(wl, start=f"seeded rock-salt lattice + jitter, Maxwell velocities "
                                     f"(seed {s.info['seed']})")}
    if "epsw" in s.info:
        out["config"]["epsw"] = s.info["epsw"]
    p = engine_params(s, "mixed", "cg")
    p.device = local_rank
    eng = ForceEngine(p, s.cell)
    itime = 0
    for _ in range(warmup):
        eng.md_nve(pos.data_ptr(), vel.data_ptr(), invm.data_ptr(), dt, 1, itime, energies=False)
        itime += 1
    ms, its = [], []
    for _ in range(steps):
        flush_l2(l2buf)
        torch.cuda.synchronize()
        eng.md_nve(pos.data_ptr(), vel.data_ptr(), invm.data_ptr(), dt, 1, itime, energies=False)
        itime += 1
        st = eng.stats()
        ms.append(st["ms_last"])
        its.append(st["n_pol_iter"])
    out["mixed"] = {"steps_per_s": 1e3 / float(np.mean(ms)), "ms_per_step": float(np.mean(ms)),
                    "cg_iters_mean": float(np.mean(its)), "nk": st["nk"], "kES": st["kES"]}
    pos_h = pos.cpu().numpy()
    soa = tuple(np.ascontiguousarray(pos_h[a]) for a in range(3))
    hist = eng.aspc_history()
    eng.close()
    runs = [("fp64_scf", "fp64", "scf")] + ([("fp64_cg", "fp64", "cg")] if pim else [])
    for tag, prec, solver in runs:
        pe = engine_params(s, prec, solver)
        pe.device = local_rank
        with ForceEngine(pe, s.cell) as e2:
            e2.set_aspc_history(hist)
            p2, v2, it = pos.clone(), vel.clone(), itime
            ms, its = [], []
            for k in range(fp64_steps + 2):
                flush_l2(l2buf)
                torch.cuda.synchronize()
                e2.md_nve(p2.data_ptr(), v2.data_ptr(), invm.data_ptr(), dt, 1, it, energies=False)
                it += 1
                if k >= 2:
                    st = e2.stats()
                    ms.append(st["ms_last"])
                    its.append(st["n_pol_iter"])
        out[tag] = {"steps_per_s": 1e3 / float(np.mean(ms)), "ms_per_step": float(np.mean(ms)),
                    "iters_mean": float(np.mean(its))}
    for tag in [r[0] for r in runs]:
        out["speedup_mixed_vs_" + tag] = out["mixed"]["steps_per_s"] / out[tag]["steps_per_s"]
    if cpu:
        at = gpu_at_point(s, hist, itime, soa, local_rank)
        dt_s, nscf, cores, ro = cpu_baseline_sample(s, hist, itime, soa)
        out["cpu_baseline"] = dict({"value": 1.0 / dt_s, "unit": "steps/s", "kind": "port",
                                    "sample": f"one warm-start engforce (= one MD step, {nscf} SCF "
                                              f"iterations) at the last configuration"},
                                   **host_cores(cores))
        out["vs_oracle"] = {
            "fp64_scf": dict(errors_vs_oracle(at["fp64_scf"], ro), scf_iters=at["fp64_scf"]["n_iter"],
                             oracle_scf_iters=nscf),
            "mixed": dict(errors_vs_oracle(at["mixed"], ro), cg_iters=at["mixed"]["n_iter"])}
    torch.cuda.synchronize()
    return out


def run_batch_bench(local_rank, cpu=True):
    """Batched evaluation: 256 independent rock-salt boxes (NaCl / MgO type,
    64-1000 ions, seed 99) per call through the persistent cluster kernel;
    mixed and FP64, launch shape from the autotuner, device time (CUDA events
    in the library) and end to end with host arrays."""
    import torch
    from mdff_b200 import _abi, systems
    from mdff_b200.engine import BatchEngine
    out = {"workload": "256 cubic rock-salt boxes, NaCl/MgO type, 64-1000 ions (seed 99)"}
    forces = {}
    for prec, tag in ((_abi.PREC_MIXED, "mixed"), (_abi.PREC_FP64, "fp64")):
        ps, cf, pos = systems.batch(nconf=256, seed=99, precision=prec)
        P = np.concatenate(pos)
        for p in ps:
            p.device = local_rank
        with BatchEngine(ps, cf) as eng:
            r = eng.engforce(P[:, 0], P[:, 1], P[:, 2])
            shape = eng.tune()
            ms = []
            for _ in range(10):
                eng.engforce(P[:, 0], P[:, 1], P[:, 2])
                ms.append(eng.info()["ms_last"])
            # end to end: host positions in, host forces / dipoles / fields out
            t0 = time.perf_counter()
            for _ in range(5):
                r = eng.engforce(P[:, 0], P[:, 1], P[:, 2])
            e2e = (time.perf_counter() - t0) / 5
            forces[tag] = np.stack([r["fx"], r["fy"], r["fz"]], 1)
            its = [c["n_pol_iter"] for c in r["conf"] if c["n_pol_iter"] > 0]
            out[tag] = {"ms": float(np.median(ms)), "configs_per_s": 256e3 / float(np.median(ms)),
                        "ions_per_s": eng.ntot * 1e3 / float(np.median(ms)),
                        "e2e_configs_per_s": 256 / e2e, "shape": {"cluster": shape[0],
                                                                   "threads": shape[1]},
                        "cg_iters_mean": float(np.mean(its)) if its else 0.0}
            out["ntot"] = eng.ntot
    f64 = forces["fp64"]
    out["force_err_rms_rel_mixed_vs_fp64"] = float(np.sqrt(((forces["mixed"] - f64) ** 2).sum() /
                                                           (f64 ** 2).sum()))
    if cpu:
        # CPU oracle on a sample of the same boxes (OpenMP, all host threads)
        from oracle import oracle as orc
        ps, cf, pos = systems.batch(nconf=256, seed=99, precision=_abi.PREC_FP64)
        idx = list(range(0, 256, 32))
        t0 = time.perf_counter()
        nat = 0
        for k in idx:
            p = systems.config_params(ps, cf[k])
            p.solver = _abi.SOLVER_SCF
            orc.Oracle(p, cf[k][2]).engforce(pos[k][:, 0], pos[k][:, 1], pos[k][:, 2])
            nat += pos[k].shape[0]
        dt = time.perf_counter() - t0
        out["cpu_oracle"] = {"configs_per_s": len(idx) / dt, "sample": f"{len(idx)} of the 256 boxes "
                             f"({nat} ions), SCF to 1e-8", "cores": orc.lib().or_get_threads()}
    torch.cuda.synchronize()
    return out


def run_fit_bench(local_rank):
    """Differentiable fitting: 64 MgO-type boxes of 216-512 ions, 10 parameters,
    force-matching loss against forces of the FP64 engine at parameters
    perturbed by 5 % (seeded).  Times one loss + gradient (forward + adjoint),
    checks the gradient against central differences (h = 1e-5 relative) and
    runs a short L-BFGS fit from the unperturbed start."""
    import torch
    from mdff_b200 import fit
    psets, configs, pos, theta_true = fit.fitting_workload()
    for p in psets:
        p.device = local_rank
    ff = fit.BatchForceField(psets, configs, fit.MGO_FIT)
    Fn = fit.EngForceFn()
    P = torch.tensor(np.ascontiguousarray(np.concatenate(pos).T), dtype=torch.float64,
                     device=f"cuda:{local_rank}")
    with torch.no_grad():
        Ft = Fn.apply(torch.tensor(theta_true), ff, P)[1].clone()
    theta0 = ff.theta0.copy()

    def loss_grad(th_np):
        th = torch.tensor(th_np, dtype=torch.float64, requires_grad=True)
        U, F, mu = Fn.apply(th, ff, P)
        loss = ((F - Ft) ** 2).sum()
        loss.backward()
        return float(loss.detach()), th.grad.numpy().copy()

    loss_grad(theta0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(5):
        l0, g0 = loss_grad(theta0)
    torch.cuda.synchronize()
    t_lg = (time.perf_counter() - t0) / 5
    info = ff.engine.info()
    # central differences of the loss
    fd = np.zeros_like(theta0)
    for k in range(theta0.size):
        h = 1e-5 * max(abs(theta0[k]), 1.0)
        tp, tm = theta0.copy(), theta0.copy()
        tp[k] += h
        tm[k] -= h
        with torch.no_grad():
            lp = float(((Fn.apply(torch.tensor(tp), ff, P)[1] - Ft) ** 2).sum())
            lm = float(((Fn.apply(torch.tensor(tm), ff, P)[1] - Ft) ** 2).sum())
        fd[k] = (lp - lm) / (2 * h)
    sc = np.maximum(np.abs(theta0), 1.0)
    err = np.abs(sc * (g0 - fd)) / np.abs(sc * fd).max()
    # short fit in scaled variables
    from scipy.optimize import minimize
    res = minimize(lambda z: (lambda lg: (lg[0], lg[1] * sc))(loss_grad(z * sc)), theta0 / sc,
                   jac=True, method="L-BFGS-B", options={"maxiter": 40})
    th_fit = res.x * sc
    ff.close()
    return {"workload": "64 MgO-type boxes, 216-512 ions, 10 parameters, FP64 (seed 2027)",
            "ntot": int(P.shape[1]), "ms_loss_and_grad": 1e3 * t_lg,
            "ms_forward_device": info["ms_last"], "loss0": l0,
            "fd_check_max_scaled_err": float(err.max()),
            "fd_check": dict(zip(fit.param_names(fit.MGO_FIT), [float(e) for e in err])),
            "lbfgs": {"iterations": int(res.nit), "evaluations": int(res.nfev),
                      "loss_final": float(res.fun),
                      "max_rel_err_vs_true_params": float(np.max(np.abs(th_fit - theta_true) /
                                                                 np.maximum(np.abs(theta_true), 1.0)))}}


def main():
    args = parse()
    if args.write_decks:
        for name, d in write_decks(args.write_decks).items():
            print(f"{name}: {d}")
        return
    rank, world, local_rank = replicas.world()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from mdff_b200 import build
    build.build()
    res, extra = run_ours(args, rank, world, local_rank)
    if rank == 0:
        wl = res["wl"]
        line = {
            "metric": METRIC,
            "value": res["value"], "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded)",
            "config": dict(wl, precision="mixed", solver="cg", cg_tol=1e-8,
                           parallelism=f"replicas x{world}",
                           l2="flushed between steps (256 MiB write)"),
            "ns_per_day": res["value"] / world * 86400 * DT_FS * 1e-6,
            "atom_steps_per_s": res["value"] * wl["natm"],
            "cg_iters_mean": res["cg_iters_mean"],
            "cg_first_residual_rmsd_mean": res["cg_first_residual_rmsd_mean"],
            "cg_fp64_residuals_mean": res["cg_fp64_residuals_mean"],
            "gpu_launches": int(res["launches"]),
            "clocks": res["clocks"],
        }
        line.update({k: v for k, v in extra.items() if not k.startswith("_") and k != "stats"})
        if "fp64_scf_steps_per_s" in extra:
            line["speedup_vs_fp64_scf"] = res["value"] / world / extra["fp64_scf_steps_per_s"]
            line["speedup_vs_fp64_cg"] = res["value"] / world / extra["fp64_cg_steps_per_s"]
        line["roofline"] = roofline_block(res, extra)
        if world == 1 and not args.no_cpu:
            s, _ = make_system(args.workload)
            soa, hist, itime = extra["_cpu_point"]
            dt_s, nscf, cores, ro = cpu_baseline_sample(s, hist, itime, soa)
            line["cpu_baseline"] = dict({
                "value": 1.0 / dt_s, "unit": "steps/s", "kind": "port",
                "sample": f"one warm-start engforce (= one MD step, SCF to 1e-8, {nscf} iterations) "
                          f"of the {wl['natm']}-ion workload at the GPU run's last configuration; "
                          f"C restatement of the reference engforce, OpenMP {cores} threads"},
                **host_cores(cores))
            at = extra["_at_point"]
            line["vs_oracle"] = {
                "point": "the GPU run's last configuration, ASPC history of the run, calc md; "
                         "oracle = C restatement of engforce (FP64, SCF to 1e-8)",
                "oracle_scf_iters": nscf,
                "fp64_scf": dict(errors_vs_oracle(at["fp64_scf"], ro), scf_iters=at["fp64_scf"]["n_iter"]),
                "mixed": dict(errors_vs_oracle(at["mixed"], ro), cg_iters=at["mixed"]["n_iter"])}
            line["force_err_rms_rel_vs_oracle"] = line["vs_oracle"]["mixed"]["force_rms_rel"]
        if world == 1 and not args.no_configs and args.workload == "sio2":
            import torch
            l2buf = torch.zeros(256 * 2 ** 20 // 4, dtype=torch.float32, device=f"cuda:{local_rank}")
            line["configs"] = {n: run_config_record(n, local_rank, l2buf, cpu=not args.no_cpu)
                               for n in ("mgo", "nacl")}
            del l2buf
        if world == 1 and not args.no_batch:
            line["batch"] = run_batch_bench(local_rank, cpu=not args.no_cpu)
        if world == 1 and not args.no_fit:
            line["fitting"] = run_fit_bench(local_rank)
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
