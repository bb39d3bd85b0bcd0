"""Batched engine (mdff_gpu_batch_*): every configuration of a batch must
equal the single-configuration engforce on the same inputs.

FP64: against the CPU oracle per configuration (the reference's SCF run to a
tight tolerance; the batch's PCG to the same tolerance), 1e-9 relative on
polarisable boxes (two converged solvers), 1e-10 elsewhere.  Mixed precision:
force error <= 1e-5 relative RMS against the FP64 batch.  Edge cases: the
reference's ex04 decks (static dipoles, reduced units, surface term, four
types), a triclinic box, boxes smaller than the cluster, every launch shape."""
import numpy as np
import pytest

from mdff_b200 import _abi, systems
from mdff_b200.engine import BatchEngine, ForceEngine
from mdff_b200.params import params_copy

from .gpu_util import compare, forces, rel, rms_rel, small_systems

pytestmark = pytest.mark.gpu


def _tight(p, tol=1e-12):
    p = params_copy(p)
    p.conv_tol_ind = tol
    p.cg_tol = tol
    p.max_scf_pol_iter = 2000
    p.cg_max_iter = 2000
    p.calc = _abi.CALC_OTHER
    return p


def _as_batch(syslist, precision=_abi.PREC_FP64, tol=1e-12):
    psets, configs, pos = [], [], []
    for k, s in enumerate(syslist):
        p = _tight(s.params, tol)
        p.precision = precision
        p.solver = _abi.SOLVER_CG
        psets.append(p)
        configs.append((k, [p.natmi[t] for t in range(p.ntype)], s.cell))
        pos.append(s.pos)
    return psets, configs, pos


def _split(out, eng):
    res = []
    for c in range(eng.nconf):
        a, b = eng.offsets[c], eng.offsets[c + 1]
        d = {k: out[k][a:b] for k in ("fx", "fy", "fz", "mu", "ef")}
        d.update(out["conf"][c])
        res.append(d)
    return res


def _run(psets, configs, pos, shape=None):
    with BatchEngine(psets, configs) as eng:
        if shape:
            eng.set_shape(*shape)
        P = np.concatenate(pos)
        out = eng.engforce(P[:, 0], P[:, 1], P[:, 2])
        return _split(out, eng), eng.offsets


def _oracle_of(oracle, psets, conf, pos):
    p = systems.config_params(psets, conf)
    p.solver = _abi.SOLVER_SCF
    o = oracle.Oracle(p, conf[2])
    return o.engforce(pos[:, 0], pos[:, 1], pos[:, 2])


EDGE = [s for s in small_systems() if s.params.ntype <= _abi.BATCH_MAXTYPES]


@pytest.mark.parametrize("shape", [(2, 256), (8, 256)])
def test_batch_fp64_matches_oracle_edge_systems(oracle, shape):
    # (8, 256) puts the 2- and 4-ion ex04 boxes on 8 CTAs: most own no ion
    psets, configs, pos = _as_batch(EDGE)
    res, _ = _run(psets, configs, pos, shape=shape)
    for k in range(len(EDGE)):
        o = _oracle_of(oracle, psets, configs[k], pos[k])
        compare(res[k], o, 1e-9)


def test_batch_fp64_matches_oracle_rocksalt(oracle):
    psets, configs, pos = systems.batch(nconf=10, seed=5, nmin=64, nmax=400,
                                        precision=_abi.PREC_FP64, cg_tol=1e-12)
    for p in psets:
        p.cg_max_iter = 2000
    res, _ = _run(psets, configs, pos)
    for k in range(len(configs)):
        o = _oracle_of(oracle, [_tight(p) for p in psets], configs[k], pos[k])
        compare(res[k], o, 1e-9)
        assert res[k]["converged"] == 1


@pytest.mark.parametrize("shape", [(1, 256), (2, 256), (4, 512), (8, 256), (8, 512)])
def test_batch_every_shape_same_result(shape):
    # includes boxes of fewer ions than 8 CTAs x 32 lanes and a 2-ion box
    psets, configs, pos = systems.batch(nconf=6, seed=11, nmin=64, nmax=300,
                                        precision=_abi.PREC_FP64, cg_tol=1e-12)
    psets[1].cg_max_iter = 2000
    ref, _ = _run(psets, configs, pos, shape=(1, 256))
    got, _ = _run(psets, configs, pos, shape=shape)
    for a, b in zip(got, ref):
        assert rel(forces(a), forces(b)) < 1e-11
        assert rel(a["mu"], b["mu"]) < 1e-10
        assert abs(a["u_coul"] - b["u_coul"]) <= 1e-11 * abs(b["u_coul"])


def test_batch_repeat_calls_bitwise():
    psets, configs, pos = systems.batch(nconf=5, seed=13, nmin=64, nmax=500)
    with BatchEngine(psets, configs) as eng:
        P = np.concatenate(pos)
        a = eng.engforce(P[:, 0], P[:, 1], P[:, 2])
        b = eng.engforce(P[:, 0], P[:, 1], P[:, 2])
    for k in ("fx", "fy", "fz", "mu", "ef"):
        assert np.array_equal(a[k], b[k]), k


def test_batch_mixed_error_vs_fp64():
    psets64, configs, pos = systems.batch(nconf=12, seed=17, nmin=64, nmax=1000,
                                          precision=_abi.PREC_FP64, cg_tol=1e-10)
    psetsmx, _, _ = systems.batch(nconf=12, seed=17, nmin=64, nmax=1000,
                                  precision=_abi.PREC_MIXED, cg_tol=1e-8)
    r64, _ = _run(psets64, configs, pos)
    rmx, _ = _run(psetsmx, configs, pos)
    for a, b in zip(rmx, r64):
        assert rms_rel(forces(a), forces(b)) <= 1e-5
        assert abs(a["u_coul"] - b["u_coul"]) <= 1e-6 * abs(b["u_coul"])
        if np.abs(b["mu"]).max() > 0:
            assert rms_rel(a["mu"], b["mu"]) <= 1e-5


def test_batch_matches_single_engine():
    psets, configs, pos = systems.batch(nconf=4, seed=19, nmin=200, nmax=600,
                                        precision=_abi.PREC_FP64, cg_tol=1e-11)
    res, _ = _run(psets, configs, pos)
    for k, conf in enumerate(configs):
        p = systems.config_params(psets, conf)
        with ForceEngine(p, conf[2]) as eng:
            g = eng.engforce(pos[k][:, 0], pos[k][:, 1], pos[k][:, 2])
        compare(res[k], g, 1e-9)


def test_batch_tune_picks_a_shape():
    psets, configs, pos = systems.batch(nconf=32, seed=23, nmin=64, nmax=1000)
    with BatchEngine(psets, configs) as eng:
        P = np.concatenate(pos)
        a = eng.engforce(P[:, 0], P[:, 1], P[:, 2])
        c, t, ms = eng.tune()
        assert c in (1, 2, 4, 8) and t in (256, 512) and ms > 0
        b = eng.engforce(P[:, 0], P[:, 1], P[:, 2])
        assert eng.info()["cluster"] == c
    assert rms_rel(forces(a), forces(b)) < 1e-6
