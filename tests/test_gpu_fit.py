"""Force-field gradients of the batched engine (mdff_gpu_batch_adjoint behind
mdff_b200.fit.EngForceFn) against central finite differences.

For the 10 MgO fit parameters (Buckingham A / rho / C of Mg-O and O-O, O
polarisability, Tang-Toennies b / c, charge scale) the adjoint gradient of
(a) the total energy, (b) a force-matching loss against forces made at
perturbed parameters and (c) a random linear function of the dipoles must
match central differences of the same FP64 engine (h = 1e-5 relative) to
1e-6, each parameter's error measured as |theta_k (g_k - fd_k)| against the
largest |theta_j fd_j| (the parameters carry different units).  (d) The
same gradient against central differences of the CPU oracle (the
reference's algorithm), h = 1e-4, to 1e-5."""
import numpy as np
import pytest

from mdff_b200 import _abi, fit, systems

from .gpu_util import forces

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _workload(nconf=3, nmin=64, nmax=216, seed=31, tol=1e-13):
    psets, configs, pos, theta_true = fit.fitting_workload(nconf=nconf, seed=seed, nmin=nmin,
                                                           nmax=nmax)
    for p in psets:
        p.cg_tol = tol
        p.conv_tol_ind = tol
        p.cg_max_iter = 3000
    return psets, configs, pos, theta_true


def _scaled_err(theta, g, fd):
    sc = np.maximum(np.abs(theta), 1.0)
    den = np.abs(sc * fd).max()
    return np.abs(sc * (g - fd)) / den


def _fd(fun, theta, rel=1e-5):
    out = np.zeros(theta.size)
    for k in range(theta.size):
        h = rel * max(abs(theta[k]), 1.0)
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        out[k] = (fun(tp) - fun(tm)) / (2 * h)
    return out


class _Setup:
    def __init__(self, **kw):
        self.psets, self.configs, pos, self.theta_true = _workload(**kw)
        self.ff = fit.BatchForceField(self.psets, self.configs, fit.MGO_FIT)
        P = np.concatenate(pos)
        self.P = P
        self.pos = torch.tensor(np.ascontiguousarray(P.T), dtype=torch.float64, device="cuda")
        self.theta0 = self.ff.theta0.copy()
        self.Fn = fit.EngForceFn()

    def run(self, theta):
        th = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
        U, F, mu = self.Fn.apply(th, self.ff, self.pos)
        return th, U, F, mu


@pytest.fixture(scope="module")
def S():
    s = _Setup()
    yield s
    s.ff.close()


def test_theta0_matches_the_parameter_set(S):
    p = S.psets[1]
    assert S.theta0[0] == pytest.approx(p.Abmhftd[0][1])
    assert S.theta0[1] == pytest.approx(1.0 / p.Bbmhftd[0][1])
    assert S.theta0[6] == pytest.approx(p.poldip[1][0][0])
    assert S.theta0[7] == pytest.approx(p.pol_damp_b[1][0][1])
    assert S.theta0[9] == 1.0


def test_energy_gradient_vs_fd(S):
    th, U, F, mu = S.run(S.theta0)
    U.sum().backward()
    g = th.grad.numpy().copy()

    def energy(t):
        with torch.no_grad():
            return float(S.run(t)[1].sum())

    fd = _fd(energy, S.theta0)
    err = _scaled_err(S.theta0, g, fd)
    assert err.max() <= 1e-6, dict(zip(fit.param_names(fit.MGO_FIT), err))


def test_force_matching_gradient_vs_fd(S):
    with torch.no_grad():
        Ft = S.run(S.theta_true)[2].clone()

    def loss_of(t):
        with torch.no_grad():
            F = S.run(t)[2]
            return float(((F - Ft) ** 2).sum())

    th, U, F, mu = S.run(S.theta0)
    loss = ((F - Ft) ** 2).sum()
    loss.backward()
    g = th.grad.numpy().copy()
    fd = _fd(loss_of, S.theta0)
    err = _scaled_err(S.theta0, g, fd)
    assert err.max() <= 1e-6, dict(zip(fit.param_names(fit.MGO_FIT), err))
    assert float(loss.detach()) > 0


def test_dipole_and_mixed_cotangents_vs_fd(S):
    rng = np.random.default_rng(5)
    wmu = torch.tensor(rng.standard_normal((S.ff.ntot, 3)), device="cuda")
    wU = torch.tensor(rng.standard_normal(S.ff.nconf), device="cuda")
    wF = torch.tensor(rng.standard_normal((S.ff.ntot, 3)), device="cuda")

    def J_of(U, F, mu):
        return (wmu * mu).sum() + 1e-3 * (wU * U).sum() + (wF * F).sum()

    def j(t):
        with torch.no_grad():
            return float(J_of(*S.run(t)[1:]))

    th, U, F, mu = S.run(S.theta0)
    J_of(U, F, mu).backward()
    g = th.grad.numpy().copy()
    fd = _fd(j, S.theta0)
    err = _scaled_err(S.theta0, g, fd)
    assert err.max() <= 1e-6, dict(zip(fit.param_names(fit.MGO_FIT), err))


def test_gradient_vs_oracle_fd(oracle):
    # one small box: finite differences of the CPU oracle (SCF to 1e-13)
    psets, configs, pos, theta_true = _workload(nconf=1, nmin=64, nmax=64, seed=41)
    ff = fit.BatchForceField(psets, configs, fit.MGO_FIT)
    theta0 = ff.theta0.copy()
    P = pos[0]
    rng = np.random.default_rng(9)
    wF = rng.standard_normal(P.shape)
    base = systems.config_params(psets, configs[0])
    base.solver = _abi.SOLVER_SCF
    base.max_scf_pol_iter = 5000

    def j_oracle(t):
        p = fit.apply_theta(base, fit.MGO_FIT, t)
        r = oracle.Oracle(p, configs[0][2]).engforce(P[:, 0], P[:, 1], P[:, 2])
        return float((forces(r) * wF).sum() + 1e-3 * (r["u_bmhft"] + r["u_coul"]))

    eng = ff.engine
    eng.engforce(P[:, 0], P[:, 1], P[:, 2])
    g = eng.adjoint(np.array([1e-3]), wF)
    fd = _fd(j_oracle, theta0, rel=1e-4)
    err = _scaled_err(theta0, g, fd)
    ff.close()
    assert err.max() <= 1e-5, dict(zip(fit.param_names(fit.MGO_FIT), err))
