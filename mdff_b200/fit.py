"""Differentiable force-field fitting over the batched engine.

``EngForceFn`` is a ``torch.autograd.Function``: forward evaluates a batch of
configurations at parameter values ``theta`` (energies, forces, induced
dipoles); backward returns dJ/dtheta from the library's adjoint kernel
(mdff_gpu_batch_adjoint: one adjoint dipole solve per configuration), for any
upstream gradients of the three outputs.  A force-matching loss is then
plain torch:

    ff = BatchForceField(psets, configs, MGO_FIT)
    U, F, mu = EngForceFn.apply(theta, ff, pos)
    loss = ((F - F_target) ** 2).sum()
    loss.backward()          # theta.grad

No counterpart in the reference (it has no parameter derivatives); the
parameters and their units are those of its &non_bondedtag / &pimtag /
charge keywords (non_bonded.f90:135-150, pim.f90:258-279).
"""
import numpy as np

from . import _abi
from .engine import BatchEngine
from .params import params_copy

# the 10 parameters of the MgO fitting workload (types 0 = Mg, 1 = O):
# Buckingham A / rho / C of Mg-O and O-O, the O polarisability, the
# Tang-Toennies b / c of the Mg charge field on O dipoles, a charge scale
MGO_FIT = [
    (_abi.FIT_A, 0, 1), (_abi.FIT_RHO, 0, 1), (_abi.FIT_C, 0, 1),
    (_abi.FIT_A, 1, 1), (_abi.FIT_RHO, 1, 1), (_abi.FIT_C, 1, 1),
    (_abi.FIT_POL, 1, 0),
    (_abi.FIT_TTB, 1, 0), (_abi.FIT_TTC, 1, 0),
    (_abi.FIT_QSCALE, 0, 0),
]
NAMES = {_abi.FIT_A: "A", _abi.FIT_RHO: "rho", _abi.FIT_C: "C", _abi.FIT_POL: "alpha",
         _abi.FIT_TTB: "tt_b", _abi.FIT_TTC: "tt_c", _abi.FIT_QSCALE: "q_scale"}


def param_names(spec):
    return [f"{NAMES[k]}({a},{b})" if k != _abi.FIT_QSCALE else NAMES[k] for k, a, b in spec]


def apply_theta(p, spec, theta):
    """A copy of mdff_params p with the fit parameters set to theta (the host
    mirror of the library's fitted parameter sets; used to drive the oracle
    or the single-configuration engine at the same parameters)."""
    q = params_copy(p)
    for (k, a, b), v in zip(spec, theta):
        v = float(v)
        if k == _abi.FIT_A:
            q.Abmhftd[a][b] = q.Abmhftd[b][a] = v
        elif k == _abi.FIT_RHO:
            q.Bbmhftd[a][b] = q.Bbmhftd[b][a] = 1.0 / v
        elif k == _abi.FIT_C:
            q.Cbmhftd[a][b] = q.Cbmhftd[b][a] = v
        elif k == _abi.FIT_POL:
            for x in range(3):
                for y in range(3):
                    q.poldip[a][x][y] = v if x == y else 0.0
        elif k == _abi.FIT_TTB:
            q.pol_damp_b[a][a][b] = q.pol_damp_b[a][b][a] = v
        elif k == _abi.FIT_TTC:
            q.pol_damp_c[a][a][b] = q.pol_damp_c[a][b][a] = v
        elif k == _abi.FIT_QSCALE:
            for t in range(_abi.NT):
                q.qch[t] = p.qch[t] * v
    return q


class BatchForceField:
    """A BatchEngine with fit parameters declared; positions live on the GPU
    as a torch tensor (SoA [3, ntot], float64)."""

    def __init__(self, psets, configs, spec):
        self.engine = BatchEngine(psets, configs)
        self.spec = list(spec)
        self.theta0 = self.engine.fit_define(self.spec)
        self.nconf = self.engine.nconf
        self.ntot = self.engine.ntot
        self.buf = None

    def close(self):
        self.engine.close()


def _torch():
    import torch
    return torch


def _make_fn():
    torch = _torch()

    class EngForceFn(torch.autograd.Function):
        """(theta [nparam] float64, ff, pos [3, ntot] CUDA float64) ->
        U [nconf] (eV), F [ntot, 3] (eV/A), mu [ntot, 3] (induced + static
        dipoles, e A).  Backward: the adjoint kernel."""

        @staticmethod
        def forward(ctx, theta, ff, pos):
            dev = pos.device
            th = theta.detach().to("cpu", torch.float64).numpy()
            ff.engine.fit_set(th)
            pos = pos.contiguous()
            # persistent output buffers keep the evaluation's CUDA graph valid
            # between calls; the outputs handed out are copies
            if ff.buf is None or ff.buf[0].device != dev:
                ff.buf = (torch.empty((3, ff.ntot), dtype=torch.float64, device=dev),
                          torch.empty((ff.ntot, 3), dtype=torch.float64, device=dev))
            force, mu = ff.buf
            confs = ff.engine.engforce_device(pos.data_ptr(), force.data_ptr(), mu.data_ptr(), 0)
            U = torch.tensor([c["u_lj"] + c["u_bmhft"] + c["u_coul"] for c in confs],
                             dtype=torch.float64, device=dev)
            ctx.ff = ff
            ctx.dev = dev
            ctx.theta_dtype = theta.dtype
            return U, force.t().clone(), mu.clone()

        @staticmethod
        def backward(ctx, gU, gF, gmu):
            torch = _torch()
            ff, dev = ctx.ff, ctx.dev
            if gU is None:
                gU = torch.zeros(ff.nconf, dtype=torch.float64, device=dev)
            if gF is None:
                gF = torch.zeros((ff.ntot, 3), dtype=torch.float64, device=dev)
            gU = gU.to(dev, torch.float64).contiguous()
            gFs = gF.to(dev, torch.float64).t().contiguous()  # SoA [3, ntot]
            gm = None
            if gmu is not None:
                gm = gmu.to(dev, torch.float64).contiguous()
            torch.cuda.synchronize(dev)
            g = ff.engine.adjoint_device(gU.data_ptr(), gFs.data_ptr(),
                                         gm.data_ptr() if gm is not None else 0)
            return torch.tensor(g, dtype=ctx.theta_dtype), None, None

    return EngForceFn


_FN = None


def EngForceFn():
    """The autograd Function class (built on first use so that importing this
    module does not import torch)."""
    global _FN
    if _FN is None:
        _FN = _make_fn()
    return _FN


def fitting_workload(nconf=64, seed=2027, nmin=216, nmax=512, noise=0.05):
    """The fitting workload: nconf MgO-type boxes of nmin..nmax ions (batch()
    generator), FP64, and the perturbed parameters theta_true = theta0 * (1 +
    noise * N(0,1)) (seeded) at which the FP64 engine makes the target forces.
    Returns (psets, configs, positions, theta_true)."""
    from . import systems
    psets, configs, pos = systems.batch(nconf=nconf, seed=seed, nmin=nmin, nmax=nmax,
                                        kinds=("mgo",), precision=_abi.PREC_FP64, cg_tol=1e-11)
    for p in psets:
        p.cg_max_iter = 1000
    rng = np.random.default_rng(seed + 1)
    theta0 = np.array([fit_value(psets[1], k, a, b) for k, a, b in MGO_FIT])
    theta_true = theta0 * (1.0 + noise * rng.standard_normal(theta0.size))
    return psets, configs, pos, theta_true


def fit_value(p, k, a, b):
    """Current value of one fit parameter in mdff_params p."""
    if k == _abi.FIT_A:
        return p.Abmhftd[a][b]
    if k == _abi.FIT_RHO:
        return 1.0 / p.Bbmhftd[a][b]
    if k == _abi.FIT_C:
        return p.Cbmhftd[a][b]
    if k == _abi.FIT_POL:
        return p.poldip[a][0][0]
    if k == _abi.FIT_TTB:
        return p.pol_damp_b[a][b][a]
    if k == _abi.FIT_TTC:
        return p.pol_damp_c[a][b][a]
    return 1.0
