"""Seeded synthetic ionic systems (inputs for parity tests and the benchmark).

All systems are built here from published force-field parameters and
``numpy.random.default_rng(seed)``; no dataset is read.  Ions are grouped by
type in POSFF order (read_pos.f90:187-199).  Units are the reference's
internal units: Angstrom, eV, amu, charge e, time unit = A*sqrt(amu/eV)
(constants.f90:88-94).
"""
import dataclasses
import math

import numpy as np

from . import _abi
from .params import make_params

TIME_UNIT = 98.2269514139276      # ps -> internal time (constants.f90:90)
# ASPC order of the polarisable MD workloads: the order the reference's own
# MD decks use (examples/ex12/config/mdff/control_md.F:53,
# examples/ex14/config/control_md_full_run_pim.F:46)
ASPC_ORDER_MD = 4
BOLTZ_UNIT = 8.61734229648141e-05  # eV/K (constants.f90:89)
RHO_UNIT = 1.660538782             # g/cm3 -> amu/A^3 (constants.f90:93)
J_TO_EV = 1.0 / 1.602176487e-19    # constants.f90:76 evtoj


@dataclasses.dataclass
class System:
    name: str
    params: object            # _abi.MdffParams
    cell: np.ndarray          # A (3,3), columns = lattice vectors
    pos: np.ndarray           # (N,3) Cartesian
    mass: np.ndarray          # (N,) amu
    vel: np.ndarray           # (N,3) internal units
    info: dict

    @property
    def natm(self):
        return self.pos.shape[0]

    def soa(self):
        return tuple(np.ascontiguousarray(self.pos[:, a]) for a in range(3))


def box_length(n_formula, formula_mass, density_gcc):
    """Cubic box edge for n_formula units at a mass density (g/cm^3)."""
    vol = n_formula * formula_mass / (density_gcc / RHO_UNIT)
    return vol ** (1.0 / 3.0)


def ewald_kmax(alpha, rcut, epsw, anorm):
    """kmax of the DL_POLY-like rule of ewald_param (coulomb.f90:386-393)
    evaluated at a given alpha (used to state kmax for a chosen alpha)."""
    eps = min(abs(epsw), 0.5)
    tol = math.sqrt(abs(math.log(eps * rcut)))
    tol1 = math.sqrt(-math.log(eps * rcut * (2.0 * tol * alpha) ** 2))
    return int(math.floor(0.25 + anorm * alpha * tol1 / math.pi + 0.5))


def maxwell(rng, mass, temp):
    """Maxwell-Boltzmann velocities (internal units), zero total momentum."""
    sig = np.sqrt(BOLTZ_UNIT * temp / mass)[:, None]
    v = rng.standard_normal((mass.size, 3)) * sig
    p = (v * mass[:, None]).sum(0) / mass.sum()
    return v - p[None, :]


def rocksalt(ncell, a):
    """Cation and anion sites of ncell^3 conventional rock-salt cells."""
    base_c = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    base_a = base_c + np.array([0.5, 0, 0])
    g = np.stack(np.meshgrid(*[np.arange(ncell)] * 3, indexing="ij"), -1).reshape(-1, 3)
    cat = (g[:, None, :] + base_c[None]).reshape(-1, 3) * a
    ani = (g[:, None, :] + base_a[None]).reshape(-1, 3) * a
    return cat, ani


# --------------------------------------------------------------------------
# published parameters

def tosi_fumi_nacl():
    """Tosi-Fumi NaCl (J. Phys. Chem. Solids 25, 45 (1964)) in the BMH form
    A exp(-B r) - C/r^6 - D/r^8 of non_bonded.f90:107-116.
    b = 0.338e-19 J, rho = 0.317 A, sigma_Na = 1.170 A, sigma_Cl = 1.585 A,
    Pauling c_{++,+-,--} = 1.25, 1.00, 0.75, C in 1e-79 J m^6, D in 1e-99 J m^8."""
    b = 0.338e-19 * J_TO_EV
    rho = 0.317
    sig = (1.170, 1.585)
    cpa = {(0, 0): 1.25, (0, 1): 1.0, (1, 1): 0.75}
    C = {(0, 0): 1.68, (0, 1): 11.2, (1, 1): 116.0}
    D = {(0, 0): 0.8, (0, 1): 13.9, (1, 1): 233.0}
    conv = 1e-19 * J_TO_EV  # 1e-79 J m^6 = 1e-19 J A^6 ; same for 1e-99 J m^8
    A, Bt, Ct, Dt = {}, {}, {}, {}
    for (i, j), cij in cpa.items():
        A[(i, j)] = cij * b * math.exp((sig[i] + sig[j]) / rho)
        Bt[(i, j)] = 1.0 / rho
        Ct[(i, j)] = C[(i, j)] * conv
        Dt[(i, j)] = D[(i, j)] * conv
    return A, Bt, Ct, Dt


def lewis_catlow_mgo():
    """Buckingham MgO (Lewis & Catlow, J. Phys. C 18, 1149 (1985)): Mg-O
    A = 1428.5 eV, rho = 0.2945 A; O-O A = 22764 eV, rho = 0.149 A,
    C = 27.88 eV A^6.  Types: 0 = Mg, 1 = O."""
    A = {(0, 1): 1428.5, (1, 1): 22764.0}
    B = {(0, 1): 1.0 / 0.2945, (1, 1): 1.0 / 0.149}
    C = {(0, 1): 0.0, (1, 1): 27.88}
    return A, B, C


def bks_sio2():
    """BKS silica (van Beest, Kramer, van Santen, PRL 64, 1955 (1990)):
    Si-O A = 18003.7572 eV, b = 4.87318 1/A, C = 133.5381 eV A^6;
    O-O A = 1388.7730 eV, b = 2.76000 1/A, C = 175.0000 eV A^6.
    Types: 0 = Si, 1 = O."""
    A = {(0, 1): 18003.7572, (1, 1): 1388.7730}
    B = {(0, 1): 4.87318, (1, 1): 2.76000}
    C = {(0, 1): 133.5381, (1, 1): 175.0000}
    return A, B, C


# --------------------------------------------------------------------------
# the reference's ex04 decks (examples/ex04/POSFF.*, control_*.F)

def ex04(tag):
    """Nymand-Linse test systems in reduced units (examples/ex04/run_ex4.sh):
    10x10x10 box, alpha = 0.8, kmax = 11, rc = 5."""
    cell = np.eye(3) * 10.0
    common = dict(lcoulomb=1, lreduced=1, cutlongrange=5.0, cutshortrange=0.0,
                  alphaES=0.8, kES=(11, 11, 11), calc=_abi.CALC_OTHER)
    if tag == "twocharges":
        p = make_params([1, 1], qch=[1.0, -1.0], **common)
        pos = np.array([[-0.5, 0, 0], [0.5, 0, 0]], dtype=np.float64)
    elif tag == "twodipoles":
        p = make_params([1, 1], dip={(0, 0): 1.0, (1, 0): 1.0}, **common)
        pos = np.array([[-0.5, 0, 0], [0.5, 0, 0]], dtype=np.float64)
    elif tag == "twocharges_twopola":
        pol = np.zeros((4, 3, 3))
        pol[2, 0, 0] = 0.1
        pol[3] = np.eye(3) * 0.1
        p = make_params([1, 1, 1, 1], qch=[1.0, -1.0, 0.0, 0.0], lsurf=1,
                        ldip_polar=[0, 0, 1, 1], poldip=pol, conv_tol_ind=1e-12,
                        min_scf_pol_iter=3, max_scf_pol_iter=500, **common)
        pos = np.array([[-0.5, 0, 0], [0.5, 0, 0], [-0.5, 1, 0], [0.5, 1, 1]],
                       dtype=np.float64)
    else:
        raise KeyError(tag)
    n = pos.shape[0]
    return System("ex04_" + tag, p, cell, pos, np.ones(n), np.zeros((n, 3)), {})


# --------------------------------------------------------------------------
# benchmark systems

def nacl(ncell=6, seed=1234, density=1.55, jitter=0.3, temp=1200.0, rcut=12.0,
         alpha=0.3, kmax=10, skin=1.0, **extra):
    """Molten NaCl: rock-salt ncell^3 conventional cells, Tosi-Fumi BMH +
    Ewald; Na +1 then Cl -1."""
    rng = np.random.default_rng(seed)
    nf = 4 * ncell ** 3
    L = box_length(nf, 22.98977 + 35.453, density)
    cat, ani = rocksalt(ncell, L / ncell)
    pos = np.concatenate([cat, ani]) + rng.uniform(-jitter, jitter, (2 * nf, 3))
    A, B, C, D = tosi_fumi_nacl()
    rc = min(rcut, 0.5 * L)
    kw = dict(lcoulomb=1, lbmhft=1, cutshortrange=rc, cutlongrange=rc, skindiff=skin,
              qch=[1.0, -1.0], Abmhftd=A, Bbmhftd=B, Cbmhftd=C, Dbmhftd=D,
              alphaES=alpha, kES=(kmax,) * 3)
    kw.update(extra)
    p = make_params([nf, nf], **kw)
    mass = np.concatenate([np.full(nf, 22.98977), np.full(nf, 35.453)])
    vel = maxwell(rng, mass, temp)
    return System(f"nacl{2 * nf}", p, np.eye(3) * L, pos, mass, vel,
                  dict(L=L, seed=seed, density=density))


def mgo(ncell=10, seed=4321, density=3.58, jitter=0.2, temp=2000.0, rcut=10.0,
        alpha=0.35, epsw=1e-7, skin=1.0, kmax=None, **extra):
    """Polarisable MgO: Lewis-Catlow Buckingham, O polarisability 1.6 A^3,
    Tang-Toennies damping (b = 3.0 1/A, c = 1.0, order 4) of the Mg charge ->
    O dipole field (ldip_damping(O, Mg, O): the reference symmetrises the
    last two indices from the upper triangle, pim.f90:189-199, so the entry
    is given with the lower type index second, like ldip_damping(1,1,2) in
    examples/ex09/config/pot_mdff/PIMD.POT); Ewald alpha 0.35 with kmax from the ewald_param rule at
    epsw.  Types: 0 = Mg (+2), 1 = O (-2)."""
    rng = np.random.default_rng(seed)
    nf = 4 * ncell ** 3
    L = box_length(nf, 24.305 + 15.9994, density)
    cat, ani = rocksalt(ncell, L / ncell)
    pos = np.concatenate([cat, ani]) + rng.uniform(-jitter, jitter, (2 * nf, 3))
    A, B, C = lewis_catlow_mgo()
    rc = min(rcut, 0.5 * L)
    if kmax is None:
        kmax = ewald_kmax(alpha, rc, epsw, L)
    kw = dict(lcoulomb=1, lbmhft=1, cutshortrange=rc, cutlongrange=rc, skindiff=skin,
              qch=[2.0, -2.0], Abmhftd=A, Bbmhftd=B, Cbmhftd=C,
              alphaES=alpha, kES=(kmax,) * 3, epsw=epsw,
              ldip_polar=[0, 1], poldip_iso={1: 1.6},
              ldip_damping={(1, 0, 1): 1}, pol_damp_b={(1, 0, 1): 3.0},
              pol_damp_c={(1, 0, 1): 1.0}, pol_damp_k={(1, 0, 1): 4},
              conv_tol_ind=1e-8, extrapolate_order=ASPC_ORDER_MD)
    kw.update(extra)
    p = make_params([nf, nf], **kw)
    mass = np.concatenate([np.full(nf, 24.305), np.full(nf, 15.9994)])
    vel = maxwell(rng, mass, temp)
    return System(f"mgo{2 * nf}", p, np.eye(3) * L, pos, mass, vel,
                  dict(L=L, seed=seed, kmax=kmax, epsw=epsw))


def rsi(rng, n_per_type, L, dmin):
    """Random sequential insertion in a periodic cubic box with per-type-pair
    minimum separations dmin[ti][tj]; types inserted in order."""
    dmax = max(max(r) for r in dmin)
    nc = max(1, int(L // dmax))
    w = L / nc
    cells = {}
    pos, typ = [], []
    for t, n in enumerate(n_per_type):
        placed, tries = 0, 0
        while placed < n:
            tries += 1
            if tries > 2000 * n:
                raise RuntimeError("random sequential insertion jammed")
            x = rng.uniform(0, L, 3)
            c = tuple((x // w).astype(int) % nc)
            ok = True
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        key = ((c[0] + dx) % nc, (c[1] + dy) % nc, (c[2] + dz) % nc)
                        for j in cells.get(key, ()):
                            d = x - pos[j]
                            d -= L * np.round(d / L)
                            if d @ d < dmin[t][typ[j]] ** 2:
                                ok = False
                                break
                        if not ok:
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                cells.setdefault(c, []).append(len(pos))
                pos.append(x)
                typ.append(t)
                placed += 1
    return np.array(pos)


def sio2(nsio2=4000, seed=2024, density=2.2, temp=300.0, rcut=10.0, alpha=0.3, kmax=12,
         skin=1.0, dmin_sio=1.4, dmin_oo=2.2, dmin_sisi=2.5, place=True, **extra):
    """SiO2-like glass: 3*nsio2 ions (Si +2.4 then O -1.2) by seeded random
    sequential insertion; BKS Buckingham plus a (sigma/r)^24 eV wall on every
    pair (sigma Si-O 1.2, O-O 1.9, Si-Si 2.4 A: BKS alone has an unphysical
    Si-O well below 1.2 A and no Si-Si repulsion, and O-O pairs must stay out of
    the dipole catastrophe radius); O polarisability 1.3 A^3 with Tang-Toennies damping
    of the fields on O (b, c, order from examples/ex09/config/pot_mdff/PIMD.POT:
    O-O 5.584/2.890/4, O-Si 3.664/1.446/4); Ewald alpha 0.3, kmax 12, rc 10.
    Minimum separations: Si-O 1.4 A; O-O and Si-Si larger (2.2 / 2.5 A) so no
    O-O pair starts inside the undamped dipole-dipole catastrophe radius
    (2*alpha_O)^(1/3) = 1.375 A."""
    rng = np.random.default_rng(seed)
    L = box_length(nsio2, 28.0855 + 2 * 15.9994, density)
    dmin = [[dmin_sisi, dmin_sio], [dmin_sio, dmin_oo]]
    # place=False skips the insertion (positions then come from a prepared state)
    pos = rsi(rng, [nsio2, 2 * nsio2], L, dmin) if place else np.zeros((3 * nsio2, 3))
    A, B, C = bks_sio2()
    rc = min(rcut, 0.5 * L)
    kw = dict(lcoulomb=1, lbmhft=1, cutshortrange=rc, cutlongrange=rc, skindiff=skin,
              qch=[2.4, -1.2], Abmhftd=A, Bbmhftd=B, Cbmhftd=C,
              wall24={(0, 1): 1.2 ** 24, (1, 1): 1.9 ** 24, (0, 0): 2.4 ** 24},
              alphaES=alpha, kES=(kmax,) * 3,
              ldip_polar=[0, 1], poldip_iso={1: 1.3},
              ldip_damping={(1, 1, 1): 1, (1, 0, 1): 1},
              pol_damp_b={(1, 1, 1): 5.58406251008641721012, (1, 0, 1): 3.66418041600447487325},
              pol_damp_c={(1, 1, 1): 2.8904937083, (1, 0, 1): 1.4460000000},
              pol_damp_k={(1, 1, 1): 4, (1, 0, 1): 4},
              conv_tol_ind=1e-8, extrapolate_order=ASPC_ORDER_MD)
    kw.update(extra)
    p = make_params([nsio2, 2 * nsio2], **kw)
    mass = np.concatenate([np.full(nsio2, 28.0855), np.full(2 * nsio2, 15.9994)])
    vel = maxwell(rng, mass, temp)
    return System(f"sio2_{3 * nsio2}", p, np.eye(3) * L, pos, mass, vel,
                  dict(L=L, seed=seed))


def random_ionic(n_per_type=(20, 20), L=14.0, seed=7, q=(1.5, -1.5), pol=(0.0, 1.1),
                 triclinic=False, **extra):
    """Small seeded test box (rock-salt-free): random positions with a 1.6 A
    minimum separation, optional triclinic cell (sheared cube); exercises every term."""
    rng = np.random.default_rng(seed)
    nt = len(n_per_type)
    dmin = [[1.9] * nt for _ in range(nt)]
    pos = rsi(rng, list(n_per_type), L, dmin)
    cell = np.eye(3) * L
    if triclinic:
        cell = np.array([[L, 0.15 * L, 0.1 * L], [0.0, 0.95 * L, -0.08 * L], [0.0, 0.0, 1.05 * L]])
        frac = pos / L
        pos = frac @ cell.T
    rc = min(6.0, 0.45 * L)
    kw = dict(lcoulomb=1, lbmhft=1, cutshortrange=rc, cutlongrange=rc, skindiff=0.7,
              qch=list(q), Abmhftd={(0, 1): 1500.0, (1, 1): 900.0, (0, 0): 300.0},
              Bbmhftd={(0, 1): 3.3, (1, 1): 3.0, (0, 0): 3.5},
              Cbmhftd={(0, 1): 5.0, (1, 1): 20.0, (0, 0): 1.0},
              alphaES=0.45, kES=(7, 7, 7),
              ldip_polar=[1 if a > 0 else 0 for a in pol],
              poldip_iso={i: a for i, a in enumerate(pol) if a > 0},
              conv_tol_ind=1e-11, max_scf_pol_iter=300)
    kw.update(extra)
    p = make_params(list(n_per_type), **kw)
    n = pos.shape[0]
    mass = np.full(n, 20.0)
    vel = maxwell(rng, mass, 1000.0)
    return System("random_ionic", p, cell, pos, mass, vel, dict(L=L, seed=seed))


def wannier_box(n_pairs=16, L=9.0, seed=31, nwfc=4, d_wfc=0.35, pol_cation=0.5, **extra):
    """Seeded box with Wannier centres (pim.f90:93-96): n_pairs cations M (+2,
    polarisable, lwfc 0) and anions O (+6, lwfc = nwfc), each O carrying nwfc
    centres W (-2, lwfc -1) at d_wfc A along tetrahedral directions jittered
    by 0.05 A; types in the order M, O, W (centres last)."""
    rng = np.random.default_rng(seed)
    base = rsi(rng, [n_pairs, n_pairs], L, [[2.4, 2.2], [2.2, 2.6]])
    tet = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], dtype=np.float64) / np.sqrt(3.0)
    w = []
    for o in base[n_pairs:]:
        for k in range(nwfc):
            v = tet[k % 4] * d_wfc + rng.uniform(-0.05, 0.05, 3)
            w.append(o + v)
    pos = np.concatenate([base, np.array(w)]) % L
    cell = np.eye(3) * L
    rc = 0.45 * L
    kw = dict(lcoulomb=1, cutlongrange=rc, skindiff=0.5, qch=[2.0, 6.0, -2.0], alphaES=0.6,
              kES=(8, 8, 8), ldip_polar=[1, 0, 0], poldip_iso={0: pol_cation},
              lwfc=[0, nwfc, -1], conv_tol_ind=1e-11, max_scf_pol_iter=300)
    kw.update(extra)
    p = make_params([n_pairs, n_pairs, n_pairs * nwfc], **kw)
    n = pos.shape[0]
    mass = np.full(n, 20.0)
    vel = np.zeros((n, 3))
    return System("wannier_box", p, cell, pos, mass, vel, dict(L=L, seed=seed))


# --------------------------------------------------------------------------
# batched workloads: many small independent boxes

FORMULA = {"nacl": (22.98977 + 35.453, 1.55), "mgo": (24.305 + 15.9994, 3.58)}


def batch_psets(precision=_abi.PREC_MIXED, cg_tol=1e-8, epsw=1e-6, cg_max_iter=200):
    """Parameter sets of the batched workloads.  0 = NaCl type: Tosi-Fumi BMH,
    charges +1/-1, no polarisation.  1 = MgO type: Lewis-Catlow Buckingham,
    charges +2/-2, O polarisability 1.6 A^3 with Tang-Toennies damping
    (b 3.0, c 1.0, order 4) of the Mg charge field on O, as mgo().  Ewald
    alpha and kmax per box from the ewald_param rule (lautoES, coulomb.f90:
    363-410) at epsw; the real-space cutoff is clamped to half of each box.
    Short-range cutoffs 6 A (NaCl) and 4 A (MgO) fit the smallest boxes."""
    A, B, C, D = tosi_fumi_nacl()
    common = dict(lcoulomb=1, lbmhft=1, cutlongrange=12.0, lautoES=1, epsw=epsw,
                  precision=precision, solver=_abi.SOLVER_CG, cg_tol=cg_tol,
                  cg_max_iter=cg_max_iter, conv_tol_ind=cg_tol, calc=_abi.CALC_OTHER)
    nacl = make_params([1, 1], cutshortrange=6.0, qch=[1.0, -1.0], Abmhftd=A, Bbmhftd=B,
                       Cbmhftd=C, Dbmhftd=D, **common)
    Am, Bm, Cm = lewis_catlow_mgo()
    mgo_p = make_params([1, 1], cutshortrange=4.0, qch=[2.0, -2.0], Abmhftd=Am, Bbmhftd=Bm,
                        Cbmhftd=Cm, ldip_polar=[0, 1], poldip_iso={1: 1.6},
                        ldip_damping={(1, 0, 1): 1}, pol_damp_b={(1, 0, 1): 3.0},
                        pol_damp_c={(1, 0, 1): 1.0}, pol_damp_k={(1, 0, 1): 4}, **common)
    return [nacl, mgo_p]


# minimum separations enforced on the jittered MgO-type boxes (cation-anion,
# anion-anion, cation-cation; A): with the O polarisability 1.6 A^3 the
# undamped dipole-dipole coupling of O-O pairs below ~1.9 A, or a Mg charge
# within ~1.3 A of an O, drives the reference's SCF into the polarisation
# catastrophe (moment_from_pola.f90:176-216)
DMIN = {"nacl": None, "mgo": (1.5, 2.0, 2.0)}


def rocksalt_box(rng, n_ions, kind, density, jitter):
    """n_ions (even) of a rock-salt compound in a cubic box: the smallest m^3
    conventional-cell lattice with room for n_ions/2 cations and anions, its
    lattice constant that of the full crystal at the given mass density, sites
    drawn without replacement (equal numbers of vacancies on both
    sublattices, so the ion density is the lattice's times the filled
    fraction), positions jittered by U(-jitter, jitter) per component.  Where
    DMIN gives minimum separations, an ion's jitter is redrawn (up to 200
    times) until it keeps them to every ion placed before it.  Cations first,
    then anions.  Returns (positions, box edge)."""
    nf = n_ions // 2
    fmass = FORMULA[kind][0]
    m = 1
    while 4 * m ** 3 < nf:
        m += 1
    L = m * box_length(4, fmass, density)
    cat, ani = rocksalt(m, L / m)
    ci = np.sort(rng.choice(len(cat), nf, replace=False))
    ai = np.sort(rng.choice(len(ani), nf, replace=False))
    sites = np.concatenate([cat[ci], ani[ai]])
    dmin = DMIN[kind]
    if dmin is None:
        return sites + rng.uniform(-jitter, jitter, (2 * nf, 3)), L
    pos = np.zeros_like(sites)
    anion = np.arange(2 * nf) >= nf
    for i in range(2 * nf):
        for _ in range(200):
            x = sites[i] + rng.uniform(-jitter, jitter, 3)
            if i == 0:
                break
            d = pos[:i] - x
            d -= L * np.round(d / L)
            r = np.sqrt((d * d).sum(1))
            lim = np.where(anion[:i] != anion[i], dmin[0], dmin[1] if anion[i] else dmin[2])
            if (r >= lim).all():
                break
        else:
            raise RuntimeError("rocksalt_box: jitter rejection failed")
        pos[i] = x
    return pos, L


def batch(nconf=256, seed=99, nmin=64, nmax=1000, jitter=0.3, density_spread=0.1,
          kinds=("nacl", "mgo"), precision=_abi.PREC_MIXED, cg_tol=1e-8, epsw=1e-6):
    """Seeded batch of independent cubic rock-salt boxes: per box a kind
    (uniform over kinds), an even ion count uniform in [nmin, nmax], a lattice
    density uniform within +-density_spread of the kind's nominal (NaCl 1.55,
    MgO 3.58 g/cm^3; vacancies fill the lattice up, rocksalt_box) and +-jitter
    positions.  Returns (psets, configs, positions):
    configs[c] = (pset index, [n_cation, n_anion], cell), positions a list of
    (n_c, 3) arrays in the configuration order."""
    rng = np.random.default_rng(seed)
    psets = batch_psets(precision=precision, cg_tol=cg_tol, epsw=epsw)
    index = {"nacl": 0, "mgo": 1}
    configs, pos = [], []
    for _ in range(nconf):
        kind = kinds[int(rng.integers(len(kinds)))]
        n = 2 * int(rng.integers(nmin // 2, nmax // 2 + 1))
        dens = FORMULA[kind][1] * rng.uniform(1 - density_spread, 1 + density_spread)
        p, L = rocksalt_box(rng, n, kind, dens, jitter)
        configs.append((index[kind], [n // 2, n // 2], np.eye(3) * L))
        pos.append(p)
    return psets, configs, pos


def config_params(psets, conf):
    """The single-configuration parameters of one batch entry (for the
    single engine or the oracle)."""
    from .params import params_copy
    p = params_copy(psets[conf[0]])
    for t in range(_abi.NT):
        p.natmi[t] = conf[1][t] if t < len(conf[1]) else 0
    p.natm = int(sum(conf[1]))
    return p
