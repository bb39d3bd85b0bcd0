"""The reference's input formats: POSFF configurations and control files of
Fortran namelists, so that the engine runs the reference's own decks and
writes decks the reference binary reads.

* POSFF (read_pos.f90:36-158): natm, system name, the three lattice vectors
  (one per line; columns of simu_cell%A), ntype, type names, ions per type,
  'Direct'/'D' or 'Cartesian'/'C', then one line per ion: type name and
  position (+ velocity (+ force) for posff_data 'rvn' / 'rvf').  Positions are
  wrapped as the reader does: kardir, periodicbc (s - NINT(s)), dirkar
  (read_pos.f90:148-150, lattice.f90:276-295).
* Control files: namelist groups &controltag, &fieldtag, &non_bondedtag,
  &coulombtag, &pimtag, &mdtag, ... (control.f90:128-161, field.f90:126-130,
  non_bonded.f90:135-150, coulomb.f90:97-106, pim.f90:258-279), with the
  reference's defaults (the *_default_tag routines).  '!INCLUDE <file>' lines
  are replaced by the file, as the examples' deck generator does
  (examples/ex09/config/gen_tests, include()).
* Outputs: CONTFF (config.f90:208-252: the POSFF header with fixed formats,
  positions wrapped, then type, position, velocity, force per ion), DIPFF
  (field.f90:300-337: list-directed header, then ion number, type and the
  three dipole components) and EFGALL (field.f90:392-448, formatted variant:
  the six independent components vxx vyy vzz vxy vxz vyz per ion).  Fixed
  formats (i8, 3f20.12, e24.16, ...) are written as Fortran writes them;
  list-directed lines follow gfortran's layout (their widths differ between
  compilers; the readers here and the reference's parse them by blanks).
"""
import os
import re

import numpy as np

from . import _abi
from .params import make_params

# ---------------------------------------------------------------------------
# POSFF


def read_posff(path, posff_data="rnn"):
    """Returns dict(natm, system, cell (3x3, columns = lattice vectors), ntype,
    names, natmi, pos (natm, 3) Cartesian, wrapped), plus vel / force for
    posff_data 'rvn' / 'rvf'."""
    with open(path) as f:
        lines = [ln for ln in f.read().splitlines()]
    k = 0

    def nxt():
        nonlocal k
        while k < len(lines) and not lines[k].strip():
            k += 1
        ln = lines[k]
        k += 1
        return ln.split()

    natm = int(nxt()[0])
    system = " ".join(nxt())
    cols = [[float(x.replace("d", "e").replace("D", "e")) for x in nxt()[:3]] for _ in range(3)]
    A = np.array(cols).T  # A(:, j) = lattice vector j
    ntype = int(nxt()[0])
    names = nxt()[:ntype]
    natmi = [int(x) for x in nxt()[:ntype]]
    cpos = nxt()[0]
    if cpos not in ("Direct", "D", "Cartesian", "C"):
        raise ValueError(f"POSFF coordinate tag {cpos!r} (read_pos.f90:80)")
    ncol = {"rnn": 3, "rvn": 6, "rvf": 9}[posff_data]
    typ, data = [], []
    for _ in range(natm):
        t = nxt()
        typ.append(t[0])
        data.append([float(x.replace("d", "e").replace("D", "e")) for x in t[1:1 + ncol]])
    data = np.array(data, dtype=np.float64)
    pos = data[:, :3].copy()
    if cpos in ("Direct", "D"):
        pos = pos @ A.T
    B = np.linalg.inv(A)
    s = pos @ B.T
    s = s - np.where(s >= 0, np.floor(s + 0.5), np.ceil(s - 0.5))  # Fortran NINT
    pos = s @ A.T
    out = dict(natm=natm, system=system, cell=A, ntype=ntype, names=names, natmi=natmi,
               pos=pos, types=typ)
    if ncol >= 6:
        out["vel"] = data[:, 3:6].copy()
    if ncol == 9:
        out["force"] = data[:, 6:9].copy()
    return out


def write_posff(path, system, cell, names, natmi, pos, vel=None, force=None):
    """POSFF in Cartesian coordinates (ions grouped by type in names order)."""
    A = np.asarray(cell, dtype=np.float64)
    pos = np.asarray(pos, dtype=np.float64)
    natm = pos.shape[0]
    typ = np.repeat(np.arange(len(names)), natmi)
    with open(path, "w") as f:
        f.write(f"{natm}\n{system}\n")
        for j in range(3):
            f.write(" ".join(f"{A[a, j]:20.12f}" for a in range(3)) + "\n")
        f.write(f"{len(names)}\n{' '.join(names)}\n{' '.join(str(n) for n in natmi)}\nCartesian\n")
        for i in range(natm):
            cols = list(pos[i])
            if vel is not None:
                cols += list(vel[i])
            if force is not None:
                cols += list(force[i])
            f.write(f"{names[typ[i]]:>3s} " + " ".join(f"{x:22.14e}" for x in cols) + "\n")


def fortran_e(x, w=24, d=16):
    """Fortran Ew.d: 0.<d digits>E<sign><2 digits>, right-justified in w."""
    x = float(x)
    if x == 0.0:
        body, ex = "0." + "0" * d, 0
    else:
        m, e = f"{abs(x):.{d - 1}e}".split("e")
        body, ex = "0." + m.replace(".", ""), int(e) + 1
    sgn = "-" if x < 0 or (x == 0.0 and str(x).startswith("-")) else ""
    es = f"E{ex:+03d}" if abs(ex) < 100 else f"{ex:+04d}"
    return f"{sgn}{body}{es}".rjust(w)


def _ld_real(x):
    # list-directed REAL(8) as gfortran writes it (17 significant digits)
    return f"{float(x):26.17G}"


def _ld_int(n):
    return f"{int(n):12d}"


def _wrap(A, pos):
    B = np.linalg.inv(A)
    s = np.asarray(pos, dtype=np.float64) @ B.T
    s = s - np.where(s >= 0, np.floor(s + 0.5), np.ceil(s - 0.5))  # Fortran NINT
    return s @ A.T


def _ld_header(f, natm, system, A, names, natmi):
    f.write(_ld_int(natm) + "\n")
    f.write(" " + system + "\n")
    for j in range(3):
        f.write("".join(_ld_real(A[a, j]) for a in range(3)) + "\n")
    f.write(_ld_int(len(names)) + "\n")
    f.write(" " + " ".join(f"{n:3s}" for n in names) + "\n")
    f.write("".join(_ld_int(n) for n in natmi) + "\n")


def write_contff(path, system, cell, names, natmi, pos, vel, force):
    """CONTFF: last configuration with velocities and forces (config.f90:208-252);
    positions wrapped by kardir / periodicbc / dirkar as the writer does."""
    A = np.asarray(cell, dtype=np.float64)
    pos = _wrap(A, pos)
    vel = np.asarray(vel, dtype=np.float64)
    force = np.asarray(force, dtype=np.float64)
    natm = pos.shape[0]
    typ = np.repeat(np.arange(len(names)), natmi)
    with open(path, "w") as f:
        f.write(f"{natm:8d}\n{system}\n")
        for j in range(3):
            f.write("".join(f"{A[a, j]:20.12f}" for a in range(3)) + "\n")
        f.write(f"{len(names):4d}\n")
        f.write(" " + " ".join(f"{n:3s}" for n in names) + "\n")
        f.write("".join(_ld_int(n) for n in natmi) + "\n")
        f.write("Cartesian\n")
        for i in range(natm):
            vals = list(pos[i]) + list(vel[i]) + list(force[i])
            f.write(f"{names[typ[i]]:3s}" + "".join(fortran_e(v) for v in vals) + "\n")


def write_dipff(path, system, cell, names, natmi, mu):
    """DIPFF: dipoles at the ions (field.f90:300-337)."""
    A = np.asarray(cell, dtype=np.float64)
    mu = np.asarray(mu, dtype=np.float64).reshape(-1, 3)
    typ = np.repeat(np.arange(len(names)), natmi)
    with open(path, "w") as f:
        _ld_header(f, mu.shape[0], system, A, names, natmi)
        f.write("      ia type                   mux                  muy                 muz\n")
        for i in range(mu.shape[0]):
            f.write(f"{i + 1:8d}  {names[typ[i]]:3s}" + "".join(fortran_e(v) for v in mu[i]) + "\n")


PRESS_UNIT = 0.00624150964712042   # GPa -> eV / A^3 (constants.f90:88)
BOLTZ_UNIT = 8.61734229648141e-05   # eV / K (constants.f90:89)
_OSZ_HEADER = ("     step      Time/Temp   Etot/Pressure    Ekin/Pvir_nb  Utot/Pvir_coul"
               "      U_nb/Omega     U_coul/Htot")


def thermo_nve(res, natm, omega, e_kin, temp, lreducedN=False):
    """calc_thermo (thermo.f90:122-211) for an NVE run with no Morse, harmonic
    or tail terms: the quantities write_thermo prints, from one engforce
    result (u_lj, u_bmhft, u_coul, vir_lj, vir_bmhft, pvirial_coul), the cell
    volume and the caller's kinetic energy (eV) and temperature (K).  With
    lreducedN energies and virial pressures are per ion."""
    nr = float(natm) if lreducedN else 1.0
    u_lj_r, u_bmhft_r, u_coul_r = res["u_lj"] / nr, res["u_bmhft"] / nr, res["u_coul"] / nr
    e_kin_r = e_kin / nr
    u_tot = (u_lj_r + u_coul_r) + u_bmhft_r
    e_tot = u_tot + e_kin_r
    pv_lj_r = (res["vir_lj"] / omega) / nr
    pv_bmhft_r = (res["vir_bmhft"] / omega) / nr
    pv_coul_r = res["pvirial_coul"] / nr
    pv_tot_r = (pv_lj_r + pv_coul_r) + pv_bmhft_r
    pressure_tot_r = (pv_tot_r + float(natm) * temp * BOLTZ_UNIT / omega) / PRESS_UNIT
    return dict(e_tot=e_tot, e_kin_r=e_kin_r, u_tot=u_tot, u_vdw_r=u_lj_r + u_bmhft_r, u_coul_r=u_coul_r,
                temp_r=temp, pressure_tot_r=pressure_tot_r, pvirial_vdw_r=pv_lj_r + pv_bmhft_r,
                pvirial_coul_r=pv_coul_r, pvirial_tot_r=pv_tot_r, omega=omega, h_tot=e_tot)


def write_osziff(f, step, time_ps, th, oszcall):
    """One write_thermo(..., 'osz') record (thermo.f90:370-385) into the open
    file f: every tenth call a 110-dash separator, the column header and a
    separator, then two lines I9,2X,6E16.8.  Returns the next oszcall."""
    if oszcall % 10 == 0:
        f.write("-" * 110 + "\n" + _OSZ_HEADER + "\n" + "-" * 110 + "\n")
    row1 = (time_ps, th["e_tot"], th["e_kin_r"], th["u_tot"], th["u_vdw_r"], th["u_coul_r"])
    row2 = (th["temp_r"], th["pressure_tot_r"], th["pvirial_vdw_r"], th["pvirial_coul_r"], th["omega"],
            th["h_tot"])
    for row in (row1, row2):
        f.write(f"{int(step):9d}  " + "".join(fortran_e(v, 16, 8) for v in row) + "\n")
    return oszcall + 1


def read_osziff(path):
    """OSZIFF records (write_thermo 'osz', thermo.f90:370-385) as a dict of
    arrays keyed like thermo_nve's output plus step and time; separator and
    header lines are skipped."""
    keys1 = ("time", "e_tot", "e_kin_r", "u_tot", "u_vdw_r", "u_coul_r")
    keys2 = ("temp_r", "pressure_tot_r", "pvirial_vdw_r", "pvirial_coul_r", "omega", "h_tot")
    rows = []
    for ln in open(path).read().splitlines():
        t = ln.split()
        if len(t) != 7 or not t[0].isdigit():
            continue
        rows.append((int(t[0]), [float(x.replace("D", "E")) for x in t[1:]]))
    if len(rows) % 2:
        raise ValueError("OSZIFF: records come in pairs of lines")
    out = {k: [] for k in ("step",) + keys1 + keys2}
    for (s1, v1), (s2, v2) in zip(rows[0::2], rows[1::2]):
        if s1 != s2:
            raise ValueError("OSZIFF: the two lines of a record carry different steps")
        out["step"].append(s1)
        for k, v in zip(keys1, v1):
            out[k].append(v)
        for k, v in zip(keys2, v2):
            out[k].append(v)
    return {k: np.array(v) for k, v in out.items()}


def write_dipwfc(path, names, natmi, mu, lwfc):
    """DIPWFC (lwrite_dip_wfc, moment_from_pola.f90:775-782): per ion of a type
    with lwfc >= 0, the type label (a3) and its Wannier-centre dipole in
    3e16.8; mu is the centres' dipoles (natm, 3)."""
    mu = np.asarray(mu, dtype=np.float64).reshape(-1, 3)
    typ = np.repeat(np.arange(len(names)), natmi)
    with open(path, "w") as f:
        for i in range(mu.shape[0]):
            if lwfc[typ[i]] < 0:
                continue
            f.write(f"{names[typ[i]]:3.3s}" + "".join(fortran_e(v, 16, 8) for v in mu[i]) + "\n")


def write_efgall(path, system, cell, names, natmi, efg, lwfc=None):
    """EFGALL, formatted variant (iefgall_format /= 0, field.f90:392-448):
    vxx vyy vzz vxy vxz vyz per ion; efg is (natm, 3, 3) or (natm, 9).  Ions
    of Wannier-centre types (lwfc < 0 per type) are left out (field.f90:422)."""
    A = np.asarray(cell, dtype=np.float64)
    v = np.asarray(efg, dtype=np.float64).reshape(-1, 3, 3)
    typ = np.repeat(np.arange(len(names)), natmi)
    with open(path, "w") as f:
        _ld_header(f, v.shape[0], system, A, names, natmi)
        f.write("      ia type                   vxx                     vyy                     vzz"
                "                     vxy                     vxz                     vyz\n")
        for i in range(v.shape[0]):
            if lwfc is not None and lwfc[typ[i]] < 0:
                continue
            e = v[i]
            vals = (e[0, 0], e[1, 1], e[2, 2], e[0, 1], e[0, 2], e[1, 2])
            f.write(f"{i + 1:8d}  {names[typ[i]]:3s}" + "".join(fortran_e(x) for x in vals) + "\n")


def _read_ld_table(path, ncol):
    with open(path) as f:
        lines = [ln for ln in f.read().splitlines() if ln.strip()]
    natm = int(lines[0].split()[0])
    system = lines[1].strip()
    A = np.array([[float(x) for x in lines[2 + j].split()[:3]] for j in range(3)]).T
    ntype = int(lines[5].split()[0])
    names = lines[6].split()[:ntype]
    natmi = [int(x) for x in lines[7].split()[:ntype]]
    rows = [ln.split() for ln in lines[9:9 + natm]]
    data = np.array([[float(x) for x in r[2:2 + ncol]] for r in rows], dtype=np.float64)
    return dict(natm=natm, system=system, cell=A, names=names, natmi=natmi,
                types=[r[1] for r in rows], data=data)


def read_dipff(path):
    """Returns the header fields and mu (natm, 3)."""
    d = _read_ld_table(path, 3)
    d["mu"] = d.pop("data")
    return d


def read_efgall(path):
    """Returns the header fields and efg (natm, 3, 3), symmetric."""
    d = _read_ld_table(path, 6)
    x = d.pop("data")
    v = np.zeros((x.shape[0], 3, 3))
    v[:, 0, 0], v[:, 1, 1], v[:, 2, 2] = x[:, 0], x[:, 1], x[:, 2]
    v[:, 0, 1] = v[:, 1, 0] = x[:, 3]
    v[:, 0, 2] = v[:, 2, 0] = x[:, 4]
    v[:, 1, 2] = v[:, 2, 1] = x[:, 5]
    d["efg"] = v
    return d


# ---------------------------------------------------------------------------
# Fortran namelists


def expand_includes(text, directory):
    """Replace every line containing '!INCLUDE <file>' by the file's text
    (the deck generator's sed include of examples/ex09/config/gen_tests)."""
    out = []
    for ln in text.splitlines():
        m = re.search(r"!INCLUDE\s*<([^>]+)>", ln)
        if m:
            with open(os.path.join(directory, m.group(1))) as f:
                out.extend(f.read().splitlines())
        else:
            out.append(ln)
    return "\n".join(out)


def _strip_comment(ln):
    q = None
    for i, ch in enumerate(ln):
        if q:
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
        elif ch == "!":
            return ln[:i]
    return ln


def _value(tok):
    t = tok.strip()
    if not t:
        return None
    if t[0] in "'\"":
        return t[1:-1]
    low = t.lower()
    if low in (".true.", "t", ".t."):
        return True
    if low in (".false.", "f", ".f."):
        return False
    try:
        if re.fullmatch(r"[+-]?\d+", t):
            return int(t)
        return float(low.replace("d", "e"))
    except ValueError:
        return t


def _split_values(s):
    vals, cur, q = [], "", None
    for ch in s:
        if q:
            cur += ch
            if ch == q:
                q = None
            continue
        if ch in "'\"":
            q = ch
            cur += ch
        elif ch in ", \t\n":
            if cur:
                vals.append(cur)
            cur = ""
        else:
            cur += ch
    if cur:
        vals.append(cur)
    out = []
    for v in vals:
        m = re.fullmatch(r"(\d+)\*(.+)", v)
        if m:
            out.extend([_value(m.group(2))] * int(m.group(1)))
        else:
            out.append(_value(v))
    return out


def read_namelists(text):
    """Parse every namelist group of a control file.  Returns {group:
    {name: value}} with names lower case; a plain assignment gives a value or
    a list (list-directed fill from element 1), an indexed one gives
    {(i, j, ...): value} entries (1-based indices as written)."""
    groups = {}
    clean = "\n".join(_strip_comment(ln) for ln in text.splitlines())
    for m in re.finditer(r"&(\w+)(.*?)(?:&end\b|^\s*/\s*$)", clean, re.S | re.I | re.M):
        name = m.group(1).lower()
        if name == "end":
            continue
        body = m.group(2)
        g = groups.setdefault(name, {})
        asg = list(re.finditer(r"([A-Za-z_]\w*)\s*(\(([^)]*)\))?\s*=", body))
        for a, b in zip(asg, asg[1:] + [None]):
            key = a.group(1).lower()
            seg = body[a.end(): b.start() if b else len(body)]
            vals = _split_values(seg)
            if a.group(2):
                idx = tuple(int(x) for x in a.group(3).split(","))
                ent = g.setdefault(key, {})
                if not isinstance(ent, dict):
                    ent = g[key] = {(i + 1,): v for i, v in enumerate(ent)}
                if len(vals) == 1:
                    ent[idx] = vals[0]
                else:  # list-directed fill along the first index
                    for k, v in enumerate(vals):
                        ent[(idx[0] + k,) + idx[1:]] = v
            else:
                g[key] = vals[0] if len(vals) == 1 else vals
    return groups


def read_control(path, include_dir=None):
    with open(path) as f:
        text = f.read()
    return read_namelists(expand_includes(text, include_dir or os.path.dirname(path) or "."))


# ---------------------------------------------------------------------------
# namelists -> mdff_params

_CALC = {"md": _abi.CALC_MD, "opt": _abi.CALC_OPT}
_TRUNC = {"notrunc": _abi.TRUNC_NONE, "linear": _abi.TRUNC_LINEAR, "quadratic": _abi.TRUNC_QUADRATIC}


def _table(v, ndim, ntype):
    """A per-type namelist entry as a {0-based index tuple: value} table."""
    if v is None:
        return None
    if isinstance(v, dict):
        return {tuple(i - 1 for i in k): x for k, x in v.items()}
    vals = v if isinstance(v, list) else [v]
    if ndim == 1:
        return {(i,): x for i, x in enumerate(vals)}
    raise ValueError("multi-index table given as a plain list")


_THOLE = {"linear": _abi.THOLE_LINEAR, "expon1": _abi.THOLE_EXPON1,
          "expon2": _abi.THOLE_EXPON2, "gauss": _abi.THOLE_GAUSS}
_THOLE_FIXED = {"expon1": 0.572, "expon2": 1.9088, "gauss": 0.957}
# algo_moment_from_pola_allowed / algo_ext_dipole_allowed (pim.f90:85-91)
_ALGO = {"scf": _abi.ALGO_SCF, "scf_ko_v1": _abi.ALGO_KO_V1, "scf_ko_v2": _abi.ALGO_KO_V2,
         "scf_ko_v3": _abi.ALGO_KO_V3, "scf_ko_v4_1": _abi.ALGO_KO_V4_1,
         "scf_ko_v4_2": _abi.ALGO_KO_V4_2}
_ALGO_NAME = {_abi.ALGO_SCF: "scf", _abi.ALGO_KO_V1: "scf_kO_v1", _abi.ALGO_KO_V2: "scf_kO_v2",
              _abi.ALGO_KO_V3: "scf_kO_v3", _abi.ALGO_KO_V4_1: "scf_kO_v4_1",
              _abi.ALGO_KO_V4_2: "scf_kO_v4_2"}
_EXT = {"aspc": _abi.EXT_ASPC, "poly": _abi.EXT_POLY}


def params_from_namelists(nl, natmi, **extra):
    """mdff_params for the ions per type natmi from parsed namelists, with the
    reference's defaults for everything not given.  Unsupported switches of
    the path (Morse, direct Coulomb, quadrupoles) raise ValueError.  Thole
    functions (coulombtag: thole_functions, thole_function_type, thole_param)
    follow coulomb_check_tag (coulomb.f90:228-234): expon1 / expon2 / gauss
    replace every thole_param by 0.572 / 1.9088 / 0.957.  pimtag's
    algo_moment_from_pola, algo_ext_dipole, omegakO (pim.f90:85-131) and the
    Wannier-centre keywords lwfc, ldip_wfc, rcut_wfc (:93-136) map onto their
    fields; extra keywords (e.g. the engine's precision, solver) override."""
    ntype = len(natmi)
    c = nl.get("controltag", {})
    fd = nl.get("fieldtag", {})
    nb = nl.get("non_bondedtag", {})
    cl = nl.get("coulombtag", {})
    pm = nl.get("pimtag", {})
    if c.get("lmorse", False):
        raise ValueError("lmorse: Morse is never dispatched by engforce")
    if str(c.get("longrange", "ewald")).lower() != "ewald":
        raise ValueError("longrange must be 'ewald'")
    kw = {}
    if cl.get("thole_functions", False):
        ttype = str(cl.get("thole_function_type", "linear")).lower()
        if ttype not in _THOLE:
            raise ValueError(f"thole_function_type {ttype!r} (coulomb.f90:72)")
        kw["thole_type"] = _THOLE[ttype]
        tp = np.full((_abi.NT, _abi.NT), 1.662)
        if "thole_param" in cl:
            for (i, j), v in _table(cl["thole_param"], 2, ntype).items():
                tp[i, j] = float(v)
        if ttype in _THOLE_FIXED:
            tp[:] = _THOLE_FIXED[ttype]
        kw["thole_param"] = tp
    for k in ("lcoulomb", "lbmhft", "lbmhftd", "lnmlj", "lsurf", "lreduced"):
        if k in c:
            kw[k] = int(bool(c[k]))
    for k in ("cutshortrange", "cutlongrange", "skindiff"):
        if k in c:
            kw[k] = float(c[k])
    calc = str(c.get("calc", "md")).lower()
    kw["calc"] = _CALC.get(calc, _abi.CALC_OTHER)
    if "ctrunc" in nb:
        kw["trunc"] = _TRUNC[str(nb["ctrunc"]).lower()]
    if "symmetric_pot" in nb:
        kw["symmetric_pot_nb"] = int(bool(nb["symmetric_pot"]))
    for k in ("epslj", "sigmalj", "plj", "qlj", "abmhftd", "bbmhftd", "cbmhftd", "dbmhftd",
              "bdbmhftd"):
        if k in nb:
            name = {"abmhftd": "Abmhftd", "bbmhftd": "Bbmhftd", "cbmhftd": "Cbmhftd",
                    "dbmhftd": "Dbmhftd", "bdbmhftd": "BDbmhftd"}.get(k, k)
            kw[name] = _table(nb[k], 2, ntype)
    if "qch" in fd:
        q = fd["qch"]
        q = q if isinstance(q, list) else [q] if not isinstance(q, dict) else \
            [q.get((i + 1,), 0.0) for i in range(ntype)]
        kw["qch"] = [float(x) for x in q]
    if "dip" in fd:
        t = _table(fd["dip"], 2, ntype)
        dip = np.zeros((_abi.NT, 3))
        for (it, a), v in t.items():
            dip[it, a] = v
        kw["dip"] = dip
    for k in ("quad",):
        if k in fd and any(float(v) != 0.0 for v in (_table(fd[k], 3, ntype) or {}).values()):
            raise ValueError("quadrupoles are not built")
    if "lautoes" in cl:
        kw["lautoES"] = int(bool(cl["lautoes"]))
    if "epsw" in cl:
        kw["epsw"] = float(cl["epsw"])
    if "alphaes" in cl:
        kw["alphaES"] = float(cl["alphaes"])
    if "kes" in cl:
        k3 = cl["kes"]
        kw["kES"] = tuple(int(x) for x in (k3 if isinstance(k3, list) else [k3] * 3))
    if "symmetric_pot" in pm:
        kw["symmetric_pot_pim"] = int(bool(pm["symmetric_pot"]))
    for k in ("conv_tol_ind",):
        if k in pm:
            kw[k] = float(pm[k])
    for k in ("min_scf_pol_iter", "max_scf_pol_iter", "extrapolate_order"):
        if k in pm:
            kw[k] = int(pm[k])
    if "algo_moment_from_pola" in pm:
        a = str(pm["algo_moment_from_pola"]).lower()
        if a not in _ALGO:
            raise ValueError(f"algo_moment_from_pola {a!r} (pim.f90:89-91)")
        kw["algo_moment_from_pola"] = _ALGO[a]
    if "algo_ext_dipole" in pm:
        a = str(pm["algo_ext_dipole"]).lower()
        if a not in _EXT:
            raise ValueError(f"algo_ext_dipole {a!r} (pim.f90:85-87)")
        kw["algo_ext_dipole"] = _EXT[a]
    if "omegako" in pm:
        kw["omegakO"] = float(pm["omegako"])
    if "lwfc" in pm:  # Wannier centres (pim.f90:93-96)
        t = _table(pm["lwfc"], 1, ntype)
        kw["lwfc"] = [int(t.get((i,), 0)) for i in range(ntype)]
    if "ldip_wfc" in pm:
        kw["ldip_wfc"] = int(bool(pm["ldip_wfc"]))
    if "rcut_wfc" in pm:
        kw["rcut_wfc"] = float(pm["rcut_wfc"])
    if "ldip_polar" in pm:
        t = _table(pm["ldip_polar"], 1, ntype)
        kw["ldip_polar"] = [int(bool(t.get((i,), False))) for i in range(ntype)]
    if "poldip" in pm:
        t = _table(pm["poldip"], 3, ntype)
        pol = np.zeros((_abi.NT, 3, 3))
        for (it, a, b), v in t.items():
            pol[it, a, b] = v
        kw["poldip"] = pol
    if "poldip_iso" in pm:  # pim.f90:222-226
        t = _table(pm["poldip_iso"], 1, ntype)
        pol = kw.get("poldip", np.zeros((_abi.NT, 3, 3)))
        for (it,), v in t.items():
            if float(v) != 0.0:
                pol[it] = np.eye(3) * float(v)
        kw["poldip"] = pol
    for k in ("ldip_damping", "pol_damp_b", "pol_damp_c", "pol_damp_k"):
        if k in pm:
            t = _table(pm[k], 3, ntype)
            if k == "ldip_damping":
                t = {i: int(bool(v)) for i, v in t.items()}
            kw[k] = t
    kw.update(extra)
    return make_params(list(natmi), **kw)


# ---------------------------------------------------------------------------
# mdff_params -> control file


def load_deck(posff_path, control_path, include_dir=None, **extra):
    """A reference run's inputs as the engine takes them: the control file's
    namelists (with its posff_data, controltag) and the POSFF it names.
    Returns dict(params, cell, pos (natm, 3), names, natmi, system[, vel,
    force]); extra keywords override the control file's (e.g. precision)."""
    nl = read_control(control_path, include_dir=include_dir)
    posff_data = str(nl.get("controltag", {}).get("posff_data", "rnn")).lower()
    d = read_posff(posff_path, posff_data=posff_data)
    p = params_from_namelists(nl, d["natmi"], **extra)
    out = dict(params=p, cell=d["cell"], pos=d["pos"], names=d["names"], natmi=d["natmi"], system=d["system"])
    for k in ("vel", "force"):
        if k in d:
            out[k] = d[k]
    return out


def _f(x):
    return f"{float(x):.16e}".replace("e", "d")


def write_control(path, p, names, masses=None, calc="md", extra_md=None):
    """A control file the reference reads for the parameters p (types named
    names): &controltag, &mdtag, &fieldtag, &non_bondedtag, &coulombtag,
    &pimtag with every non-default entry written explicitly."""
    nt = p.ntype
    L = []
    L.append("&controltag")
    L.append(f"  calc = '{calc}'")
    for k in ("lcoulomb", "lbmhft", "lbmhftd", "lnmlj", "lsurf", "lreduced"):
        L.append(f"  {k} = {'.true.' if getattr(p, k) else '.false.'}")
    for k in ("cutshortrange", "cutlongrange", "skindiff"):
        L.append(f"  {k} = {_f(getattr(p, k))}")
    L.append("  longrange = 'ewald'")
    L.append("&end")
    L.append("&mdtag")
    for k, v in (extra_md or {}).items():
        L.append(f"  {k} = {v}")
    L.append("&end")
    L.append("&fieldtag")
    if masses is not None:
        L.append("  mass = " + " ".join(_f(m) for m in masses))
    L.append("  qch = " + " ".join(_f(p.qch[i]) for i in range(nt)))
    for it in range(nt):
        for a in range(3):
            if p.dip[it][a] != 0.0:
                L.append(f"  dip({it + 1},{a + 1}) = {_f(p.dip[it][a])}")
    L.append("&end")
    L.append("&non_bondedtag")
    L.append("  ctrunc = '" + {0: "notrunc", 1: "linear", 2: "quadratic"}[p.trunc] + "'")
    L.append(f"  symmetric_pot = {'.true.' if p.symmetric_pot_nb else '.false.'}")
    for name in ("epslj", "sigmalj", "Abmhftd", "Bbmhftd", "Cbmhftd", "Dbmhftd", "BDbmhftd"):
        tab = getattr(p, name)
        for i in range(nt):
            for j in range(nt):
                if tab[i][j] != 0.0:
                    L.append(f"  {name}({i + 1},{j + 1}) = {_f(tab[i][j])}")
    for name, dflt in (("plj", 6.0), ("qlj", 12.0)):
        tab = getattr(p, name)
        for i in range(nt):
            for j in range(nt):
                if tab[i][j] != dflt:
                    L.append(f"  {name}({i + 1},{j + 1}) = {_f(tab[i][j])}")
    L.append("&end")
    L.append("&coulombtag")
    L.append(f"  lautoES = {'.true.' if p.lautoES else '.false.'}")
    L.append(f"  epsw = {_f(p.epsw)}")
    L.append(f"  alphaES = {_f(p.alphaES)}")
    L.append(f"  kES = {p.kES[0]} {p.kES[1]} {p.kES[2]}")
    if p.thole_type != _abi.THOLE_NONE:
        tname = {v: k for k, v in _THOLE.items()}[p.thole_type]
        L.append("  thole_functions = .true.")
        L.append(f"  thole_function_type = '{tname}'")
        for i in range(nt):
            for j in range(nt):
                L.append(f"  thole_param({i + 1},{j + 1}) = {_f(p.thole_param[i][j])}")
    L.append("&end")
    L.append("&pimtag")
    L.append(f"  symmetric_pot = {'.true.' if p.symmetric_pot_pim else '.false.'}")
    L.append(f"  conv_tol_ind = {_f(p.conv_tol_ind)}")
    L.append(f"  min_scf_pol_iter = {p.min_scf_pol_iter}")
    L.append(f"  max_scf_pol_iter = {p.max_scf_pol_iter}")
    L.append(f"  extrapolate_order = {p.extrapolate_order}")
    L.append(f"  algo_moment_from_pola = '{_ALGO_NAME[p.algo_moment_from_pola]}'")
    L.append(f"  algo_ext_dipole = '{'poly' if p.algo_ext_dipole == _abi.EXT_POLY else 'aspc'}'")
    L.append(f"  omegakO = {_f(p.omegakO)}")
    if any(p.lwfc[it] != 0 for it in range(nt)):
        L.append(f"  ldip_wfc = {'.true.' if p.ldip_wfc else '.false.'}")
        L.append(f"  rcut_wfc = {_f(p.rcut_wfc)}")
        for it in range(nt):
            L.append(f"  lwfc({it + 1}) = {p.lwfc[it]}")
    for it in range(nt):
        if p.ldip_polar[it]:
            L.append(f"  ldip_polar({it + 1}) = .true.")
        for a in range(3):
            for b in range(3):
                if p.poldip[it][a][b] != 0.0:
                    L.append(f"  poldip({it + 1},{a + 1},{b + 1}) = {_f(p.poldip[it][a][b])}")
    for i in range(nt):
        for j in range(nt):
            for k in range(nt):
                if p.ldip_damping[i][j][k]:
                    L.append(f"  ldip_damping({i + 1},{j + 1},{k + 1}) = .true.")
                    L.append(f"  pol_damp_b({i + 1},{j + 1},{k + 1}) = {_f(p.pol_damp_b[i][j][k])}")
                    L.append(f"  pol_damp_c({i + 1},{j + 1},{k + 1}) = {_f(p.pol_damp_c[i][j][k])}")
                    L.append(f"  pol_damp_k({i + 1},{j + 1},{k + 1}) = {p.pol_damp_k[i][j][k]}")
    L.append("&end")
    with open(path, "w") as f:
        f.write("\n".join(L) + "\n")
