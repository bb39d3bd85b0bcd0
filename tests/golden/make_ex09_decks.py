"""Builds tests/golden/ex09_decks.npz from the reference's ex09 inputs
(examples/ex09/config: POSFF, pot_mdff/control_template.F, the *.POT decks,
test.config): the 11 force-field combinations of its test table, each control
file assembled the way examples/ex09/config/gen_tests does it (placeholders
from test.config, '!INCLUDE <file>' expanded) and read with mdff_b200.mdffio.

The fixture stores, per test, the parsed mdff_params as raw bytes, plus the
POSFF's cell, names, ions per type and wrapped positions.  Run once with the
path of a checkout of the reference (argument, or MDFF_REFERENCE):
    python tests/golden/make_ex09_decks.py <reference checkout>
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from mdff_b200 import mdffio  # noqa: E402


def read_table(cfg):
    glob, rows = {}, []
    table = False
    for ln in open(cfg):
        t = ln.split()
        if not t:
            continue
        if t[0] == "TABLE:":
            table = True
            continue
        if table:
            cells = [c.strip() for c in ln.strip().strip("|").split("|")]
            if len(cells) == 6 and cells[0].isdigit():
                rows.append([cells[0]] + [c == "YES" for c in cells[1:]])
        elif len(t) >= 2:
            glob[t[0]] = t[1]
    return glob, rows


def assemble(pot_dir, glob, row):
    """control file text of one test (gen_tests Docontrol + its sed script)."""
    _, bmh, ftd, coul, pim, damp = row
    text = open(os.path.join(pot_dir, "control_template.F")).read()
    incl = ["IONS.POT"]
    if ftd:
        incl.append("BMHFTD.POT")
    elif bmh:
        incl.append("BMHFT.POT")
    if pim:
        incl.append("PIMD.POT" if damp else "PIM.POT")
    lines = []
    for ln in text.splitlines():
        hit = [f for f in incl if f"!INCLUDE <{f}>" in ln]
        if hit:
            lines.extend(open(os.path.join(pot_dir, hit[0])).read().splitlines())
        elif "!INCLUDE" in ln:
            continue  # includes not selected for this test are dropped
        else:
            lines.append(ln)
    text = "\n".join(lines)
    tf = lambda b: ".true." if b else ".false."
    for k, v in (("__RCUT__", glob["RCUT"]), ("__EPSW__", glob["EPSW"]), ("__BMH__", tf(bmh)),
                 ("__FT_ON__", tf(ftd)), ("__COUL__", tf(coul))):
        text = text.replace(k, v)
    return text


def main(ref):
    cfgdir = os.path.join(ref, "examples", "ex09", "config")
    pot = os.path.join(cfgdir, "pot_mdff")
    glob, rows = read_table(os.path.join(cfgdir, "test.config"))
    posff = mdffio.read_posff(os.path.join(cfgdir, "POSFF"))
    out = dict(cell=posff["cell"], pos=posff["pos"], natmi=np.array(posff["natmi"]),
               names=np.array(posff["names"]))
    tests = []
    for row in rows:
        nl = mdffio.read_namelists(assemble(pot, glob, row))
        p = mdffio.params_from_namelists(nl, posff["natmi"])
        out[f"params_{row[0]}"] = np.frombuffer(bytes(p), dtype=np.uint8).copy()
        tests.append([int(row[0])] + [int(x) for x in row[1:]])
    out["tests"] = np.array(tests)
    np.savez_compressed(os.path.join(HERE, "ex09_decks.npz"), **out)
    print("wrote", len(tests), "decks")


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MDFF_REFERENCE", "")
    if not ref:
        sys.exit("usage: make_ex09_decks.py <reference checkout> (or set MDFF_REFERENCE)")
    main(ref)
