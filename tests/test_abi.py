"""The C-ABI library loads and exports every symbol include/mdff_gpu.h
declares, with the struct layouts the Python mirror assumes (no GPU needed:
no compute entry point is called)."""
import ctypes
import os
import re

import pytest

from mdff_b200 import _abi

HDR = os.path.join(os.path.dirname(__file__), "..", "include", "mdff_gpu.h")


def _declared():
    txt = open(HDR).read()
    return sorted(set(re.findall(r"\b(mdff_gpu_\w+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    from mdff_b200 import build
    build.build()
    return _abi.load_library()


def test_every_declared_symbol_is_exported(lib):
    names = _declared()
    assert len(names) >= 14
    for n in names:
        assert hasattr(lib, n), n
        assert n in _abi.SIGNATURES, n


def test_struct_layouts_match(lib):
    assert lib.mdff_gpu_abi_version() == _abi.ABI_VERSION
    assert lib.mdff_gpu_struct_size(0) == ctypes.sizeof(_abi.MdffParams)
    assert lib.mdff_gpu_struct_size(1) == ctypes.sizeof(_abi.MdffResult)
    assert lib.mdff_gpu_struct_size(2) == ctypes.sizeof(_abi.MdffStats)


def test_strerror_and_bad_args(lib):
    assert lib.mdff_gpu_strerror(_abi.MDFF_ERR_CATASTROPHE).decode().startswith("polarization")
    h = ctypes.c_void_p()
    # a NULL parameter block is rejected before any device work
    assert lib.mdff_gpu_create(None, None, ctypes.byref(h)) == _abi.MDFF_ERR_BAD_ARGS


def test_c_consumer_sees_the_library_layouts(lib, tmp_path):
    """A gcc-compiled C program (tests/c_abi/abi_layout.c) linked against the
    library: C and the library agree on every ABI struct's size."""
    import subprocess
    from .c_abi.build_host import compile_c
    exe = compile_c("abi_layout", tmp_path)
    if exe is None:
        pytest.skip("no C compiler")
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "layouts agree" in r.stdout


def test_c_host_program_reaches_the_engine(lib, tmp_path):
    """The C host driver (tests/c_abi/engforce_host.c) reads its inputs and
    calls mdff_gpu_create; without a device that returns MDFF_ERR_NO_DEVICE
    (the GPU run is in tests/test_gpu_c_host.py)."""
    import subprocess
    import numpy as np
    from mdff_b200 import systems
    from .c_abi.build_host import compile_c
    exe = compile_c("engforce_host", tmp_path)
    if exe is None:
        pytest.skip("no C compiler")
    s = systems.random_ionic((6, 6), L=9.0, seed=3, calc=_abi.CALC_OTHER)
    (tmp_path / "p.bin").write_bytes(bytes(s.params))
    np.ascontiguousarray(s.cell, dtype=np.float64).tofile(str(tmp_path / "c.bin"))
    np.ascontiguousarray(np.concatenate(s.soa())).tofile(str(tmp_path / "x.bin"))
    r = subprocess.run([exe, str(tmp_path / "p.bin"), str(tmp_path / "c.bin"), str(tmp_path / "x.bin"),
                        str(tmp_path / "o.bin"), "1"], capture_output=True, text=True)
    assert r.returncode in (0, _abi.MDFF_ERR_NO_DEVICE), r.stderr
    # a truncated parameter file is refused before the library is called
    (tmp_path / "q.bin").write_bytes(bytes(s.params)[:-8])
    r = subprocess.run([exe, str(tmp_path / "q.bin"), str(tmp_path / "c.bin"), str(tmp_path / "x.bin"),
                        str(tmp_path / "o.bin"), "1"], capture_output=True, text=True)
    assert r.returncode == 102


def _fortran_layout(block):
    """(name, offset, size) of each field of a Fortran bind(c) derived type,
    laid out by the C interoperability rules (natural alignment)."""
    kinds = {"integer(c_int)": 4, "real(c_double)": 8, "type(c_ptr)": 8}
    NT = _abi.NT
    out, off = [], 0
    for ln in block:
        ln = ln.split("!")[0].strip()
        if "::" not in ln:
            continue
        decl, names = (x.strip() for x in ln.split("::", 1))
        w = kinds[decl.replace(" ", "").lower()]
        for m in re.finditer(r"(\w+)\s*(\(([^)]*)\))?", names):
            n = 1
            if m.group(3):
                for d in m.group(3).split(","):
                    n *= NT if d.strip() == "NT" else int(d)
            off = (off + w - 1) // w * w
            out.append((m.group(1).lower(), off, w * n))
            off += w * n
    return out, (off + 7) // 8 * 8


@pytest.mark.parametrize("tname,ctype", [("mdff_params", _abi.MdffParams), ("mdff_result", _abi.MdffResult),
                                         ("mdff_stats", _abi.MdffStats)])
def test_fortran_shim_type_matches_header(tname, ctype):
    """The bind(c) derived types of the Fortran shim include/engforce_gpu.f90
    have the header's fields, in order, at the header's offsets, and the
    header's size."""
    txt = open(os.path.join(os.path.dirname(HDR), "engforce_gpu.f90")).read().splitlines()
    i0 = next(i for i, l in enumerate(txt) if re.match(rf"\s*TYPE, bind\(c\) :: {tname}\s*$", l))
    i1 = next(i for i in range(i0, len(txt)) if txt[i].strip() == "END TYPE")
    fields, size = _fortran_layout(txt[i0 + 1:i1])
    ref = [(n.lower(), getattr(ctype, n).offset, getattr(ctype, n).size) for n, _ in ctype._fields_]
    assert fields == ref
    assert size == ctypes.sizeof(ctype)
