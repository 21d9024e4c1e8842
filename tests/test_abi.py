"""The C-ABI library loads without a GPU and exports every entry point of include/mdft_b200.h."""
import ctypes
import os
import re

import pytest

from mdft_b200 import engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "mdft_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(mdft_\w+)\s*\(", text, re.M)))


def test_header_and_binding_agree():
    assert declared_functions() == sorted(engine.SIGNATURES)


def test_library_exports_every_symbol():
    if not os.path.exists(engine.library_path()):
        pytest.fail("libmdft_b200.so not built")
    L = ctypes.CDLL(engine.library_path())
    for name in declared_functions():
        assert hasattr(L, name), name


def test_argument_errors_without_gpu():
    L = engine.lib()
    d = engine._Desc(15, 16, 16, 8.0, 8.0, 8.0, 1, 2, 298.0, 0.0333, b"/nonexistent", 0, 0)
    h = ctypes.c_void_p()
    assert L.mdft_create(ctypes.byref(d), ctypes.byref(h)) == -1
    assert b"even" in L.mdft_last_error()
    d = engine._Desc(16, 16, 16, 8.0, 8.0, 8.0, 7, 2, 298.0, 0.0333, b"/nonexistent", 0, 0)
    assert L.mdft_create(ctypes.byref(d), ctypes.byref(h)) == -1
    d = engine._Desc(16, 16, 16, 8.0, 8.0, 8.0, 1, 2, 298.0, 0.0333, b"/nonexistent/ck", 0, 0)
    assert L.mdft_create(ctypes.byref(d), ctypes.byref(h)) == -2
    assert b"cannot open" in L.mdft_last_error()
    assert L.mdft_destroy(None) == 0


def test_batch_argument_errors_without_gpu():
    L = engine.lib()
    o = engine._MinOpts(5, 1e-4, -1.0, 100, 0, 0.0, 1)
    out = (ctypes.c_double * 6)()
    res = (engine._MinRes * 1)()
    # no handle
    assert L.mdft_solve_batch(None, 0, None, 0, 0, None, None, None, None, 10.0, 71.0, ctypes.byref(o), None, None, None) == -1
    # a solute pointing past the handle array is rejected before any handle is touched
    hs = (ctypes.c_void_p * 1)(ctypes.c_void_p(1))
    sol = (engine._Solute * 1)()
    sol[0] = engine._Solute(1, None, None, None, None, 3, None)
    rc = L.mdft_solve_batch(hs, 1, ctypes.cast(sol, ctypes.c_void_p), 1, 0, None, None, None, None, 10.0, 71.0,
                            ctypes.byref(o), ctypes.cast(out, engine._DP), ctypes.cast(res, ctypes.c_void_p), None)
    assert rc == -1
    assert b"out of range" in L.mdft_last_error()


def _c_fields(text, name):
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), text, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    out = []
    for decl in body.split(";"):
        decl = decl.strip()
        if decl:
            out += [re.sub(r"[\s*]", "", v).split("[")[0] for v in re.split(r",", re.sub(r"^[\w\s]+?\s(?=[\w*]+(\s*,|$))", "", decl))]
    return out


def _f_fields(text, name):
    body = re.search(r"type, bind\(C\) :: %s\n(.*?)end type" % name, text, re.S).group(1)
    out = []
    for line in body.splitlines():
        if "::" in line:
            out += [v.strip() for v in line.split("::")[1].split("!")[0].split(",")]
    return out


@pytest.mark.parametrize("name", ["mdft_desc", "mdft_minimize_opts", "mdft_minimize_result"])
def test_fortran_interface_types_match_the_header(name):
    h = open(os.path.join(ROOT, "include", "mdft_b200.h")).read()
    f = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    assert _f_fields(f, name) == _c_fields(h, name)


def test_ck_table_checks_without_gpu(tmp_path):
    # the reference's c(k) assertions (src/module_read_c_luc.f90:102-108, src/module_input.f90:638-646)
    # run before any device call: a table shorter than the grid's qmax, and a non-uniform abscissa
    from mdft_b200 import synth
    L = engine.lib()
    h = ctypes.c_void_p()
    short = str(tmp_path / "short.txt")
    synth.make_ck_file(short, 1, kmax=2.0, dk=0.02)
    d = engine._Desc(16, 16, 16, 8.0, 8.0, 8.0, 1, 2, 298.0, 0.0333, short.encode(), 0, 0)
    assert L.mdft_create(ctypes.byref(d), ctypes.byref(h)) == -2
    assert b"rows needed" in L.mdft_last_error()
    lines = open(short).read().split("\n")
    first = next(i for i, l in enumerate(lines) if i > 15 and l.strip()[:1].isdigit())  # first data row
    parts = lines[first + 5].split(None, 1)
    lines[first + 5] = "%.6f %s" % (float(parts[0]) + 0.005, parts[1])
    bad = str(tmp_path / "bad.txt")
    open(bad, "w").write("\n".join(lines))
    d = engine._Desc(16, 16, 16, 8.0, 8.0, 8.0, 1, 2, 298.0, 0.0333, bad.encode(), 0, 0)
    assert L.mdft_create(ctypes.byref(d), ctypes.byref(h)) == -2
    assert b"uniform" in L.mdft_last_error()


def test_bridge_and_mixture_host_checks_without_gpu():
    L = engine.lib()
    v = ctypes.c_double()
    # c00_000 of src/module_coarse_grained_gageat_bridge.f90:260-263
    assert L.mdft_cgb_c00(b"spce", 0, ctypes.byref(v)) == 0 and v.value == -14.64872
    assert L.mdft_cgb_c00(b"spce", 3, ctypes.byref(v)) == 0 and v.value == -13.665
    assert L.mdft_cgb_c00(b"tip3p", 1, ctypes.byref(v)) == 0 and v.value == -11.9078
    assert L.mdft_cgb_c00(b"acetonitrile", 1, ctypes.byref(v)) == -1
    assert b"acetonitrile" in L.mdft_last_error()
    assert L.mdft_set_bridge_cgb(None, 1, 0.0, 1.0, -13.665) == -1
    m = ctypes.c_void_p()
    x = (ctypes.c_double * 2)(0.5, 0.5)
    hs = (ctypes.c_void_p * 2)(None, None)
    assert L.mdft_mixture_create(hs, 1, x, ctypes.byref(m)) == -1
    assert b"at least two" in L.mdft_last_error()
    assert L.mdft_mixture_create(hs, 2, x, ctypes.byref(m)) == -1
    assert b"null species" in L.mdft_last_error()
    hs9 = (ctypes.c_void_p * 9)(*([None] * 9))
    x9 = (ctypes.c_double * 9)(*([1.0 / 9] * 9))
    assert L.mdft_mixture_create(hs9, 9, x9, ctypes.byref(m)) == -1
    assert b"at most 8" in L.mdft_last_error()
    assert L.mdft_mixture_destroy(None) == 0
