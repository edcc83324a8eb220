"""CPU checks of the C ABI: the in-tree library loads and exports every
function that include/verona_b200.h declares, and argument validation that
needs no GPU behaves as documented. No compute calls are made here."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(vb\w+)\s*\(", txt, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_the_api():
    names = declared_functions()
    for n in ("vb_create", "vb_step", "vb_load_prims", "vb_store_prims", "vb_destroy", "vb_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from verona_b200 import _lib

    L = _lib.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (vb\w+)", out))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in declared_functions():
        assert getattr(L, n) is not None


def test_default_options_are_the_reference_defaults():
    from verona_b200 import _lib

    o = _lib.default_options()
    assert o.version == _lib.ABI_VERSION
    assert (o.recon, o.riemann, o.rk, o.precision, o.guess) == (2, 0, 2, 0, 0)
    assert o.n_iter == 50 and o.tol == 1e-10 and o.floor_ == 1e-7


@pytest.mark.parametrize(
    "args,needle",
    [
        ((4, 8, 8, 8, 3), "dims"),
        ((2, 0, 8, 1, 3), "interior size"),
        ((2, 8, 8, 1, 0), "nghost"),
        ((3, 8, 8, 8, 2), "nghost"),
    ],
)
def test_create_rejects_bad_arguments_without_a_gpu(args, needle):
    from verona_b200 import _lib

    h = C.c_void_p()
    o = _lib.default_options()
    rc = _lib.lib().vb_create(C.byref(h), *args, C.byref(o))
    assert rc == _lib.ERR_ARG
    assert needle in _lib.lib().vb_last_error(None).decode()
    assert not h.value


def test_create_rejects_bad_options_without_a_gpu():
    from verona_b200 import _lib

    L = _lib.lib()
    h = C.c_void_p()
    for kw, code in (({"rk": 4}, _lib.ERR_ARG), ({"recon": 7}, _lib.ERR_ARG), ({"n_iter": 0}, _lib.ERR_ARG),
                     ({"guess": 1}, _lib.ERR_UNSUPPORTED)):
        o = _lib.default_options(**kw)
        assert L.vb_create(C.byref(h), 2, 8, 8, 1, 3, C.byref(o)) == code, kw
    # the previous-W guess runs in 2D and 3D, not 1D
    o = _lib.default_options(guess=2)
    assert L.vb_create(C.byref(h), 1, 8, 1, 1, 3, C.byref(o)) == _lib.ERR_UNSUPPORTED
    o = _lib.default_options()
    o.version = 99
    assert L.vb_create(C.byref(h), 2, 8, 8, 1, 3, C.byref(o)) == _lib.ERR_ARG
    assert L.vb_step(None, 0.1, 1, None) == _lib.ERR_ARG


def test_grid_entry_points_reject_bad_arguments_without_a_gpu():
    import ctypes as C

    from verona_b200 import _lib as L

    lib = L.lib()
    vp, d, i = C.c_void_p, C.c_double, C.c_int
    lib.vb_grid_fluxes.argtypes = [i, i, i, i, vp, d, d, i, i, i, vp, vp]
    lib.vb_grid_limit.argtypes = [i, i, i, i, vp, d, vp]
    lib.vb_grid_last_error.restype = C.c_char_p
    assert lib.vb_grid_fluxes(2, 8, 8, 1, None, 4 / 3, 1e-8, 0, 2, 1, None, None) == L.ERR_ARG
    assert b"null" in lib.vb_grid_last_error()
    assert lib.vb_grid_fluxes(2, 8, 8, 1, C.c_void_p(16), 4 / 3, 1e-8, 2, 2, 1, C.c_void_p(16), None) == L.ERR_ARG
    assert b"axis 2" in lib.vb_grid_last_error()
    assert lib.vb_grid_limit(4, 8, 8, 8, None, 0.0, None) == L.ERR_ARG
    assert b"dims 4" in lib.vb_grid_last_error()


def test_default_ic_is_the_examples():
    import ctypes as C

    from verona_b200 import _lib

    ic = _lib.VBIcParams()
    assert _lib.lib().vb_default_ic(3, 1, C.byref(ic)) == 0
    assert (ic.version, ic.kind, ic.seed, ic.noise) == (_lib.ABI_VERSION, 1, 42, 3e-2)
    assert tuple(ic.box) == (480.0, 120.0, 120.0) and ic.r_eng == 5.0 and ic.engine_rho == 1e-2
    assert _lib.lib().vb_default_ic(2, 1, C.byref(ic)) == 0
    assert tuple(ic.box)[:2] == (800.0, 200.0) and ic.r_eng == 2.0 and ic.engine_rho == 1e-3
    assert _lib.lib().vb_default_ic(3, 5, C.byref(ic)) == -1  # VB_ERR_ARG


def test_struct_layouts_match_the_ctypes_mirrors(tmp_path):
    """Every POD struct of the header has the size and field offsets of its
    ctypes mirror (and so of the Julia structs written after the same layout):
    a C program built by gcc prints them with sizeof / offsetof."""
    import shutil

    from verona_b200 import _lib
    from verona_b200.batch import BatchProblem

    gcc = shutil.which("gcc") or shutil.which("cc")
    if gcc is None:
        pytest.skip("no C compiler")
    mirrors = {"vb_options": _lib.VBOptions, "vb_tuning": _lib.VBTuning, "vb_ic_params": _lib.VBIcParams,
               "vb_batch_problem": BatchProblem}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "verona_b200.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'    printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'    printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = str(tmp_path / "layout")
    r = subprocess.run([gcc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = {}
    for line in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.splitlines():
        cname, field, val = line.split()
        got[(cname, field)] = int(val)
    for cname, py in mirrors.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)
