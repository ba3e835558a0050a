"""The C ABI library loads and exports every entry point include/shock_b200.h declares."""
import ctypes
import os
import re

import shock_b200

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "shock_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(shock_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_declared_symbols():
    lib = shock_b200.lib()
    syms = declared_symbols()
    assert len(syms) >= 15
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, f"not exported: {missing}"


def test_params_struct_matches_header():
    txt = open(os.path.join(ROOT, "include", "shock_b200.h")).read()
    body = txt[txt.index("typedef struct shock_params"):txt.index("} shock_params;")]
    names = re.findall(r"\b(?:int|double)\s+([a-z_0-9, ]+)(?:\[\d\])?;", body)
    fields = []
    for n in names:
        fields += [x.strip() for x in n.split(",")]
    assert fields == [f[0] for f in shock_b200.Params._fields_]


def test_errors_are_codes_not_exits():
    lib = shock_b200.lib()
    p = shock_b200.Params()
    p.dim = 4
    h = ctypes.c_void_p()
    rc = lib.shock_create(ctypes.byref(p), *([None] * 8), 0, ctypes.byref(h))
    assert rc == -1
    assert b"null" in lib.shock_last_error() or b"dim" in lib.shock_last_error()
