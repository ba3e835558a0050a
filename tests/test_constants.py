"""The Python package's copies of the C-ABI constants, and the case
builders' face-type names, agree with include/shock_b200.h."""
import os
import re

import shock_b200
from shock_b200 import cases

ROOT = os.path.join(os.path.dirname(__file__), "..")


def _header_defines():
    text = open(os.path.join(ROOT, "include", "shock_b200.h")).read()
    return {m.group(1): int(m.group(2)) for m in re.finditer(r"^#define (SHOCK_\w+) \(?(-?\d+)\)?", text, re.M)}


def test_python_constants_match_header():
    h = _header_defines()
    names = [n for n in dir(shock_b200) if re.fullmatch(r"SHOCK_(BC_\w+|FP64|MIXED|E\w+)", n)]
    assert names
    for n in names:
        assert n in h, n
        assert getattr(shock_b200, n) == h[n], n
    # every face type of the header has its Python constant
    for n in h:
        if n.startswith("SHOCK_BC_"):
            assert getattr(shock_b200, n) == h[n], n


def test_case_face_names_cover_every_face_type():
    h = _header_defines()
    types = {v for n, v in h.items() if n.startswith("SHOCK_BC_") and n != "SHOCK_BC_AUTO"}
    assert set(cases.BC_NAMES.values()) == types
    for name, code in cases.BC_NAMES.items():
        assert h["SHOCK_BC_" + name.upper()] == code, name
