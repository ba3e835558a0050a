"""config.ini read by the library (shock_params_from_ini) against SHOCK's
own reader of the same file: ConfigImport (src/Import.c:17-275) with the
iniparser SHOCK ships, built unmodified into oracle/_ref/libshockini_3d.so
and run in a child process.  Every field the library fills must come out
equal, bit for bit, for SHOCK's own config.ini and for files that exercise
iniparser's rules (quotes, comments, continuation lines, case, duplicate
keys, sections, integer bases, booleans, empty values, the longest line it
takes); files iniparser rejects (a line of more than 1022 characters, a
last line without a newline) must be rejected by both."""
import math
import os

import pytest

import shock_b200
from refbind import config_available, config_import

pytestmark = pytest.mark.skipif(not config_available(),
                                reason="configuration oracle absent (make -C oracle with the reference sources)")

# SHOCK's config.ini, in the reference tree beside this repository
SHIPPED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "..", "reference", "config.ini")

# the defaults ConfigImport gives a missing key (src/Import.c:48-145, 225-247)
SHOCK_DEFAULTS = dict(time_order=4, tau=-1.0, mach=-1.0, reynolds=-1.0, prandtl=-1.0, gamma=-1.0, gas_r=-1.0,
                      t0=-1.0, l0=-1.0, t_wall=1.0, rho_inflow=1.0, p_inflow=1.0, p_outflow=1.0, inviscid=0, mms=0)

BASE = """; a configuration in SHOCK's layout
[General]
Iterations\t\t=100\t;total iterations
MeshPath\t\t=/data/mesh.cgns
SwapDivFile\t\t=0

[Numerics]
TimeOrder\t\t=4\t;3 or 4
Tau\t\t\t=0.001

[BoundaryConditions]
Inflow-Normal-Subsonic\t=FALSE
Inflow-Riemann-Subsonic\t=TRUE
Inflow-Isentrop-Subsonic\t=FALSE
Inflow-Normal-Supersonic\t=FALSE
rho_Inflow\t\t=1.2
p_Inflow\t\t=0.9
AoA\t\t\t=12.5\t;degrees
Outflow-Normal-Subsonic\t=FALSE
Outflow-Riemann-Subsonic\t=TRUE
Outflow-Rudy-Subsonic\t=FALSE
p_Outflow\t\t=0.95
T_Wall\t\t\t=1.1

[FluidProperties]
Mach\t\t\t=0.7
Reynolds\t\t=500000.0
Prandtl\t\t\t=0.72
Gamma\t\t\t=1.4
R\t\t\t=287.0
T\t\t\t=300.0
L\t\t\t=1.0

[InitializeValues]
u0\t\t\t=1.3

[Options]
Inviscid\t\t=FALSE
ManufacturedSolution\t=FALSE
"""

VARIANTS = {
    "as_written": lambda s: s,
    "crlf_line_ends": lambda s: s.replace("\n", "\r\n"),
    "double_quoted": lambda s: s.replace("Mach\t\t\t=0.7", 'Mach = "0.3" ; quoted'),
    "single_quoted": lambda s: s.replace("Mach\t\t\t=0.7", "Mach = '  0.25 '"),
    "empty_quotes": lambda s: s.replace("Mach\t\t\t=0.7", 'Mach = ""'),
    "unterminated_quote": lambda s: s.replace("Mach\t\t\t=0.7", 'Mach = "0.45'),
    "hash_comment": lambda s: s.replace("Prandtl\t\t\t=0.72", "Prandtl = 0.5 # comment"),
    "value_is_a_comment": lambda s: s.replace("Prandtl\t\t\t=0.72", "Prandtl = ;0.5"),
    "empty_value": lambda s: s.replace("T_Wall\t\t\t=1.1", "T_Wall ="),
    "upper_case_names": lambda s: s.replace("[FluidProperties]", "[FLUIDPROPERTIES]").replace("Reynolds", "REYNOLDS"),
    "spaced_section": lambda s: s.replace("[FluidProperties]", "[  FluidProperties ]"),
    "blank_section": lambda s: s.replace("[FluidProperties]", "[ ]"),
    "empty_section": lambda s: s.replace("[FluidProperties]", "[]"),
    "unclosed_section": lambda s: s.replace("[FluidProperties]", "[FluidProperties"),
    "duplicate_key": lambda s: s.replace("Tau\t\t\t=0.001", "Tau = 0.5\nTau = 2e-4"),
    "continued_value": lambda s: s.replace("Reynolds\t\t=500000.0", "Reynolds = 5000\\\n00.0"),
    "continued_by_blank": lambda s: s.replace("Reynolds\t\t=500000.0", "Reynolds = 1000\\\n\n"),
    "octal_time_order": lambda s: s.replace("TimeOrder\t\t=4", "TimeOrder = 03"),
    "bad_octal_time_order": lambda s: s.replace("TimeOrder\t\t=4", "TimeOrder = 08"),
    "hex_time_order": lambda s: s.replace("TimeOrder\t\t=4", "TimeOrder = 0x3"),
    "bare_exponent": lambda s: s.replace("Tau\t\t\t=0.001", "Tau = .5e-3"),
    "boolean_words": lambda s: s.replace("Inviscid\t\t=FALSE", "Inviscid = yes").replace(
        "ManufacturedSolution\t=FALSE", "ManufacturedSolution = True"),
    "boolean_other": lambda s: s.replace("Inviscid\t\t=FALSE", "Inviscid = 2"),
    "boolean_empty": lambda s: s.replace("Inviscid\t\t=FALSE", "Inviscid ="),
    "line_without_equals": lambda s: s.replace("Mach\t\t\t=0.7", "Mach 0.3\nMach=0.4"),
    "key_with_inner_space": lambda s: s.replace("Gamma\t\t\t=1.4", "Gam ma = 1.3\nGamma\t=\t1.35\t"),
    "missing_keys": lambda s: s.replace("u0\t\t\t=1.3", "").replace("Prandtl\t\t\t=0.72", ""),
    "missing_inflow_velocity": lambda s: s.replace("u0\t\t\t=1.3", "").replace("AoA\t\t\t=12.5\t;degrees", ""),
    "last_line_a_comment_without_newline": lambda s: s + ";",
    "longest_line": lambda s: s.replace("[Numerics]", "[Numerics]\n; " + "x" * 1020),
    "longest_continued_line": lambda s: s.replace("Tau\t\t\t=0.001", "Tau = 0.002 ;" + "y" * 500 + "\\\n" + "z" * 500),
}

REJECTED = {
    "last_line_without_newline": lambda s: s + "L = 2.0",
    "line_too_long": lambda s: s.replace("[Numerics]", "[Numerics]\n; " + "x" * 1021),
    "continued_line_too_long": lambda s: s.replace("Tau\t\t\t=0.001", "Tau = 0.002 ;" + "y" * 500 + "\\\n" + "z" * 510),
}


def _library(path):
    p = shock_b200.Params()
    for k, v in SHOCK_DEFAULTS.items():
        setattr(p, k, v)
    # ConfigImport's inflow velocity without AoA and u0: cos(0) * 1, sin(0) * 1
    p.u_inflow[0], p.u_inflow[1], p.u_inflow[2] = 1.0, 0.0, 0.0
    p = shock_b200.params_from_ini(str(path), p)
    out = {k: getattr(p, k) for k in SHOCK_DEFAULTS}
    out.update(u_inflow=p.u_inflow[0], v_inflow=p.u_inflow[1], w_inflow=p.u_inflow[2])
    return out


def _compare(path):
    mine = _library(path)
    ref = config_import(path)
    diff = {k: (mine[k], ref[k]) for k in mine if not (mine[k] == ref[k] or (math.isnan(mine[k]) and math.isnan(ref[k])))}
    assert not diff, diff


@pytest.mark.parametrize("name", sorted(VARIANTS))
def test_config_ini_read_as_shock_reads_it(tmp_path, name):
    path = tmp_path / "config.ini"
    path.write_bytes(VARIANTS[name](BASE).encode())
    _compare(path)


def test_shipped_config_ini():
    if not os.path.exists(SHIPPED):
        pytest.skip("SHOCK's config.ini is not beside this repository")
    _compare(SHIPPED)


@pytest.mark.parametrize("name", sorted(REJECTED))
def test_config_ini_rejected_as_shock_rejects_it(tmp_path, name):
    path = tmp_path / "config.ini"
    path.write_bytes(REJECTED[name](BASE).encode())
    with pytest.raises(RuntimeError):
        config_import(path)
    with pytest.raises(shock_b200.ShockError):
        shock_b200.params_from_ini(str(path), shock_b200.Params())
