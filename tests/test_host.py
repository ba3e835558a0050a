"""Host-side pieces that need no GPU: config.ini reading, batch member sizes,
the seeded serving stream and the tuning table keys."""
import math

import numpy as np

import shock_b200
from shock_b200 import autotune, cases

CONFIG = """[General]
Initializationtype\t\t=0\t;(0=New,_1=Use_Existing_Results)
Iterations\t\t\t=100\t;Total_iterations

[Numerics]
TimeOrder\t\t\t=3\t;3_or_4_--_RK3TVD_or_4_RK4
Tau\t\t\t\t=0.00025\t;Numerical_Delta_T

[FluidProperties]
Mach\t\t\t\t=0.1
Reynolds\t\t\t=1600.0
Prandtl\t\t\t\t=0.72
Gamma\t\t\t\t=1.4\t;Isentropic_exponent
R\t\t\t\t=287.0
T\t\t\t\t=300.0
L\t\t\t\t=1.0

[Options]
inviscid\t\t\t=TRUE\t;Viscous(0)/Inviscid(1)
ManufacturedSolution\t\t=no

[BoundaryConditions]
T_wall\t\t\t\t=1.25
rho_inflow\t\t\t=1.1
p_inflow\t\t\t=0.9
p_outflow\t\t\t=0.8
AoA\t\t\t\t=30

[InitializeValues]
u0\t\t\t\t=2.0
"""


def test_params_from_ini(tmp_path):
    f = tmp_path / "config.ini"
    f.write_text(CONFIG)
    base = shock_b200.Params()
    base.dim, base.order, base.ni = 3, 9, 64
    p = shock_b200.params_from_ini(str(f), base)
    assert (p.time_order, p.tau, p.mach, p.reynolds) == (3, 0.00025, 0.1, 1600.0)
    assert (p.prandtl, p.gamma, p.gas_r, p.t0, p.l0) == (0.72, 1.4, 287.0, 300.0, 1.0)
    assert p.inviscid == 1 and p.mms == 0 and p.t_wall == 1.25
    assert (p.rho_inflow, p.p_inflow, p.p_outflow) == (1.1, 0.9, 0.8)
    assert abs(p.u_inflow[0] - 2.0 * math.cos(math.pi / 6)) < 1e-15 and abs(p.u_inflow[1] - 1.0) < 1e-15
    assert (p.dim, p.order, p.ni) == (3, 9, 64)      # not config.ini keys: untouched


def test_params_from_ini_missing_file():
    import pytest
    with pytest.raises(shock_b200.ShockError):
        shock_b200.params_from_ini("/nonexistent/config.ini")


def test_member_bytes():
    c = cases.isentropic_vortex(32, 3.0, 0.5)            # inviscid 2D W5: 39 fields of 38^2 points
    assert shock_b200.member_bytes(c) == (38 * 38 * 39 * 8 + 255) // 256 * 256
    t = cases.taylor_green(16, order=9)                   # viscous 3D W9: 51 fields of 26^3 points
    assert shock_b200.member_bytes(t) == (26 ** 3 * 51 * 8 + 255) // 256 * 256


def test_serving_stream_is_seeded_and_in_range():
    a = cases.serving_stream(12, seed=5)
    b = cases.serving_stream(12, seed=5)
    assert [(t, c.name, n) for t, c, n in a] == [(t, c.name, n) for t, c, n in b]
    times = [t for t, _, _ in a]
    assert times == sorted(times) and times[0] > 0
    for _, c, n in a:
        assert 20 <= n <= 500 and c.order in (5, 9) and c.dim in (2, 3)
        assert 0.0 < c.tau and np.isfinite(c.tau)


def test_tuning_key_groups_similar_batches():
    cs = [cases.isentropic_vortex(n, 2.0, 0.5) for n in (32, 48, 64)]
    k1 = autotune.class_key(2, 5, shock_b200.SHOCK_MIXED, cs)
    k2 = autotune.class_key(2, 5, shock_b200.SHOCK_MIXED, list(reversed(cs)))
    assert k1 == k2 and k1.startswith("2d_w5_mixed_inv_")
    assert k1 != autotune.class_key(2, 5, shock_b200.SHOCK_FP64, cs)
