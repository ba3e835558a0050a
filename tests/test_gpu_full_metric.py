"""The full 3D curvilinear metric on the GPU (shock_params.full_metric = 1):
WENO faces with all three normal components and full characteristic rows,
viscous faces with all 30 flux factors (src/ZD.c:47-694,
src/Functions.c:6245-6386), SHOCK's zeta viscous stencil centred on j kept.

Reference: SHOCK's CPU build without the zeroing of the metric's cross
derivatives (src/Functions.c:6479-6484), FP64 and 80-bit (its rounding
floor).  Bounds, normwise per variable over the real points: one RHS and the
state after 20 RK4 steps within max(1e-12, 2*floor) of both builds."""
import numpy as np
import pytest

import shock_b200
from _util import real, rel_err
from refbind import RefSolver, ref_available
from shock_b200 import cases
from test_full_metric_host import skewed, skewed_bounded

pytestmark = pytest.mark.gpu

TOL = 1e-12
NSTEPS = 20


def _with(c, **kw):
    for k, v in kw.items():
        setattr(c, k, v)
    return c


CASES = {
    "tgv16_w5": lambda: cases.taylor_green(16, order=5),
    "tgv16_w9": lambda: cases.taylor_green(16, order=9),
    "skewed_w5": lambda: skewed(5, (18, 14, 16), 3),
    "skewed_w9": lambda: skewed(9, (20, 16, 17), 5),
    "skewed_w5_inviscid": lambda: _with(skewed(5, (16, 15, 17), 4), inviscid=True),
    # faces: no-slip, slip and isothermal walls, farfield, inflow and outflow
    "channel_wall_viscous_w5": lambda: skewed_bounded(cases.channel(3, 5, (16, 12, 14), bc="wall_viscous")),
    "channel_wall_inviscid_w9": lambda: skewed_bounded(cases.channel(3, 9, (18, 14, 16), bc="wall_inviscid")),
    "channel_wall_isothermal_w5": lambda: skewed_bounded(cases.channel(3, 5, (16, 12, 14), bc="wall_isothermal",
                                                                       t_wall=1.1)),
    "channel_farfield_w5": lambda: skewed_bounded(cases.channel(3, 5, (16, 12, 14), bc="farfield")),
    "duct_riemann_rudy_w5": lambda: skewed_bounded(_with(cases.duct(3, 5, (18, 12, 13), inflow="inflow_riemann",
                                                                    outflow="outflow_rudy"), l0=200.0)),
    "duct_subsonic_w9": lambda: skewed_bounded(cases.duct(3, 9, (20, 14, 15))),
}


def _refs(c):
    if not (ref_available(c.order, 3, full=True) and ref_available(c.order, 3, extended=True, full=True)):
        pytest.skip("full-metric reference builds absent (make -C oracle)")
    return RefSolver(c, full=True), RefSolver(c, extended=True, full=True)


@pytest.mark.parametrize("name", sorted(CASES))
def test_full_metric_rhs(name, parity):
    c = CASES[name]()
    r64, r80 = _refs(c)
    q64, q80 = real(c, r64.rhs()), real(c, r80.rhs())
    floor = rel_err(q64, q80)
    tol = np.maximum(TOL, 2 * floor)
    s = shock_b200.Solver(c, full_metric=True)
    q = real(c, s.rhs())
    parity(name, c.name, "full metric rhs vs SHOCK FP64", rel_err(q, q64), tol, floor)
    assert (rel_err(q, q64) <= tol).all(), (rel_err(q, q64), tol)
    assert (rel_err(q, q80) <= tol).all(), (rel_err(q, q80), tol)
    # the cross terms matter: the diagonal form is far from this answer
    qd = real(c, shock_b200.Solver(c).rhs())
    assert rel_err(qd, q64).max() > 1e3 * tol.max()


@pytest.mark.parametrize("name", sorted(CASES))
def test_full_metric_steps(name, parity):
    c = CASES[name]()
    r64, r80 = _refs(c)
    r64.steps(NSTEPS)
    r80.steps(NSTEPS)
    a64, a80 = real(c, r64.state()[:5]), real(c, r80.state()[:5])
    floor = rel_err(a64, a80)
    tol = np.maximum(TOL, 2 * floor)
    s = shock_b200.Solver(c, full_metric=True)
    s.steps(NSTEPS)
    st = real(c, s.state())
    idx = [0, 1, 2, 4] if not np.abs(a64[3]).max() else [0, 1, 2, 3, 4]
    parity(name, c.name, f"full metric {NSTEPS} steps vs SHOCK FP64", rel_err(st, a64)[idx], tol[idx], floor[idx])
    assert (rel_err(st, a64)[idx] <= tol[idx]).all(), (rel_err(st, a64), tol)
    assert (rel_err(st, a80)[idx] <= tol[idx]).all(), (rel_err(st, a80), tol)


def test_full_metric_mixed_refused():
    c = cases.taylor_green(8, order=5)
    with pytest.raises(shock_b200.ShockError):
        shock_b200.Solver(c, precision=shock_b200.SHOCK_MIXED, full_metric=True)
