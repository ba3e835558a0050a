"""Wall and farfield faces on the GPU against SHOCK's own BC code.

The reference is SHOCK's CPU build with the face BC names set as its
loader sets them (BCWallViscous, BCWallInviscid, BCFarfield,
BCWallViscousIsothermal, BCInflow, BCOutflow; src/BC.c) and the inflow /
outflow options of its config.ini (Normal-Subsonic, Normal-Supersonic,
Riemann-Subsonic, Isentrop-Subsonic, Rudy-Subsonic).
Tolerances as in test_gpu_parity.py: one right-hand side within
max(1e-12, 2 * SHOCK's own FP64-vs-80-bit distance) per variable, and the
state after 20 RK steps within max(1e-10, 2 * that distance) relative L2.
"""
import numpy as np
import pytest

import shock_b200
from _util import l2_rel, real, rel_err
from refbind import DropinSolver, RefSolver, dropin_available, ref_available
from shock_b200 import cases

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-12
L2_TOL = 1e-10

CASES = {
    "noslip_3d_w5": lambda: cases.channel(3, 5, (16, 12, 14), bc="wall_viscous", stretch=1.2),
    "slip_3d_w9_euler": lambda: cases.channel(3, 9, (14, 12, 14), bc="wall_inviscid", inviscid=True),
    "farfield_3d_w5": lambda: cases.channel(3, 5, (16, 12, 14), bc="farfield"),
    "noslip_2d_w5": lambda: cases.channel(2, 5, (24, 20, 1), bc="wall_viscous", stretch=1.0),
    "slip_2d_w9": lambda: cases.channel(2, 9, (24, 20, 1), bc="wall_inviscid"),
    "noslip_box_2d_w5": lambda: cases.channel(2, 5, (20, 18, 1), bc="wall_viscous", walls_i=True),
    # Prandtl 0.7 != the 0.72 SHOCK hard-codes for the wall's Gamma
    "isothermal_3d_w5": lambda: cases.channel(3, 5, (16, 12, 14), bc="wall_isothermal", stretch=1.2,
                                              prandtl=0.7, t_wall=1.05),
    "isothermal_2d_w9": lambda: cases.channel(2, 9, (24, 20, 1), bc="wall_isothermal", prandtl=0.7, t_wall=0.95),
    # through-flow: inflow on the x-lower face, subsonic outflow on the x-upper face
    "duct_sub_3d_w5": lambda: cases.duct(3, 5, (20, 12, 14)),
    "duct_super_3d_w9_euler": lambda: cases.duct(3, 9, (20, 12, 14), inflow="inflow_supersonic", mach=2.0,
                                                 inviscid=True),
    "duct_sub_walls_2d_w5": lambda: cases.duct(2, 5, (28, 18, 1), walls="wall_viscous"),
    "duct_super_2d_w9": lambda: cases.duct(2, 9, (28, 20, 1), inflow="inflow_supersonic", mach=2.0),
    # Riemann-invariant inflow and outflow, isentropic inflow
    "duct_riemann_3d_w5": lambda: cases.duct(3, 5, (20, 12, 14), inflow="inflow_riemann", outflow="outflow_riemann"),
    "duct_riemann_walls_2d_w9": lambda: cases.duct(2, 9, (28, 20, 1), inflow="inflow_riemann",
                                                   outflow="outflow_riemann", walls="wall_viscous"),
    "duct_isentropic_3d_w9_euler": lambda: cases.duct(3, 9, (20, 12, 14), inflow="inflow_isentropic",
                                                      inviscid=True),
    "duct_isentropic_slip_2d_w5": lambda: cases.duct(2, 5, (28, 18, 1), inflow="inflow_isentropic",
                                                     outflow="outflow_riemann", walls="wall_inviscid"),
    # Rudy's outflow: U_lastStep's ghost pressure relaxed towards p_outflow;
    # L0 = 200 m makes AlphaNonRef * tau about 1e-3 per step
    "duct_rudy_3d_w5": lambda: cases.duct(3, 5, (20, 12, 14), outflow="outflow_rudy"),
    "duct_rudy_walls_2d_w9": lambda: _with(cases.duct(2, 9, (28, 20, 1), inflow="inflow_riemann",
                                                      outflow="outflow_rudy", walls="wall_viscous"), l0=200.0),
    "duct_rudy_slip_3d_w9_euler": lambda: _with(cases.duct(3, 9, (20, 12, 14), outflow="outflow_rudy",
                                                           walls="wall_inviscid", inviscid=True), l0=200.0),
    # Rudy faces on two axes sharing a corner, walls on the others
    "box_rudy_2d_w5": lambda: _with(cases.duct(2, 5, (28, 18, 1), outflow="outflow_rudy", walls="wall_viscous"),
                                    bc=(1, 11, 1, 11, 0, 0), l0=200.0),
    # three-stage RK: the step ends on another state buffer
    "duct_rudy_rk3_2d_w5": lambda: _with(cases.duct(2, 5, (28, 18, 1), inflow="inflow_riemann", outflow="outflow_rudy",
                                                    walls="wall_viscous", time_order=3), l0=200.0),
}


def _with(c, **kw):
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def _need(c):
    if not ref_available(c.order, c.dim) or not ref_available(c.order, c.dim, extended=True):
        pytest.skip("reference build not present")


@pytest.mark.parametrize("name", sorted(CASES))
def test_wall_rhs_matches_reference(name):
    c = CASES[name]()
    _need(c)
    q = real(c, shock_b200.Solver(c).rhs())
    ref, ref80 = real(c, RefSolver(c).rhs()), real(c, RefSolver(c, extended=True).rhs())
    tol = np.maximum(RHS_TOL, 2.0 * rel_err(ref, ref80))
    assert (rel_err(q, ref) <= tol).all(), (rel_err(q, ref), tol)


def _check_steps(c, nsteps, parity, label):
    """The GPU state after nsteps against SHOCK's FP64 and 80-bit builds.
    Bound, per variable (relative L2): 1e-10, or where SHOCK's own FP64 build
    drifts further than that from its 80-bit build (floor; the WENO9 and
    supersonic ducts amplify rounding, up to 3e-8 in 20 steps), the GPU must
    stay within 2 floors of the 80-bit answer, i.e. about as accurate as
    SHOCK's FP64 build, and so within 3 floors of the FP64 build."""
    s = shock_b200.Solver(c)
    r, r80 = RefSolver(c), RefSolver(c, extended=True)
    for x in (s, r, r80):
        x.steps(nsteps)
    ref, ref80, st = real(c, r.state()[:5]), real(c, r80.state()[:5]), real(c, s.state())
    floor = l2_rel(ref, ref80)
    err64, err80 = l2_rel(st, ref), l2_rel(st, ref80)
    parity(label, c.name, f"{nsteps} steps L2 vs SHOCK FP64", err64, np.maximum(L2_TOL, 3.0 * floor), floor)
    assert (err80 <= np.maximum(L2_TOL, 2.0 * floor)).all(), (err80, floor)
    assert (err64 <= np.maximum(L2_TOL, 3.0 * floor)).all(), (err64, floor)


@pytest.mark.parametrize("name", sorted(CASES))
def test_wall_steps_match_reference(name, parity):
    """20 steps (bound: _check_steps)."""
    c = CASES[name]()
    _need(c)
    _check_steps(c, 20, parity, "walls_20")


@pytest.mark.parametrize("name", ["noslip_3d_w5", "duct_rudy_walls_2d_w9", "duct_isentropic_slip_2d_w5"])
def test_wall_100_steps_match_reference(name, parity):
    """100 RK steps (bound: _check_steps), the length of the periodic parity
    tests."""
    c = CASES[name]()
    _need(c)
    _check_steps(c, 100, parity, "walls_100")


@pytest.mark.parametrize("name", ["duct_rudy_walls_2d_w9", "box_rudy_2d_w5"])
def test_rudy_reset_to_backup_matches_reference(name):
    """SHOCK's NaN reset reloads U_RK and U_lastStep, p included, from a
    backup (src/SHOCK.c:598-601, 661-664): both solvers go back to SHOCK's
    state after 3 steps once they have run 7, then run 10 more.  The Rudy
    faces start again from the backup's ghost pressure."""
    c = CASES[name]()
    _need(c)
    refs = [RefSolver(c), RefSolver(c, extended=True)]
    backups = []
    for r in refs:
        r.steps(3)
        backups.append(r.state())
        r.steps(4)
    s = shock_b200.Solver(c)
    s.steps(7)
    for r, b in zip(refs, backups):
        r.set_state(b[:5])
        r.set_last_pressure(b[5])
    s.set_state(backups[0][:5])
    s.set_last_pressure(backups[0][5])
    for x in refs + [s]:
        x.steps(10)
    ref = real(c, refs[0].state()[:5])
    tol = np.maximum(L2_TOL, 2.0 * l2_rel(ref, real(c, refs[1].state()[:5])))
    err = l2_rel(real(c, s.state()), ref)
    assert (err <= tol).all(), (err, tol)


@pytest.mark.parametrize("name", ["noslip_3d_w5", "duct_rudy_3d_w5", "duct_riemann_walls_2d_w9"])
def test_wall_mixed_precision_l2(name):
    c = CASES[name]()
    a = shock_b200.Solver(c)
    b = shock_b200.Solver(c, precision=shock_b200.SHOCK_MIXED)
    a.steps(20)
    b.steps(20)
    err = l2_rel(real(c, b.state()), real(c, a.state()))
    assert (err <= 1e-6).all(), err


@pytest.mark.parametrize("name", ["noslip_3d_w5", "duct_sub_3d_w5", "duct_riemann_3d_w5", "duct_rudy_3d_w5",
                                  "duct_isentropic_slip_2d_w5"])
def test_wall_dropin_loop_matches_reference_loop(name):
    """SHOCK's own time loop with the binding (GPU.c) in place of
    CalcRungeKutta: the binding maps SHOCK's face names and inflow /
    outflow option flags to the library's face types."""
    c = CASES[name]()
    if not dropin_available(c.order, c.dim):
        pytest.skip("drop-in harness not built")
    r, r80 = RefSolver(c), RefSolver(c, extended=True)
    r.steps(20)
    r80.steps(20)
    d = DropinSolver(c, device=0)
    try:
        d.steps(20)
        d.sync()
        st = real(c, d.state()[:5])
    finally:
        d.close()
    ref = real(c, r.state()[:5])
    tol = np.maximum(L2_TOL, 2.0 * l2_rel(ref, real(c, r80.state()[:5])))
    err = l2_rel(st, ref)
    assert (err <= tol).all(), (err, tol)
