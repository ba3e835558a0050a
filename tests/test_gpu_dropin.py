"""SHOCK's own set-up and time loop with its time steps on the GPU.

oracle/_ref/libshockdropin_*.so is ref_harness.c (SHOCK's set-up chain and
the core of startSimulation over the unmodified reference sources) calling
the SHOCK-side binding shock_b200/dropin/GPU.c: GPU_Create after the
set-up, GPU_CalcRungeKutta in place of CalcRungeKutta, GPU_SyncHost before
the state is read.  The same loop with SHOCK's CalcRungeKutta on the CPU is
the reference; after 20 steps the states agree within 1e-10 relative L2
(the bound of the 100-step parity tests).
"""
import pytest

from _util import l2_rel, real
from refbind import DropinSolver, RefSolver, dropin_available
from shock_b200 import cases

pytestmark = pytest.mark.gpu

L2_TOL = 1e-10
NSTEPS = 20

CASES = {
    "tgv16_w5_3d": lambda: cases.taylor_green(16, order=5),
    "random_w9_3d_rk3": lambda: cases.smooth_random(3, 9, (16, 14, 15), seed=9, time_order=3),
    "random_w5_2d": lambda: cases.smooth_random(2, 5, (24, 20, 1), seed=4),
    "mms32_w5_2d": lambda: cases.mms_square(32, 5, family="reference", mms_case=0),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_dropin_loop_matches_reference_loop(name):
    c = CASES[name]()
    if not dropin_available(c.order, c.dim):
        pytest.skip("drop-in harness not built (make -C oracle with the reference sources)")
    ref = RefSolver(c)
    ref.steps(NSTEPS)
    so = real(c, ref.state()[:5])
    d = DropinSolver(c, device=0)
    try:
        d.steps(NSTEPS)
        d.sync()
        st = real(c, d.state()[:5])
    finally:
        d.close()
    err = l2_rel(st, so)
    assert (err <= L2_TOL).all(), err


def _with(case, **kw):
    for k, v in kw.items():
        setattr(case, k, v)
    return case


LOOP_CASES = {
    "tgv16_w5_3d": lambda: cases.taylor_green(16, order=5),
    "random_w9_2d": lambda: cases.smooth_random(2, 9, (24, 20, 1), seed=4),
    # Rudy's outflow relaxes its ghost pressure over tau (src/BC.c:2643-2646)
    "duct_rudy_walls_2d_w5": lambda: _with(cases.duct(2, 5, (28, 18, 1), inflow="inflow_riemann",
                                                      outflow="outflow_rudy", walls="wall_viscous"), l0=200.0),
}


@pytest.mark.parametrize("name", sorted(LOOP_CASES))
def test_dropin_control_loop_matches_reference(name):
    """SHOCK's time-loop control around the step (src/SHOCK.c:557-663) with
    the step on the GPU: numericalTau changes during the run (x 1.1 every 4
    iterations, the accelerator; x 0.7 after a NaN reset, the decelerator),
    a NaN density planted in U_RK on the host at iteration 7 is found by
    GPU_CheckNAN (a device scan, no download while the state is finite) and
    the loop reloads the backup of iteration 5 through GPU_UploadState.  The
    same loop with SHOCK's CalcRungeKutta and checkNAN on the CPU is the
    reference: the same number of resets, the same final tau, and the states
    within 1e-10 relative L2."""
    c = LOOP_CASES[name]()
    if not dropin_available(c.order, c.dim):
        pytest.skip("drop-in harness not built (make -C oracle with the reference sources)")
    kw = dict(nsteps=16, nan_at=7, decel=0.7, accel_every=4, accel=1.1, backup_every=5)
    ref = RefSolver(c)
    resets_ref = ref.control_loop(**kw)
    so, tau_ref = real(c, ref.state()[:5]), ref.tau()
    d = DropinSolver(c, device=0)
    try:
        resets = d.control_loop(**kw)
        st, tau = real(c, d.state()[:5]), d.tau()
    finally:
        d.close()
    assert resets == resets_ref == 1
    assert tau == tau_ref and tau != c.tau
    err = l2_rel(st, so)
    idx = [0, 1, 2, 3, 4] if c.dim == 3 else [0, 1, 2, 4]
    assert (err[idx] <= L2_TOL).all(), err
