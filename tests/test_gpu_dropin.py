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
