"""The full 3D curvilinear metric (shock_params.full_metric = 1) on the host:
the geometry set-up keeps the cross derivatives of the coordinates that
SHOCK zeroes (src/Functions.c:6479-6484).  Reference: SHOCK's set-up chain
built without those six lines (oracle/_ref/libshockreffull_*, patched at
build time by oracle/Makefile); the coordinates, Jacobian and all nine
metric terms must agree bit for bit."""
import math

import numpy as np
import pytest

import shock_b200
from refbind import RefSolver, ref_available
from shock_b200 import cases


def skewed(order, n, seed):
    """A smooth random periodic state on a sheared periodic box: each
    coordinate displaced by 4 % of its period times a product of sines of
    the other two, so every cross metric term is of order 0.1."""
    c = cases.smooth_random(3, order, n, seed=seed)
    L = c.period
    X, Y, Z = c.x.copy(), c.y.copy(), c.z.copy()
    tp = 2 * math.pi
    c.x = X + 0.04 * L[0] * np.sin(tp * Y / L[1]) * np.sin(tp * Z / L[2])
    c.y = Y + 0.04 * L[1] * np.sin(tp * X / L[0]) * np.sin(tp * Z / L[2])
    c.z = Z + 0.04 * L[2] * np.sin(tp * X / L[0]) * np.sin(tp * Y / L[1])
    c.tau = cases.cfl_tau(c)
    c.name = f"skewed{n[0]}x{n[1]}x{n[2]}_w{order}"
    return c


def skewed_bounded(c):
    """The same shear on a block with wall, farfield, inflow or outflow
    faces: the displacements keep the periodic axes periodic and move the
    bounded faces off their planes."""
    L = c.period
    X, Y, Z = c.x.copy(), c.y.copy(), c.z.copy()
    tp = 2 * math.pi
    per = c.periodic

    def wave(a, arr):   # periodic along a periodic axis, a half wave across a bounded one
        return np.sin(tp * arr / L[a]) if per[a] else np.cos(math.pi * arr / L[a])

    c.x = X + 0.03 * L[0] * wave(1, Y) * wave(2, Z)
    c.y = Y + 0.03 * L[1] * wave(0, X) * wave(2, Z)
    c.z = Z + 0.03 * L[2] * wave(0, X) * wave(1, Y)
    c.tau = cases.cfl_tau(c)
    c.name = "skewed_" + c.name
    return c


CASES = {
    "tgv12_w5": lambda: cases.taylor_green(12, order=5),
    "tgv12_w9": lambda: cases.taylor_green(12, order=9),
    "skewed_w5": lambda: skewed(5, (14, 11, 13), 3),
    "skewed_channel_w5": lambda: skewed_bounded(cases.channel(3, 5, (14, 11, 12), bc="wall_inviscid")),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_full_geometry_matches_patched_shock(name):
    c = CASES[name]()
    if not ref_available(c.order, 3, full=True):
        pytest.skip("full-metric reference build absent (make -C oracle)")
    got = shock_b200.host_geometry(c, full_metric=True)
    ref = RefSolver(c, full=True).geometry()
    assert got.shape == ref.shape
    assert np.array_equal(got, ref)
    # the cross terms are there, and the diagonal form zeroes exactly them
    g = c.ghosts
    sl = (slice(g, g + c.ni), slice(g, g + c.nj), slice(g, g + c.nk))
    cross = [5, 6, 7, 9, 10, 11]   # xi_y xi_z eta_x eta_z zeta_x zeta_y
    assert min(np.abs(got[k][sl]).max() for k in cross) > 1e-3
    diag = shock_b200.host_geometry(c)
    assert not any(diag[k][sl].any() for k in cross)


def test_full_metric_rejections():
    """The full metric is a 3D FP64 form: the static entry point refuses it
    in the mixed form before it touches a device (the pointers are host
    buffers that are never read)."""
    import ctypes as C
    c = cases.taylor_green(8, order=5)
    p = shock_b200.params_from_case(c, precision=shock_b200.SHOCK_MIXED, full_metric=True)
    buf = np.zeros(16)
    ptr = buf.ctypes.data_as(C.c_void_p)
    assert shock_b200.lib().shock_rhs_static(C.byref(p), ptr, ptr, ptr, None) == shock_b200.SHOCK_EINVAL
    assert b"full_metric" in shock_b200.lib().shock_last_error()
