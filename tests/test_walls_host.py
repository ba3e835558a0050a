"""Wall and farfield faces on the host (no GPU): the block geometry built by
the library (ghost metric mirrored at wall and farfield faces,
src/Functions.c:6849-7015) against SHOCK's own set-up, bitwise; and the
argument checks of the boundary-condition field."""
import ctypes as C

import numpy as np
import pytest

import shock_b200
from refbind import RefSolver, ref_available
from shock_b200 import cases

CASES = [
    (3, 5, (16, 12, 14), "wall_viscous", 1.2, False),
    (3, 9, (14, 12, 14), "wall_inviscid", 0.0, False),
    (2, 5, (24, 20, 1), "farfield", 0.0, False),
    (2, 5, (20, 18, 1), "wall_viscous", 1.0, True),
    (3, 5, (16, 12, 14), "wall_isothermal", 1.2, False),
]


@pytest.mark.parametrize("inflow,walls,outflow", [("inflow_subsonic", "", "outflow_subsonic"),
                                                   ("inflow_supersonic", "wall_viscous", "outflow_subsonic"),
                                                   ("inflow_riemann", "", "outflow_riemann"),
                                                   ("inflow_isentropic", "wall_inviscid", "outflow_riemann")])
def test_duct_geometry_matches_reference(inflow, walls, outflow):
    if not ref_available(5, 2):
        pytest.skip("reference build not present")
    c = cases.duct(2, 5, (28, 18, 1), inflow=inflow, walls=walls, outflow=outflow)
    assert np.array_equal(shock_b200.host_geometry(c), RefSolver(c).geometry())


@pytest.mark.parametrize("face,bc", [(1, shock_b200.SHOCK_BC_INFLOW_SUPERSONIC),
                                     (1, shock_b200.SHOCK_BC_INFLOW_RIEMANN),
                                     (0, shock_b200.SHOCK_BC_OUTFLOW_RIEMANN)])
def test_mixed_inflow_outflow_options_rejected(face, bc):
    """SHOCK takes one inflow and one outflow option per run: a block with
    subsonic inflow on the x-lower face and subsonic outflow on the x-upper
    face cannot also carry another inflow or outflow kind."""
    c = cases.duct(2, 5, (28, 18, 1), walls="wall_viscous")
    p = shock_b200.params_from_case(c)
    p.bc[2 + face] = bc
    x, y, z = (np.ascontiguousarray(a.transpose(2, 1, 0)).ravel() for a in (c.x, c.y, c.z))
    out = np.zeros((13,) + (c.ni + 6, c.nj + 6, 1))
    dp = C.POINTER(C.c_double)
    rc = shock_b200.lib().shock_host_geometry(C.byref(p), x.ctypes.data_as(dp), y.ctypes.data_as(dp),
                                              z.ctypes.data_as(dp), out.ctypes.data_as(dp))
    assert rc == shock_b200.SHOCK_EINVAL
    p.bc[2 + face] = shock_b200.SHOCK_BC_WALL_VISCOUS
    assert shock_b200.lib().shock_host_geometry(C.byref(p), x.ctypes.data_as(dp), y.ctypes.data_as(dp),
                                                z.ctypes.data_as(dp), out.ctypes.data_as(dp)) == 0


def test_rudy_outflow_checks():
    """Rudy's outflow takes an inflow face on its own axis only (on another
    axis the inflow's set-up fill would give U_lastStep a speed of sound at
    the outflow's interior points) and needs L0, R, T0 for AlphaNonRef."""
    c = cases.duct(2, 5, (28, 18, 1), outflow="outflow_rudy", walls="wall_viscous")
    x, y, z = (np.ascontiguousarray(a.transpose(2, 1, 0)).ravel() for a in (c.x, c.y, c.z))
    out = np.zeros((13,) + (c.ni + 6, c.nj + 6, 1))
    dp = C.POINTER(C.c_double)

    def geom(p):
        return shock_b200.lib().shock_host_geometry(C.byref(p), x.ctypes.data_as(dp), y.ctypes.data_as(dp),
                                                    z.ctypes.data_as(dp), out.ctypes.data_as(dp))

    assert geom(shock_b200.params_from_case(c)) == 0
    p = shock_b200.params_from_case(c)
    p.bc[3] = shock_b200.SHOCK_BC_INFLOW_SUBSONIC
    assert geom(p) == shock_b200.SHOCK_EINVAL
    # Rudy faces on two axes: the x-lower inflow shares points with the y one
    p = shock_b200.params_from_case(c)
    p.bc[3] = shock_b200.SHOCK_BC_OUTFLOW_RUDY
    assert geom(p) == shock_b200.SHOCK_EINVAL
    p.bc[0] = shock_b200.SHOCK_BC_WALL_VISCOUS
    assert geom(p) == 0
    p = shock_b200.params_from_case(c)
    p.l0 = 0.0
    assert geom(p) == shock_b200.SHOCK_EINVAL


@pytest.mark.parametrize("dim,order,n,bc,stretch,walls_i", CASES)
def test_wall_geometry_matches_reference(dim, order, n, bc, stretch, walls_i):
    if not ref_available(order, dim):
        pytest.skip("reference build not present")
    c = cases.channel(dim, order, n, bc=bc, stretch=stretch, walls_i=walls_i)
    assert np.array_equal(shock_b200.host_geometry(c), RefSolver(c).geometry())


def test_bc_argument_checks():
    c = cases.channel(2, 5, (24, 20, 1), bc="wall_viscous")
    lib = shock_b200.lib()
    out = np.zeros((13,) + (c.ni + 6, c.nj + 6, 1))
    x, y, z = (np.ascontiguousarray(a.transpose(2, 1, 0)).ravel() for a in (c.x, c.y, c.z))
    dp = C.POINTER(C.c_double)

    def geom(p):
        return lib.shock_host_geometry(C.byref(p), x.ctypes.data_as(dp), y.ctypes.data_as(dp),
                                       z.ctypes.data_as(dp), out.ctypes.data_as(dp))

    ok = shock_b200.params_from_case(c)
    assert geom(ok) == 0
    bad = shock_b200.params_from_case(c)
    bad.bc[0] = 1                      # a wall on a periodic axis
    assert geom(bad) == shock_b200.SHOCK_EINVAL
    bad = shock_b200.params_from_case(c)
    bad.bc[2] = 12                     # unknown type
    assert geom(bad) == shock_b200.SHOCK_EINVAL
    bad = shock_b200.params_from_case(c)
    bad.bc[2] = 0                      # a non-periodic face with nothing to fill it
    assert geom(bad) == shock_b200.SHOCK_EINVAL
