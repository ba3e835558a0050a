"""Probe placement on the host: the points shock_locate_probes picks for
PressureHistory / VelocityHistory locations against the points SHOCK's own
preparePressureHistoryValues picks on the same block (oracle/_ref, after
SHOCK's set-up, ghost coordinates included): the same point for every
probe, and the same verdict on whether the block records it (a location
nearest to a ghost point belongs to another block).  Locations inside and
around the block, on grid points and halfway between two of them."""
import numpy as np
import pytest

import shock_b200
from refbind import RefSolver, ref_available
from shock_b200 import cases

CASES = {
    "periodic_3d_w5": lambda: cases.smooth_random(3, 5, (12, 10, 9), seed=2, stretch=0.06),
    "channel_2d_w9": lambda: cases.channel(2, 9, (16, 14, 1), stretch=1.5),
    "walled_box_3d_w5": lambda: cases.channel(3, 5, (10, 12, 8), walls_i=True, stretch=1.1),
}


def _locations(case, rng, n=60):
    x, y, z = case.x, case.y, case.z
    lo = np.array([x.min(), y.min(), z.min()])
    hi = np.array([x.max(), y.max(), z.max()])
    pad = 0.25 * (hi - lo)
    pts = [lo - pad + rng.random(3) * (hi - lo + 2 * pad) for _ in range(n)]
    flat = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    for o in rng.integers(0, len(flat) - 1, size=10):
        pts.append(flat[o])                                    # on a grid point
        pts.append(0.5 * (flat[o] + flat[o + 1]))               # halfway to the next one
    out = np.array(pts)
    if case.dim == 2:
        out[:, 2] = 0.0
    return out


@pytest.mark.parametrize("name", sorted(CASES))
def test_probe_points_as_shock_places_them(name):
    case = CASES[name]()
    if not ref_available(case.order, case.dim):
        pytest.skip("reference build absent (make -C oracle with the reference sources)")
    ref = RefSolver(case)
    geom = shock_b200.host_geometry(case)
    assert np.array_equal(geom, ref.geometry())
    xyz = _locations(case, np.random.default_rng(7))
    ijk3, found = shock_b200.locate_probes(case, geom, xyz)
    r_ijk, r_flag = ref.probe_points(xyz)
    shape = geom.shape[1:]
    linear = np.where(ijk3[:, 0] >= 0, (ijk3[:, 0] * shape[1] + ijk3[:, 1]) * shape[2] + ijk3[:, 2], -1)
    assert np.array_equal(found, r_flag.astype(bool)), name
    assert np.array_equal(linear, r_ijk), name
    assert found.any() and not found.all()
