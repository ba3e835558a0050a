"""Divisions (blocks of one zone, SHOCK's .sddc layout) on the host: the
geometry set-up with the interfaces exchanged (shock_host_multi_geometry)
against SHOCK's own multi-rank run of the same division (oracle/_ref/
libshockmpi_*: SHOCK's TransferMeshParameter between ranks over the forked
shared-memory stand-in for MPI), bit for bit on every ghosted point of
every block; and the division bookkeeping."""
import numpy as np
import pytest

import shock_b200
from refbind import multirank_available, run_multirank
from shock_b200 import cases

DIVISIONS = {
    "tgv16_w5_2x2x2": lambda: (cases.taylor_green(16, order=5), (2, 2, 2)),
    "smooth2d_w5_2x2": lambda: (cases.smooth_random(2, 5, (24, 20, 1), seed=4, stretch=0.08), (2, 2, 1)),
    "smooth3d_w9_uneven_2x1x2": lambda: (cases.smooth_random(3, 9, (21, 12, 23), seed=6, stretch=0.05), (2, 1, 2)),
    "channel3d_w5_walls_2x2x1": lambda: (cases.channel(3, 5, (16, 14, 12)), (2, 2, 1)),
}


@pytest.mark.parametrize("name", sorted(DIVISIONS))
def test_division_geometry_matches_shock_multirank(name):
    case, parts = DIVISIONS[name]()
    if not multirank_available(case.order, case.dim):
        pytest.skip("multi-rank reference build absent (make -C oracle with the reference sources)")
    d = cases.split(case, parts)
    got = shock_b200.host_multi_geometry(d)
    ref = run_multirank(d, 0)
    for b in range(len(d.blocks)):
        assert np.array_equal(got[b], ref[b]["geometry"]), (name, b)


def test_split_bookkeeping():
    c = cases.taylor_green(16, order=5)
    d = cases.split(c, (2, 2, 2))
    assert len(d.blocks) == 8 and sum(b.real_points for b in d.blocks) == c.real_points
    for b in range(8):
        for f in range(6):
            nb = d.neighbour[b, f]
            assert d.neighbour[nb, f ^ 1] == b
    # the periodic wraps carry the period, interior faces nothing
    assert d.translation[0, 0, 0] == np.float32(-c.period[0]) and d.translation[0, 1, 0] == 0.0
    ch = cases.channel(3, 5, (16, 14, 12))
    dc = cases.split(ch, (1, 2, 1))
    assert dc.neighbour[0, 2] == -1 and dc.blocks[0].bc[2] == ch.bc[2]
    assert dc.neighbour[0, 3] == 1 and dc.blocks[0].bc[3] == 0
