"""Divisions (blocks of one zone, SHOCK's .sddc layout) on the host: the
geometry set-up with the interfaces exchanged (shock_host_multi_geometry)
against SHOCK's own multi-rank run of the same division (oracle/_ref/
libshockmpi_*: SHOCK's TransferMeshParameter between ranks over the forked
shared-memory stand-in for MPI), bit for bit on every ghosted point of
every block, also for divisions whose zones are meshed in other
orientations (.sddc Transforms other than 1,2,3); and the division
bookkeeping; and C-grids whose wake cut joins mirrored blocks bottom to
bottom."""
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
    # zones meshed in other orientations (.sddc Transforms other than 1,2,3):
    # (block, its new axes in terms of its old ones, which run reversed), all
    # proper rotations.  A 3D block with permuted axes has its metric in the
    # cross terms, so those divisions take the full metric (SHOCK's
    # full-metric multi-rank build); reversed axes alone keep the diagonal one.
    "tgv16_w5_2x2x1_rotated_full": lambda: (cases.taylor_green(16, order=5), (2, 2, 1),
                                            [(1, (1, 0, 2), (True, False, False)), (3, (0, 1, 2), (True, True, False))],
                                            True),
    "tgv12_w5_2x2x2_rotated_all_full": lambda: (cases.taylor_green(12, order=5), (2, 2, 2), [
        (b, ((1, 0, 2), (2, 0, 1), (0, 2, 1), (1, 2, 0))[b % 4],
         ((1, 0, 0), (1, 1, 0), (0, 0, 1), (0, 0, 0), (0, 1, 0), (0, 1, 1), (1, 1, 1), (1, 0, 1))[b])
        for b in range(8)], True),
    "smooth2d_w5_2x2_rotated": lambda: (cases.smooth_random(2, 5, (24, 20, 1), seed=4, stretch=0.08), (2, 2, 1),
                                        [(2, (1, 0, 2), (False, True, False)), (1, (0, 1, 2), (True, True, False))]),
    "channel3d_w5_walls_2x2x1_rotated": lambda: (cases.channel(3, 5, (16, 14, 12)), (2, 2, 1),
                                                 [(0, (0, 1, 2), (True, True, False))]),
}


def division(name):
    """(case, division, full metric) of a named division, its rotated blocks applied."""
    case, parts, *more = DIVISIONS[name]()
    rot = more[0] if more else []
    full = more[1] if len(more) > 1 else False
    d = cases.split(case, parts)
    for b, axes, flips in rot:
        d = cases.rotate_block(d, b, axes, [bool(x) for x in flips])
    return case, d, full


@pytest.mark.parametrize("name", sorted(DIVISIONS))
def test_division_geometry_matches_shock_multirank(name):
    case, d, full = division(name)
    if not multirank_available(case.order, case.dim, full=full):
        pytest.skip("multi-rank reference build absent (make -C oracle with the reference sources)")
    got = shock_b200.host_multi_geometry(d, full_metric=full)
    ref = run_multirank(d, 0, full=full)
    for b in range(len(d.blocks)):
        assert np.array_equal(got[b], ref[b]["geometry"]), (name, b)


# C-grids (cases.parabolic_cgrid) divided with their wake cut (cases.wake_cut):
# the bottom faces of mirrored blocks joined with Transform (-1,-2,3), the
# topology of SHOCK's own division generator; (dim, order, points, parts,
# full metric -- 3D C-grids have their metric in the cross terms)
CGRIDS = {
    "cgrid2d_w5_4x2": (2, 5, (24, 12, 1), (4, 2, 1), False),
    "cgrid2d_w9_2x1": (2, 9, (20, 14, 1), (2, 1, 1), False),
    "cgrid3d_w5_4x2x2_full": (3, 5, (16, 10, 12), (4, 2, 2), True),
}


def cgrid_division(name):
    dim, order, n, parts, full = CGRIDS[name]
    case = cases.parabolic_cgrid(dim, order, n, seed=3)
    return case, cases.wake_cut(cases.split(case, parts)), full


@pytest.mark.parametrize("name", sorted(CGRIDS))
def test_cgrid_geometry_matches_shock_multirank(name):
    case, d, full = cgrid_division(name)
    if not multirank_available(case.order, case.dim, full=full):
        pytest.skip("multi-rank reference build absent (make -C oracle with the reference sources)")
    got = shock_b200.host_multi_geometry(d, full_metric=full)
    ref = run_multirank(d, 0, full=full)
    for b in range(len(d.blocks)):
        assert np.array_equal(got[b], ref[b]["geometry"]), (name, b)


def test_wake_cut_bookkeeping():
    """Across the cut i runs the other way and both sides are bottom faces:
    the ghost row below block b's j = 0 is its mirror block's row j = 0,
    point for point (x(xi, -eta) = x(-xi, eta) in parabolic coordinates)."""
    case, d, _ = cgrid_division("cgrid2d_w5_4x2")
    for b in range(4):
        m = 3 - b
        assert d.neighbour[b, 2] == m and d.neighbour[m, 2] == b
        assert tuple(d.transform[b, 2]) == (-1, -2, 3)
    xi = -1.5 + (np.arange(24) + 0.5) * (3.0 / 24)
    eta0 = 0.5 * 1.2 / 12
    ghost_x = 0.5 * (xi ** 2 - eta0 ** 2)
    assert np.array_equal(ghost_x, case.x[::-1, 0, 0])
    with pytest.raises(ValueError):
        cases.wake_cut(cases.split(cases.parabolic_cgrid(2, 5, (25, 12, 1)), (2, 1, 1)))


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


def test_rotated_division_bookkeeping():
    """cases.rotate_block re-indexes a block's fields and faces; every
    interface is then named from both sides with inverse Transforms, and
    turning the block back gives the original division."""
    c = cases.taylor_green(12, order=5)
    d0 = cases.split(c, (2, 2, 1))
    d = cases.rotate_block(d0, 1, (1, 0, 2), (True, False, False))
    assert d.blocks[1].ni == d0.blocks[1].nj and d.blocks[1].nj == d0.blocks[1].ni
    assert np.array_equal(d.to_block(1, np.stack([c.x, c.y])), np.stack([d.blocks[1].x, d.blocks[1].y]))
    assert np.array_equal(d.from_block(1, d.blocks[1].u[None]), d0.blocks[1].u[None])
    for b in range(4):
        for f in range(6):
            n = d.neighbour[b, f]
            if n < 0:
                continue
            t = d.transform[b, f]
            a, hi = f // 2, f % 2
            fd = 2 * (abs(t[a]) - 1) + (hi ^ int(t[a] > 0))
            assert d.neighbour[n, fd] == b
            back = d.transform[n, fd]
            for ax in range(3):
                assert back[abs(t[ax]) - 1] == np.sign(t[ax]) * (ax + 1)
    # turning block 1 back: new axis c runs along old axis (1,0,2)[c]; undo with the inverse
    d2 = cases.rotate_block(d, 1, (1, 0, 2), (False, True, False))
    assert np.array_equal(d2.blocks[1].x, d0.blocks[1].x) and np.array_equal(d2.transform, d0.transform)


def test_inconsistent_transforms_rejected():
    """An interface whose two sides do not carry inverse Transforms, or a
    Transform that is not a signed permutation, is refused (SHOCK_EINVAL)."""
    c = cases.taylor_green(12, order=5)
    d = cases.rotate_block(cases.split(c, (2, 2, 1)), 1, (1, 0, 2), (True, False, False))
    bad = cases.Division(case=d.case, parts=d.parts, blocks=d.blocks, neighbour=d.neighbour,
                         translation=d.translation, lo=d.lo, transform=d.transform.copy(), axes=d.axes,
                         flips=d.flips)
    bad.transform[0, 0] = [2, 1, 3]   # block 0's left face: not the inverse of what block 1 holds
    with pytest.raises(shock_b200.ShockError):
        shock_b200.host_multi_geometry(bad)
    bad.transform[0, 0] = [2, 2, 3]   # not a permutation
    with pytest.raises(shock_b200.ShockError):
        shock_b200.host_multi_geometry(bad)
