"""Blocks of a division on one GPU (shock_multi_*) against SHOCK's own
multi-rank run of the same division (oracle/_ref/libshockmpi_*: one
process per block, SHOCK's TransferMeshParameter and
TransferFlowParameterWithGhosts between them).

SHOCK's results depend on the division itself, not only on the whole
block: its zeta viscous stencil is centred on the block-local j index
(src/ZD.c:547-548), so a 3D viscous run split differently gives different
numbers.  The device reproduces that, block by block, so it is compared
with the reference run of the same division.  Divisions with zones meshed
in other orientations (.sddc Transforms other than 1,2,3; blocks re-indexed
by cases.rotate_block) check the transformed exchange; a 3D block with
permuted axes needs the full metric, so those run against SHOCK's
full-metric multi-rank build.  Tolerances as in the
single-block parity tests: per variable, 1e-12 normwise for one RHS and
1e-10 relative L2 after the steps, or twice SHOCK's own FP64-vs-80-bit
distance on the same division where that is larger (the Mach 0.1
Taylor-Green vortex and WENO9 are ill-conditioned)."""
import numpy as np
import pytest

import shock_b200
from _util import l2_rel, rel_err
from refbind import multirank_available, run_multirank
from shock_b200 import cases

pytestmark = pytest.mark.gpu

DIVISIONS = {
    # name: (case, parts, steps)
    "tgv16_w5_2x2x2": lambda: (cases.taylor_green(16, order=5), (2, 2, 2), 100),
    "smooth2d_w5_2x2": lambda: (cases.smooth_random(2, 5, (24, 20, 1), seed=4, stretch=0.08), (2, 2, 1), 20),
    "smooth2d_w9_3x2": lambda: (cases.smooth_random(2, 9, (33, 24, 1), seed=5), (3, 2, 1), 20),
    "smooth3d_w9_uneven_2x1x2": lambda: (cases.smooth_random(3, 9, (21, 10, 23), seed=6, stretch=0.05), (2, 1, 2), 10),
    "channel3d_w5_walls_2x2x1": lambda: (cases.channel(3, 5, (16, 14, 12)), (2, 2, 1), 20),
    "tgv16_w5_inviscid_rk3_2x2x2": lambda: (cases.taylor_green(16, order=5).replace(inviscid=True, time_order=3),
                                            (2, 2, 2), 20),
    # zones meshed in other orientations (.sddc Transforms other than 1,2,3):
    # (block, its new axes in terms of its old ones, which run reversed), all
    # proper rotations; 3D blocks with permuted axes take the full metric
    # (their metric is in the cross terms the reference mode zeroes)
    "tgv16_w5_2x2x1_rotated_full": lambda: (cases.taylor_green(16, order=5), (2, 2, 1), 20,
                                            [(1, (1, 0, 2), (True, False, False)),
                                             (3, (0, 1, 2), (True, True, False))], True),
    "smooth2d_w5_2x2_rotated": lambda: (cases.smooth_random(2, 5, (24, 20, 1), seed=4, stretch=0.08), (2, 2, 1), 20,
                                        [(2, (1, 0, 2), (False, True, False))]),
    "smooth3d_w9_2x1x2_rotated_full": lambda: (cases.smooth_random(3, 9, (21, 10, 23), seed=6, stretch=0.05),
                                               (2, 1, 2), 10, [(3, (1, 0, 2), (False, False, True))], True),
    "channel3d_w5_walls_2x2x1_rotated": lambda: (cases.channel(3, 5, (16, 14, 12)), (2, 2, 1), 20,
                                                 [(0, (0, 1, 2), (True, True, False))]),
}


def division(name):
    """(case, division, steps, full metric) of a named division, its rotated
    blocks applied."""
    case, parts, nsteps, *more = DIVISIONS[name]()
    rot = more[0] if more else []
    full = more[1] if len(more) > 1 else False
    d = cases.split(case, parts)
    for b, axes, flips in rot:
        d = cases.rotate_block(d, b, axes, flips)
    return case, d, nsteps, full


def _real(case, block, a):
    g = case.ghosts
    if case.dim == 3:
        return a[..., g:g + block.ni, g:g + block.nj, g:g + block.nk]
    return a[..., g:g + block.ni, g:g + block.nj, :]


def _assemble(d, per_block):
    c = d.case
    out = np.zeros((per_block[0].shape[0], c.ni, c.nj, c.nk if c.dim == 3 else 1))
    for b, a in enumerate(per_block):
        lo = d.lo[b]
        r = d.from_block(b, _real(c, d.blocks[b], a))
        out[:, lo[0]:lo[0] + r.shape[1], lo[1]:lo[1] + r.shape[2], lo[2]:lo[2] + r.shape[3]] = r
    return out


@pytest.mark.parametrize("name", sorted(DIVISIONS))
def test_division_matches_shock_multirank(name, parity):
    case, d, nsteps, full = division(name)
    if not multirank_available(case.order, case.dim, full=full):
        pytest.skip("multi-rank reference build absent (make -C oracle with the reference sources)")
    ref = run_multirank(d, nsteps, rhs=True, full=full)
    ref80 = run_multirank(d, nsteps, rhs=True, extended=True, full=full) \
        if multirank_available(case.order, case.dim, True, full=full) else None
    m = shock_b200.Multi(d, full_metric=full)
    try:
        for b in range(len(d.blocks)):
            assert np.array_equal(m.geometry(b), ref[b]["geometry"]), b
        q = _assemble(d, [m.rhs(b) for b in range(len(d.blocks))])
        m.steps(nsteps)
        st = _assemble(d, [m.state(b) for b in range(len(d.blocks))])
    finally:
        m.close()
    qr = _assemble(d, [r["rhs"] for r in ref])
    sr = _assemble(d, [r["state"][:5] for r in ref])
    idx = [0, 1, 2, 3, 4] if case.dim == 3 else [0, 1, 2, 4]
    tol_rhs, tol_l2 = np.full(len(idx), 1e-12), np.full(len(idx), 1e-10)
    floor = None
    if ref80 is not None:
        floor = rel_err(qr, _assemble(d, [r["rhs"] for r in ref80]))[idx]
        tol_rhs = np.maximum(tol_rhs, 2.0 * floor)
        tol_l2 = np.maximum(tol_l2, 2.0 * l2_rel(sr, _assemble(d, [r["state"][:5] for r in ref80]))[idx])
    e_rhs = rel_err(q, qr)[idx]
    parity("division", f"{name}", "rhs vs SHOCK multi-rank", e_rhs, tol_rhs, floor)
    assert (e_rhs <= tol_rhs).all(), (e_rhs, tol_rhs)
    e = l2_rel(st, sr)[idx]
    parity("division", f"{name}", f"{nsteps} steps L2 vs SHOCK multi-rank", e, tol_l2)
    assert (e <= tol_l2).all(), (e, tol_l2)


def test_division_inviscid_equals_single_block():
    """Without viscous terms the division changes nothing but where the
    ghost layers come from: the whole block solved as 2x2x2 blocks and as one
    periodic block agree to rounding."""
    c = cases.taylor_green(16, order=5).replace(inviscid=True)
    d = cases.split(c, (2, 2, 2))
    m = shock_b200.Multi(d)
    s = shock_b200.Solver(c)
    m.steps(10)
    s.steps(10)
    st = _assemble(d, [m.state(b) for b in range(8)])
    m.close()
    single = s.real(s.state())
    assert (rel_err(st, single) <= 1e-13).all(), rel_err(st, single)


def test_division_runtime_tau_and_nan():
    """shock_multi_set_tau takes effect on every block (the steps with half the
    time step differ from full ones), and the NaN scan covers every block."""
    c = cases.taylor_green(16, order=5)
    d = cases.split(c, (2, 2, 1))
    a, b = shock_b200.Multi(d), shock_b200.Multi(d)
    b.set_tau(c.tau / 2)
    a.steps(2)
    b.steps(4)
    sa = _assemble(d, [a.state(k) for k in range(4)])
    sb = _assemble(d, [b.state(k) for k in range(4)])
    assert 0 < l2_rel(sb, sa).max() < 1e-3   # same time reached, different steps
    import ctypes as C
    bad = C.c_int()
    assert a.lib.shock_multi_check_nan(a.h, C.byref(bad)) == 0 and bad.value == 0
    a.close()
    b.close()
