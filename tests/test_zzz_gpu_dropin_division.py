"""The drop-in binding's division mode end to end on a GPU: SHOCK's own
multi-rank set-up of a division on forked ranks, then GPU_Create,
GPU_CalcRungeKutta + GPU_CheckNAN and GPU_SyncHost of
shock_b200/dropin/GPU.c, rank 0 running every rank's block on its device
(oracle/_ref/libshockdropinmpireal_*), against SHOCK's own multi-rank run
of the same division on the CPU: 1e-10 relative L2 per variable after the
steps, on every rank's U_RK as GPU_SyncHost hands it back.  (Named to run
after the other GPU tests.)"""
import numpy as np
import pytest

from _util import l2_rel
from refbind import dropin_multirank_available, multirank_available, run_dropin_multirank, run_multirank
from test_dropin_division import DIVISIONS
from test_gpu_multiblock import _assemble

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["tgv12_w5_2x2x2", "smooth2d_w5_2x2_rotated", "channel3d_w5_walls_2x2x1"])
def test_dropin_division_on_gpu(name):
    d = DIVISIONS[name]()
    case = d.case
    if not dropin_multirank_available(case.order, case.dim, real=True) or not multirank_available(case.order,
                                                                                                 case.dim):
        pytest.skip("drop-in multi-rank builds absent (make -C oracle with the reference sources)")
    nsteps = 10
    res, _, _ = run_dropin_multirank(d, nsteps, real=True)
    ref = run_multirank(d, nsteps)
    got = _assemble(d, [r["after_steps"][:5] for r in res])
    want = _assemble(d, [r["state"][:5] for r in ref])
    idx = [0, 1, 2, 3, 4] if case.dim == 3 else [0, 1, 2, 4]
    e = l2_rel(got, want)[idx]
    assert (e <= 1e-10).all(), (name, e)
    assert all(r["nan_steps"] == 0 for r in res)


def test_dropin_division_histories_on_gpu():
    """The division mode's device probe histories over the library on rank
    0's GPU against the same loop with SHOCK's own steps and writers on
    every rank: the same flagged points on the same ranks, values within
    1e-12 of SHOCK's, the same times."""
    from refbind import run_dropin_multirank_histories
    d = DIVISIONS["tgv12_w5_2x2x2"]()
    c = d.case
    if not dropin_multirank_available(c.order, c.dim, real=True):
        pytest.skip("drop-in multi-rank builds absent (make -C oracle with the reference sources)")
    rng = np.random.default_rng(5)
    lo = np.array([c.x.min(), c.y.min(), c.z.min()])
    hi = np.array([c.x.max(), c.y.max(), c.z.max()])
    np_, nv, nsteps = 4, 3, 6
    xyz = lo + 0.05 * (hi - lo) + rng.random((np_ + nv, 3)) * 0.9 * (hi - lo)
    got = run_dropin_multirank_histories(d, np_, nv, xyz, nsteps, real=True)
    want = run_dropin_multirank_histories(d, np_, nv, xyz, nsteps, real=True, cpu=True)
    for b in range(len(d.blocks)):
        o = 0
        for q in range(np_ + nv):
            width = nsteps if q < np_ else 3 * nsteps
            assert got[b, o] == want[b, o] and got[b, o + 1] == want[b, o + 1], (b, q)
            a, r = got[b, o + 2:o + 2 + width], want[b, o + 2:o + 2 + width]
            scale = max(np.abs(r).max(), 1e-300)
            assert np.abs(a - r).max() <= 1e-12 * scale, (b, q)
            o += 2 + width
        assert np.array_equal(got[b, o:], want[b, o:])


def test_dropin_division_film_on_gpu():
    """The division mode's device Film over the library on rank 0's GPU
    against the same loop with SHOCK's own steps, CalcValuesForPost and
    WriteValuesFromUToFilm on every rank: frames within 1e-12 (lambda2
    1e-9), a re-taken sample in its place, the same times."""
    from _util import rel_err
    from refbind import run_dropin_multirank_film
    d = DIVISIONS["tgv12_w5_2x2x2"]()
    c = d.case
    if not dropin_multirank_available(c.order, c.dim, real=True):
        pytest.skip("drop-in multi-rank builds absent (make -C oracle with the reference sources)")
    nsamples, again = 4, 3
    got = run_dropin_multirank_film(d, nsamples, again, real=True)
    want = run_dropin_multirank_film(d, nsamples, again, real=True, cpu=True)
    for b in range(len(d.blocks)):
        nr = d.blocks[b].real_points
        fg = got[b][:8 * nsamples * nr].reshape(8, nsamples, nr)
        fw = want[b][:8 * nsamples * nr].reshape(8, nsamples, nr)
        for s in range(nsamples):
            err = rel_err(fg[:, s], fw[:, s])
            assert (err[:7] <= 1e-12).all(), (b, s, err)
            assert err[7] <= 1e-9, (b, s, err)
        assert np.array_equal(got[b][8 * nsamples * nr:], want[b][8 * nsamples * nr:])
