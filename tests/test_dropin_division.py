"""The drop-in binding's division mode on CPU: shock_b200/dropin/GPU.c with
several ranks, inside SHOCK's own multi-rank set-up (forked ranks over the
shared-memory MPI stand-in), over a host test double of the library
(oracle/ref_harness/mock_shock.c) that hands the division rank 0 assembles
to the real library's host set-up.  Checked: the block each rank describes
(sizes, the rank across each face, Transform, Translation, face types) sets
up, in the library, SHOCK's own geometry of that block bit for bit; every
rank's U_RK after GPU_SyncHost is its own block's device state; GPU_UploadState
moves every rank's state to its block; time steps changed by SHOCK's loop
reach the device; GPU_CheckNAN reports a non-finite density in any block on
every rank.  The device path itself (shock_multi_* on a B200) is covered by
the division tests of the library; this file covers the binding's MPI
plumbing."""
import numpy as np
import pytest

from refbind import dropin_multirank_available, run_dropin_multirank
from shock_b200 import cases

DIVISIONS = {
    "tgv12_w5_2x2x2": lambda: cases.split(cases.taylor_green(12, order=5), (2, 2, 2)),
    "channel3d_w5_walls_2x2x1": lambda: cases.split(cases.channel(3, 5, (16, 14, 12)), (2, 2, 1)),
    "smooth2d_w5_2x2_rotated": lambda: cases.rotate_block(
        cases.split(cases.smooth_random(2, 5, (24, 20, 1), seed=4, stretch=0.08), (2, 2, 1)), 2, (1, 0, 2),
        (False, True, False)),
    "cgrid2d_w5_4x2": lambda: cases.wake_cut(cases.split(cases.parabolic_cgrid(2, 5, (24, 12, 1), seed=3), (4, 2, 1))),
}


def _available(d):
    return dropin_multirank_available(d.case.order, d.case.dim)


@pytest.mark.parametrize("name", sorted(DIVISIONS))
def test_dropin_division_mode(name):
    d = DIVISIONS[name]()
    if not _available(d):
        pytest.skip("drop-in multi-rank harness absent (make -C oracle with the reference sources)")
    nsteps = 4
    res, steps, taus = run_dropin_multirank(d, nsteps, tau_at=2, tau_factor=0.5)
    assert steps == nsteps + 1
    assert len(taus) == 2 and taus[1] == taus[0] * 0.5
    for b, r in enumerate(res):
        # the binding's description of the block sets up SHOCK's geometry
        assert np.array_equal(r["library_geometry"], r["shock_geometry"]), (name, b)
        # every rank reads back its own block's state: the double adds
        # (block + 1) * 1e-3 to the density per step and sets p
        rho = r["initial"][0].copy()
        for _ in range(nsteps):
            rho = rho + 1e-3 * (b + 1)
        assert np.array_equal(r["after_steps"][0], rho), (name, b)
        assert np.array_equal(r["after_steps"][1:5], r["initial"][1:5]), (name, b)
        assert (r["after_steps"][5] == 2.0 + b + 0.5 * nsteps).all(), (name, b)
        # GPU_UploadState took each rank's changed state to its block
        rho2 = (r["after_steps"][0] + 0.25 * (b + 1)) + 1e-3 * (b + 1)
        assert np.array_equal(r["after_upload_step"][0], rho2), (name, b)
        assert (r["after_upload_step"][5] == 2.0 + b + 0.5 * (nsteps + 1)).all(), (name, b)
        assert r["nan_steps"] == 0


def test_dropin_division_nan_on_every_rank():
    d = DIVISIONS["tgv12_w5_2x2x2"]()
    if not _available(d):
        pytest.skip("drop-in multi-rank harness absent (make -C oracle with the reference sources)")
    nsteps, at = 5, 3
    res, _, _ = run_dropin_multirank(d, nsteps, nan=(at, 6))
    # from the step that planted it, every rank's GPU_CheckNAN reports it
    assert [r["nan_steps"] for r in res] == [nsteps - at + 1] * len(res)
    # block 6's rank brought its state to the host and SHOCK's own checkNAN
    # marked the point (1e6, src/Functions.c:5443); the others stay finite
    assert (res[6]["after_steps"][0] == 1e6).sum() == 1
    assert all(np.isfinite(r["after_steps"][0]).all() for r in res)
