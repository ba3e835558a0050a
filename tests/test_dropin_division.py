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


# One rank: the block GPU_Create describes to shock_create from SHOCK's
# set-up (its BC names and config.ini options, its periodic interfaces, its
# parameters), over the same test double.
SINGLE = {
    "tgv16_w5_periodic": lambda: cases.taylor_green(16, order=5),
    "channel3d_w5_viscous_walls": lambda: cases.channel(3, 5, (12, 10, 12)),
    "channel2d_w9_isothermal": lambda: cases.channel(2, 9, (16, 14, 1), bc="wall_isothermal", t_wall=1.3),
    "channel2d_w5_slip_box": lambda: cases.channel(2, 5, (16, 14, 1), bc="wall_inviscid", walls_i=True),
    "channel2d_w5_farfield": lambda: cases.channel(2, 5, (16, 14, 1), bc="farfield"),
    "duct2d_w5_riemann_rudy": lambda: cases.duct(2, 5, (20, 12, 1), inflow="inflow_riemann", outflow="outflow_rudy",
                                                 walls="wall_viscous"),
    "duct2d_w9_isentropic_riemann": lambda: cases.duct(2, 9, (20, 14, 1), inflow="inflow_isentropic",
                                                       outflow="outflow_riemann"),
    "duct3d_w5_supersonic_subsonic": lambda: cases.duct(3, 5, (14, 10, 10), inflow="inflow_supersonic",
                                                        outflow="outflow_subsonic", mach=1.5),
}


@pytest.mark.parametrize("name", sorted(SINGLE))
def test_dropin_single_block_description(name):
    import ctypes as C

    import shock_b200
    from refbind import RefSolver
    case = SINGLE[name]()
    try:
        ref = RefSolver(case, _lib="libshockdropinmock")
    except FileNotFoundError:
        pytest.skip("drop-in test double build absent (make -C oracle with the reference sources)")
    assert ref.lib.ref_dropin_create(0) == 0
    p = shock_b200.Params()
    assert ref.lib.mock_params(C.byref(p)) == 0
    ref.lib.ref_dropin_destroy()
    want = shock_b200.params_from_case(case)
    for k in ("dim", "order", "ni", "nj", "nk", "time_order", "tau", "mach", "reynolds", "prandtl", "gamma", "gas_r",
              "t0", "l0", "inviscid", "mms", "t_wall", "rho_inflow", "p_inflow", "p_outflow"):
        assert getattr(p, k) == getattr(want, k), (name, k, getattr(p, k), getattr(want, k))
    assert list(p.bc) == list(want.bc), (name, list(p.bc), list(want.bc))
    assert list(p.periodic) == list(want.periodic), name
    # the period travels as the float32 Translation of the .sddc row
    assert [p.period[a] for a in range(3) if want.periodic[a]] == \
        [float(np.float32(want.period[a])) for a in range(3) if want.periodic[a]], name
    assert list(p.u_inflow) == list(want.u_inflow), name


@pytest.mark.parametrize("name", ["tgv16_w5_periodic", "channel2d_w9_isothermal"])
def test_dropin_probe_histories(name):
    """GPU_EnableHistories registers the points SHOCK's own
    prepare*HistoryValues chose (flagged ones only), and the binding's
    writers put the last step's device values of each point (U_lastStep's p,
    u, v, w) and time_dim at the current iteration of SHOCK's history arrays
    (over the test double, whose values name the point and the step)."""
    import ctypes as C

    from refbind import RefSolver
    case = SINGLE[name]()
    try:
        ref = RefSolver(case, _lib="libshockdropinmock")
    except FileNotFoundError:
        pytest.skip("drop-in test double build absent (make -C oracle with the reference sources)")
    rng = np.random.default_rng(11)
    lo = np.array([case.x.min(), case.y.min(), case.z.min()])
    hi = np.array([case.x.max(), case.y.max(), case.z.max()])
    np_, nv, nsteps = 5, 4, 6
    xyz = lo - 0.2 * (hi - lo) + rng.random((np_ + nv, 3)) * 1.4 * (hi - lo)
    if case.dim == 2:
        xyz[:, 2] = 0.0
    xyz = np.ascontiguousarray(xyz)
    out = np.zeros(np_ * (2 + nsteps) + nv * (2 + 3 * nsteps) + nsteps)
    dp = C.POINTER(C.c_double)
    assert ref.lib.ref_dropin_histories(np_, nv, xyz.ctypes.data_as(dp), nsteps, 0, out.ctypes.data_as(dp)) == 0
    val = ref.lib.mock_probe_value
    val.restype = C.c_double
    o, flagged = 0, 0
    for q in range(np_):
        ijk, flag, hist = int(out[o]), int(out[o + 1]), out[o + 2:o + 2 + nsteps]
        o += 2 + nsteps
        want = [val(0, C.c_longlong(ijk), s) if flag else 0.0 for s in range(1, nsteps + 1)]
        assert list(hist) == want, (name, q)
        flagged += flag
    for q in range(nv):
        ijk, flag = int(out[o]), int(out[o + 1])
        for f in range(3):
            hist = out[o + 2 + f * nsteps:o + 2 + (f + 1) * nsteps]
            want = [val(1 + f, C.c_longlong(ijk), s) if flag else 0.0 for s in range(1, nsteps + 1)]
            assert list(hist) == want, (name, q, f)
        o += 2 + 3 * nsteps
        flagged += flag
    # time_dim, advanced by tau after every step
    assert np.allclose(out[o:o + nsteps], [case.tau * s for s in range(1, nsteps + 1)], rtol=1e-14, atol=0)
    assert 0 < flagged < np_ + nv


@pytest.mark.parametrize("name", ["tgv16_w5_periodic", "duct2d_w9_isentropic_riemann"])
def test_dropin_film(name):
    """GPU_SampleFilm takes each sample on the device and GPU_SyncFilm puts
    every frame at its sample's place in SHOCK's Film arrays, a sample taken
    again after a NaN reset overwriting the earlier one; the sample times are
    SHOCK's time_dim at each sample (over the test double, whose frames name
    the frame, the field and the point)."""
    import ctypes as C

    from refbind import RefSolver
    case = SINGLE[name]()
    try:
        ref = RefSolver(case, _lib="libshockdropinmock")
    except FileNotFoundError:
        pytest.skip("drop-in test double build absent (make -C oracle with the reference sources)")
    nsamples, again = 4, 3
    nr = case.real_points
    out = np.zeros(8 * nsamples * nr + nsamples)
    dp = C.POINTER(C.c_double)
    assert ref.lib.ref_dropin_film(nsamples, again, 0, out.ctypes.data_as(dp)) == 0
    val = ref.lib.mock_film_value
    val.restype = C.c_double
    frame_of = [0, 1, 3, 4]               # sample 2 taken again by frame 3
    t = np.arange(nr)
    for q in range(8):
        film = out[q * nsamples * nr:(q + 1) * nsamples * nr].reshape(nsamples, nr)
        for s, f in enumerate(frame_of):
            want = 10.0 * q + 0.001 * f + 1e-7 * t
            assert np.array_equal(film[s], want), (name, q, s)
            assert val(f, q, C.c_longlong(5)) == want[5]
    times = out[8 * nsamples * nr:]
    assert np.allclose(times, [case.tau * (f + 1) for f in frame_of], rtol=1e-14, atol=0)


def test_dropin_division_histories():
    """In the division mode GPU_EnableHistories sends every rank's flagged
    probe points to its block on rank 0, and the writers give every rank the
    last step's device values of its own points (over the test double, whose
    values name the block, the point and the step); each location inside
    the zone is some rank's, and only that rank's, probe."""
    from refbind import mock_div_probe_value, run_dropin_multirank_histories
    d = DIVISIONS["tgv12_w5_2x2x2"]()
    if not _available(d):
        pytest.skip("drop-in multi-rank harness absent (make -C oracle with the reference sources)")
    c = d.case
    rng = np.random.default_rng(5)
    lo = np.array([c.x.min(), c.y.min(), c.z.min()])
    hi = np.array([c.x.max(), c.y.max(), c.z.max()])
    np_, nv, nsteps = 5, 4, 5
    xyz = lo + 0.05 * (hi - lo) + rng.random((np_ + nv, 3)) * 0.9 * (hi - lo)
    out = run_dropin_multirank_histories(d, np_, nv, xyz, nsteps)
    owners = np.zeros(np_ + nv, dtype=int)
    for b in range(len(d.blocks)):
        o = 0
        for q in range(np_ + nv):
            width = nsteps if q < np_ else 3 * nsteps
            ijk, flag, hist = int(out[b, o]), int(out[b, o + 1]), out[b, o + 2:o + 2 + width]
            owners[q] += flag
            if q < np_:
                want = [mock_div_probe_value(b, 0, ijk, s) if flag else 0.0 for s in range(1, nsteps + 1)]
            else:
                want = [mock_div_probe_value(b, f, ijk, s) if flag else 0.0
                        for f in (1, 2, 3) for s in range(1, nsteps + 1)]
            assert list(hist) == want, (b, q)
            o += 2 + width
        assert np.allclose(out[b, o:], [c.tau * s for s in range(1, nsteps + 1)], rtol=1e-14, atol=0)
    assert (owners == 1).all(), owners


def test_dropin_division_film():
    """In the division mode GPU_SampleFilm has rank 0 take every block's
    frame and GPU_SyncFilm sends every rank its own block's frames, each at
    its sample's place (a re-taken sample overwriting its frame), over the
    test double whose frames name the block, the frame, the field and the
    point."""
    from refbind import run_dropin_multirank_film
    d = DIVISIONS["tgv12_w5_2x2x2"]()
    if not _available(d):
        pytest.skip("drop-in multi-rank harness absent (make -C oracle with the reference sources)")
    nsamples, again = 4, 3
    res = run_dropin_multirank_film(d, nsamples, again)
    frame_of = [0, 1, 3, 4]
    for b, r in enumerate(res):
        nr = d.blocks[b].real_points
        film = r[:8 * nsamples * nr].reshape(8, nsamples, nr)
        t = np.arange(nr)
        for q in range(8):
            for s, f in enumerate(frame_of):
                want = 1000.0 * b + 10.0 * q + 0.001 * f + 1e-7 * t
                assert np.array_equal(film[q, s], want), (b, q, s)
        assert np.allclose(r[8 * nsamples * nr:], [d.case.tau * (f + 1) for f in frame_of], rtol=1e-14, atol=0)
