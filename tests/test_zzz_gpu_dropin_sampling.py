"""The drop-in binding's device probe histories and Film end to end on a
GPU: SHOCK's set-up and loop order with the binding over the library
(GPU_EnableHistories / GPU_WriteValuesFor*History, GPU_EnableFilm /
GPU_SampleFilm / GPU_SyncFilm; oracle/_ref/libshockdropin_*) against the
same loop with SHOCK's own CalcRungeKutta, WriteValuesFor*History,
CalcValuesForPost and WriteValuesFromUToFilm (oracle/_ref/libshockref_*):
the same flagged points, histories within 1e-12 of SHOCK's per variable,
Film frames within 1e-12 (lambda2 1e-9: libm and CUDA differ in the
cubic's trigonometric roots), a sample taken again after a reset in its
place.  (Named to run after the other GPU tests.)"""
import ctypes as C

import numpy as np
import pytest

from _util import rel_err
from refbind import RefSolver, ref_available
from shock_b200 import cases

pytestmark = pytest.mark.gpu

CASES = {
    "smooth3d_w5": lambda: cases.smooth_random(3, 5, (16, 14, 15), seed=7, stretch=0.05),
    "duct2d_w9_rudy": lambda: cases.duct(2, 9, (28, 20, 1), inflow="inflow_riemann", outflow="outflow_rudy",
                                         walls="wall_viscous"),
}
DP = C.POINTER(C.c_double)


def _solvers(case):
    if not ref_available(case.order, case.dim):
        pytest.skip("reference build absent")
    try:
        return RefSolver(case), RefSolver(case, _lib="libshockdropin")
    except FileNotFoundError:
        pytest.skip("drop-in harness absent (make -C oracle with the reference sources)")


@pytest.mark.parametrize("name", sorted(CASES))
def test_dropin_histories_on_gpu(name):
    case = CASES[name]()
    rng = np.random.default_rng(3)
    lo = np.array([case.x.min(), case.y.min(), case.z.min()])
    hi = np.array([case.x.max(), case.y.max(), case.z.max()])
    np_, nv, nsteps = 4, 3, 6
    xyz = np.ascontiguousarray(lo + rng.random((np_ + nv, 3)) * (hi - lo))
    if case.dim == 2:
        xyz[:, 2] = 0.0
    n = np_ * (2 + nsteps) + nv * (2 + 3 * nsteps) + nsteps
    out_cpu, out_gpu = np.zeros(n), np.zeros(n)
    cpu, gpu = _solvers(case)
    assert cpu.lib.ref_histories(np_, nv, xyz.ctypes.data_as(DP), nsteps, out_cpu.ctypes.data_as(DP)) == 0
    rc = gpu.lib.ref_dropin_histories(np_, nv, xyz.ctypes.data_as(DP), nsteps, 0, out_gpu.ctypes.data_as(DP))
    assert rc == 0
    o = 0
    for q in range(np_ + nv):
        width = nsteps if q < np_ else 3 * nsteps
        assert out_gpu[o] == out_cpu[o] and out_gpu[o + 1] == out_cpu[o + 1], (name, q)   # same point, same flag
        a, b = out_gpu[o + 2:o + 2 + width], out_cpu[o + 2:o + 2 + width]
        scale = max(np.abs(b).max(), 1e-300)
        assert np.abs(a - b).max() <= 1e-12 * scale, (name, q, np.abs(a - b).max() / scale)
        o += 2 + width
    assert np.array_equal(out_gpu[o:], out_cpu[o:])


@pytest.mark.parametrize("name", sorted(CASES))
def test_dropin_film_on_gpu(name):
    case = CASES[name]()
    nsamples, again = 4, 3
    nr = case.real_points
    out_cpu, out_gpu = np.zeros(8 * nsamples * nr + nsamples), np.zeros(8 * nsamples * nr + nsamples)
    cpu, gpu = _solvers(case)
    assert cpu.lib.ref_film(nsamples, again, out_cpu.ctypes.data_as(DP)) == 0
    assert gpu.lib.ref_dropin_film(nsamples, again, 0, out_gpu.ctypes.data_as(DP)) == 0
    f_cpu = out_cpu[:8 * nsamples * nr].reshape(8, nsamples, nr)
    f_gpu = out_gpu[:8 * nsamples * nr].reshape(8, nsamples, nr)
    for s in range(nsamples):
        err = rel_err(f_gpu[:, s], f_cpu[:, s])
        assert (err[:7] <= 1e-12).all(), (name, s, err)
        assert err[7] <= 1e-9, (name, s, err)
    assert np.array_equal(out_gpu[8 * nsamples * nr:], out_cpu[8 * nsamples * nr:])
