"""GPU (sm_100a kernels through the C ABI) against SHOCK's results.

Tolerances (FP64 form), normwise per variable (max|a-b| / max|b| over the
real points):
  * one right-hand side within max(1e-12, 2*floor) of SHOCK's FP64 build and
    of its 80-bit build, where floor = distance between SHOCK's FP64 and
    80-bit results on the same case (its own rounding error; about 5e-15 on
    well-conditioned cases, up to 1e-11 at Mach 0.1 or with WENO9);
  * the state after 100 full RK4 steps within 1e-10 relative L2.
The GPU contracts multiply-adds into FMAs, so agreement is not bitwise.
"""
import numpy as np
import pytest

import shock_b200
from _util import golden_names, l2_rel, load_golden, real, rel_err
from refbind import Oracle, RefSolver, ref_available
from shock_b200 import cases

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-12
L2_TOL_100 = 1e-10


def _solver(case, d=None, **kw):
    d = d or {}
    return shock_b200.Solver(case, dirichlet9=d.get("dirichlet9"), source5=d.get("source5"), **kw)


def _tol(a64, a80):
    """max(1e-12, 2 * SHOCK's own FP64-vs-80-bit distance), per variable."""
    return np.maximum(RHS_TOL, 2.0 * rel_err(a64, a80))


@pytest.mark.parametrize("name", golden_names())
def test_rhs_matches_reference_golden(name, parity):
    """One RHS against SHOCK's FP64 and 80-bit builds.  Where SHOCK's own
    FP64-vs-80-bit distance is below 5e-13 the bound is 1e-12 against the
    FP64 build; on the ill-conditioned cases (Mach 0.1 Taylor-Green, WENO9)
    it is twice that distance, i.e. the GPU must be as close to the 80-bit
    answer as SHOCK's own FP64 build is."""
    case, d = load_golden(name)
    s = _solver(case, d)
    q = real(case, s.rhs())
    ref, ref80 = real(case, d["rhs"]), real(case, d["rhs80"])
    if case.mms != "none":
        scale = np.abs(real(case, d["source5"])).max()
        err = np.abs(q - ref).max() / scale
        parity(name, case.name, "rhs vs SHOCK FP64 (|JS|)", err, RHS_TOL)
        assert err <= RHS_TOL, err
    else:
        floor = rel_err(ref, ref80)
        tol = _tol(ref, ref80)
        parity(name, case.name, "rhs vs SHOCK FP64", rel_err(q, ref), tol, floor)
        parity(name, case.name, "rhs vs SHOCK 80-bit", rel_err(q, ref80), tol, floor)
        assert (tol[floor < 5e-13] == RHS_TOL).all()
        assert (rel_err(q, ref) <= tol).all(), (rel_err(q, ref), tol)
        assert (rel_err(q, ref80) <= tol).all(), (rel_err(q, ref80), tol)


@pytest.mark.parametrize("name", golden_names())
def test_steps_match_reference_golden(name, parity):
    case, d = load_golden(name)
    s = _solver(case, d)
    s.steps(int(d["nsteps"]))
    st = real(case, s.state())
    ref, ref80 = real(case, d["state"]), real(case, d["state80"])
    tol = _tol(ref, ref80)
    parity(name, case.name, f"{int(d['nsteps'])} steps vs SHOCK FP64", rel_err(st, ref), tol, rel_err(ref, ref80))
    assert (rel_err(st, ref) <= tol).all(), (rel_err(st, ref), tol)


@pytest.mark.parametrize("dim,order,inviscid,n", [
    (2, 5, False, (64, 64, 1)), (2, 9, False, (40, 36, 1)), (3, 5, False, (24, 20, 22)),
    (3, 9, False, (20, 18, 18)), (3, 5, True, (17, 19, 23)), (2, 5, True, (13, 17, 1)),
])
def test_rhs_matches_oracle_sizes(dim, order, inviscid, n, parity):
    """Ragged and odd sizes (tile remainders along every axis)."""
    c = cases.smooth_random(dim, order, n, seed=5, inviscid=inviscid, stretch=0.08)
    o = Oracle(c)
    s = _solver(c)
    assert np.array_equal(s.geometry(), o.geometry())
    q64 = real(c, o.rhs())      # the oracle is bitwise SHOCK's FP64 result
    floor = None
    if ref_available(order, dim, extended=True):
        q80 = real(c, RefSolver(c, extended=True).rhs())
        floor = rel_err(q64, q80)
        tol = _tol(q64, q80)
    else:
        tol = np.full(5, 5e-11 if order == 9 else RHS_TOL)
    err = rel_err(real(c, s.rhs()), q64)
    parity("oracle_sizes", c.name, "rhs vs SHOCK FP64", err, tol, floor)
    assert (err <= tol).all(), (err, tol)


def test_tgv_100_steps_l2(parity):
    """Curvilinear Taylor-Green (perturbed grid), 100 RK4 steps vs the oracle."""
    c = cases.taylor_green(16, order=5)
    o = Oracle(c)
    s = _solver(c)
    o.steps(100)
    s.steps(100)
    err = l2_rel(real(c, s.state()), real(c, o.state()[:5]))
    parity("tgv16", c.name, "100 steps L2 vs oracle", err, L2_TOL_100)
    assert (err <= L2_TOL_100).all(), err


def test_tgv64_100_steps_vs_shock(parity):
    """The second configuration at its stated size: 3D curvilinear
    Taylor-Green vortex, 64^3 periodic points on the perturbed grid, Ma 0.1,
    Re 1600, WENO5, viscous, RK4 at CFL 0.5, all FP64: 100 steps against
    SHOCK's own CPU build (oracle/_ref, a few minutes on one core)."""
    if not ref_available(5, 3):
        pytest.skip("reference build absent")
    c = cases.taylor_green(64, order=5)
    r = RefSolver(c)
    s = _solver(c)
    s.steps(100)
    r.steps(100)
    st, ref = real(c, s.state()), real(c, r.state()[:5])
    err = l2_rel(st, ref)
    # w is the state variable SHOCK advances; its L2 is judged against |u|
    # where the flow keeps it small (the initial w is zero)
    err[3] = np.sqrt(np.mean((st[3] - ref[3]) ** 2)) / np.sqrt(np.mean(ref[1] ** 2))
    parity("tgv64", c.name, "100 steps L2 vs SHOCK FP64", err, L2_TOL_100)
    assert (err <= L2_TOL_100).all(), err


def test_mms_100_steps_l2(parity):
    """2D manufactured solution on the unit square (64^2, WENO5, viscous), 100
    steps, SHOCK's own manufactured family (src/ManufacturedSolution.c)."""
    c = cases.mms_square(64, 5, family="reference", mms_case=0)
    if ref_available(5, 2):
        r = RefSolver(c)
        dir9, src = r.mms_exact(), r.mms_source()
    else:
        pytest.skip("reference build not present for 64^2 manufactured data")
    o = Oracle(c, dirichlet9=dir9, source5=src)
    s = _solver(c, {"dirichlet9": dir9, "source5": src})
    o.steps(100)
    s.steps(100)
    err = l2_rel(real(c, s.state()), real(c, o.state()[:5]))
    parity("mms64_reference", c.name, "100 steps L2 vs oracle", err[[0, 1, 2, 4]], L2_TOL_100)
    assert (err <= L2_TOL_100).all(), err


def test_mms_product_form_64_100_steps_vs_shock(parity):
    """The first configuration at its stated size: the product-form
    manufactured solution (rho = 1+0.1 sin 2pi x sin 2pi y, ...) on the 64^2
    unit square, gamma 1.4, Re 100, Pr 0.72, WENO5 + central viscous, RK4 at
    CFL 0.5, 100 steps, all FP64, against SHOCK's own build run with the same
    exact solution and source (ref_harness/mms_external.c in place of
    ManufacturedSolution.c)."""
    if not ref_available(5, 2):
        pytest.skip("reference build absent")
    c = cases.mms_square(64, 5, family="baseline")
    ex, js = shock_b200.host_mms_baseline(c)
    r = RefSolver(c, external=(ex, js))
    s = _solver(c, {"dirichlet9": ex, "source5": js})
    r.steps(100)
    s.steps(100)
    st, ref = real(c, s.state()), real(c, r.state()[:5])
    err = l2_rel(st, ref)[[0, 1, 2, 4]]
    parity("mms64_product", c.name, "100 steps L2 vs SHOCK FP64", err, L2_TOL_100)
    assert (err <= L2_TOL_100).all(), err
    # and the solution stays at the manufactured one (a steady state)
    assert (l2_rel(st, real(c, ex[:5]))[[0, 1, 2, 4]] < 1e-3).all()


def test_rk3_and_w9_steps():
    c = cases.smooth_random(3, 9, (16, 14, 15), seed=9, time_order=3)
    o = Oracle(c)
    s = _solver(c)
    o.steps(10)
    s.steps(10)
    err = l2_rel(real(c, s.state()), real(c, o.state()[:5]))
    assert (err <= 1e-11).all(), err


def test_deterministic():
    c = cases.smooth_random(3, 5, (20, 18, 19), seed=3)
    a = _solver(c)
    b = _solver(c)
    a.steps(5)
    b.steps(5)
    assert np.array_equal(a.state(), b.state())


def test_nan_flag():
    """Fault injected on the host: a NaN density in the uploaded state."""
    c = cases.smooth_random(2, 5, (16, 16, 1), seed=1)
    s = _solver(c)
    st = s.state()
    g = c.ghosts
    st[0, g + 3, g + 4, 0] = np.nan
    s.set_state(st)
    assert s.check_nan() == 1


def _conserved_l2(a, b):
    from _util import conserved
    return l2_rel(conserved(a), conserved(b))


@pytest.mark.parametrize("order,n,nsteps", [(5, 64, 200), (9, 24, 40)])
def test_mixed_precision_l2(order, n, nsteps, parity):
    """Mixed form (FP32 stencils, FP64 state) vs the FP64 form on the
    curvilinear Taylor-Green vortex: relative L2 per conserved variable.  The
    WENO5 case is the second configuration at its stated size and length
    (64^3, 200 steps)."""
    c = cases.taylor_green(n, order=order)
    a = _solver(c)
    b = _solver(c, precision=shock_b200.SHOCK_MIXED)
    a.steps(nsteps)
    b.steps(nsteps)
    sa, sb = real(c, a.state()), real(c, b.state())
    err = _conserved_l2(sb, sa)
    # rho*w is identically zero for this flow; measure it against |rho u|
    scale = np.sqrt(np.mean((sa[0] * sa[1]) ** 2))
    err[3] = np.sqrt(np.mean((sb[0] * sb[3] - sa[0] * sa[3]) ** 2)) / scale
    parity("mixed_tgv", c.name, f"mixed vs FP64 L2, {nsteps} steps", err, 1e-6)
    assert (err <= 1e-6).all(), err


@pytest.mark.parametrize("order", [5, 9])
def test_mixed_precision_l2_2d_vortex(order, parity):
    """Mixed vs FP64 on the 2D isentropic vortex, whose far field is nearly
    uniform: the FP32 smoothness indicators there are at their smallest."""
    c = cases.isentropic_vortex(48, 3.0, 0.5, order=order, inviscid=False, reynolds=2000.0)
    a = _solver(c)
    b = _solver(c, precision=shock_b200.SHOCK_MIXED)
    a.steps(40)
    b.steps(40)
    sa, sb = real(c, a.state()), real(c, b.state())
    assert np.isfinite(sb).all()
    err = _conserved_l2(sb, sa)
    parity("mixed_vortex", c.name, "mixed vs FP64 L2, 40 steps", err[[0, 1, 2, 4]], 1e-6)
    assert (err[[0, 1, 2, 4]] <= 1e-6).all(), err


def _truncation_l2(case, solver_rhs, J):
    q = real(case, solver_rhs)
    return np.array([np.sqrt(np.mean((q[k] / J) ** 2)) for k in (0, 1, 2, 4)])


@pytest.mark.parametrize("order,sizes,min_order,weno_eps", [
    (5, (16, 32), 3.5, 0.0), (9, (32, 64), 8.0, 0.0),          # reference mode (SHOCK's epsilon)
    (5, (16, 32, 64), 5.0, 1e-6), (9, (16, 32, 64), 8.4, 1e-6),  # clean mode
])
def test_mms_design_order(order, sizes, min_order, weno_eps, parity):
    """Manufactured-solution mode: the right-hand side at the exact solution
    (the truncation error of dU/dt) on the product-form 2D solution shrinks
    at the scheme's order, and the GPU reproduces the oracle's truncation
    errors.  Reference mode keeps SHOCK's WENO epsilon 10*sqrt(DBL_MIN)
    (src/Functions.c:1829): WENO-JS then loses order at smooth extrema, about
    4 for WENO5 on coarse grids falling towards 3 on fine ones, as SHOCK's own
    build does.  Clean mode (weno_eps = 1e-6, the value src/Functions.c:1818
    leaves commented out) restores the design order: at least 5 with WENO5
    (6 once the sixth-order viscous stencils dominate) and about 8.5-10.7 with
    WENO9 over 16 -> 32 -> 64 points."""
    errs_gpu, errs_ref = [], []
    for n in sizes:
        c = cases.mms_square(n, order, family="baseline")
        s = _solver(c, weno_eps=weno_eps)     # built-in exact solution and source
        ex, js = s.mms_baseline()
        o = Oracle(c, dirichlet9=ex, source5=js, weno_eps=weno_eps)
        J = real(c, s.geometry()[3])
        errs_gpu.append(_truncation_l2(c, s.rhs(), J))
        errs_ref.append(_truncation_l2(c, o.rhs(), J))
    p_gpu = np.array([np.log2(errs_gpu[i] / errs_gpu[i + 1]) for i in range(len(sizes) - 1)])
    p_ref = np.array([np.log2(errs_ref[i] / errs_ref[i + 1]) for i in range(len(sizes) - 1)])
    mode = "clean" if weno_eps else "reference"
    parity("design_order", f"mms_baseline_w{order} {mode}", "observed order (min)", p_gpu.min(), min_order)
    assert (p_gpu >= min_order).all(), p_gpu
    assert np.abs(p_gpu - p_ref).max() < 0.02, (p_gpu, p_ref)


@pytest.mark.parametrize("case", [
    cases.smooth_random(3, 5, (16, 14, 15), seed=7, stretch=0.05),
    cases.smooth_random(3, 9, (14, 12, 16), seed=8),
    cases.isentropic_vortex(32, 3.0, 0.5),
], ids=lambda c: c.name)
def test_post_matches_reference(case):
    """Device post-processing (Mach number, |grad rho|, lambda2) against
    SHOCK's own CalcValuesForPost on U_lastStep after two steps.  lambda2
    comes from the trigonometric roots of a cubic, whose libm and CUDA values
    differ in the last bits, so it is compared at 1e-9 of its maximum."""
    r = RefSolver(case)
    r.steps(2)
    ref = real(case, r.post())
    s = _solver(case)
    s.steps(2)
    got = real(case, s.post())
    err = rel_err(got, ref)
    assert err[0] <= RHS_TOL and err[1] <= RHS_TOL, err
    assert err[2] <= 1e-9, err
