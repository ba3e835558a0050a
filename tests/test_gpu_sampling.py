"""Sampling on the device: probes (SHOCK's pressure / velocity histories)
recorded by the step graph, and Film frames (CalcValuesForPost +
WriteValuesFromUToFilm) kept on the device, against SHOCK's own build
stepping the same block and reading U_lastStep after every step."""
import numpy as np
import pytest

import shock_b200
from _util import rel_err
from refbind import RefSolver, ref_available
from shock_b200 import cases

pytestmark = pytest.mark.gpu


def _need(c):
    if not ref_available(c.order, c.dim):
        pytest.skip("reference build absent")


@pytest.mark.parametrize("case", [
    cases.smooth_random(3, 5, (16, 14, 15), seed=7, stretch=0.05),
    cases.duct(2, 9, (28, 20, 1), inflow="inflow_riemann", outflow="outflow_rudy", walls="wall_viscous"),
], ids=lambda c: c.name)
def test_probe_history_matches_reference(case, parity):
    _need(case)
    g = case.ghosts
    pts = [(g, g, g if case.dim == 3 else 0), (g + 5, g + 3, g + 2 if case.dim == 3 else 0),
           (g + case.ni - 1, g + case.nj - 1, g + case.nk - 1 if case.dim == 3 else 0)]
    s = shock_b200.Solver(case)
    with pytest.raises(shock_b200.ShockError):
        s.set_probes([(g - 1, g, g if case.dim == 3 else 0)])     # SHOCK keeps probes on real points
    s.set_probes(pts, capacity=16)
    s.steps(6)
    hist = s.probe_history()

    def reference(extended):
        r = RefSolver(case, extended=extended)
        out = []
        for _ in range(6):
            r.steps(1)
            st = r.state(1)      # U_lastStep: rho,u,v,w,e,p,T,c,mue
            out.append([[st[5][p], st[1][p], st[2][p], st[3][p]] for p in pts])
        return np.array(out)

    ref = reference(False)
    assert hist.shape == ref.shape
    scale = np.abs(ref).max(axis=(0, 1))
    scale[scale == 0] = 1.0
    err = np.abs(hist - ref).max(axis=(0, 1)) / scale
    tol = np.full(4, 1e-12)
    if ref_available(case.order, case.dim, extended=True):
        # twice SHOCK's own FP64-vs-80-bit distance where that is larger (WENO9 ducts)
        tol = np.maximum(tol, 2.0 * np.abs(reference(True) - ref).max(axis=(0, 1)) / scale)
    parity("probes", case.name, "p,u,v,w history (6 steps)", err, tol)
    assert (err <= tol).all(), (err, tol)
    # the history was cleared, and a full history reports the lost steps
    assert s.probe_history().shape[0] == 0
    s.set_probes(pts[:1], capacity=2)
    s.steps(3)
    with pytest.raises(shock_b200.ShockError):
        s.probe_history()
    s.close()


def test_film_frames_match_reference(parity):
    case = cases.smooth_random(3, 5, (16, 14, 15), seed=7, stretch=0.05)
    _need(case)
    s = shock_b200.Solver(case)
    s.film_reserve(2)
    r = RefSolver(case)
    ref = []
    for n in (3, 2):
        s.steps(n)
        s.film_sample()
        r.steps(n)
        st, post = r.state(1), r.post()
        g = case.ghosts
        sl = (slice(g, g + case.ni), slice(g, g + case.nj), slice(g, g + case.nk))
        ref.append(np.stack([st[0][sl], st[1][sl], st[2][sl], st[3][sl], st[5][sl],
                             post[1][sl], post[0][sl], post[2][sl]]))
    film = s.film()
    with pytest.raises(shock_b200.ShockError):
        s.film_sample()          # full
    s.close()
    assert film.shape[0] == 2
    for f in range(2):
        err = rel_err(film[f], ref[f])
        parity("film", case.name, f"frame {f} (rho,u,v,w,p,|grad rho|,Ma,l2)", err, [1e-12] * 7 + [1e-9])
        assert (err[:7] <= 1e-12).all(), err
        assert err[7] <= 1e-9, err      # lambda2: libm vs CUDA cube-root trigonometry
