"""The CPU restatement (oracle/shock_oracle.c) against SHOCK's own code.

The fixtures in tests/golden/ were produced by the reference translation
units themselves (tests/golden/make_golden.py, oracle/_ref).  The
restatement keeps the reference's operation order, so geometry, one
right-hand side and the state after full RK steps must agree bit for bit
on the periodic cases.  On the manufactured-solution cases the reference
adds the long-double source in extended precision, so Q agrees to one
rounding of the source term.
"""
import numpy as np
import pytest

from _util import golden_names, load_golden, real
from refbind import Oracle, RefSolver, ref_available
from shock_b200 import cases


@pytest.mark.parametrize("name", golden_names())
def test_oracle_matches_golden(name):
    case, d = load_golden(name)
    mms = case.mms != "none"
    o = Oracle(case, dirichlet9=d.get("dirichlet9"), source5=d.get("source5"))
    geo = o.geometry()
    assert np.array_equal(geo, d["geometry"]), "geometry differs from SHOCK's set-up"
    q = o.rhs()
    if mms:
        scale = np.abs(d["source5"]).max()
        assert np.abs(q - d["rhs"]).max() <= 4e-16 * scale
    else:
        assert np.array_equal(q, d["rhs"]), "right-hand side is not bitwise equal"
    o.steps(int(d["nsteps"]))
    st = o.state()[:5]
    if mms:
        assert np.abs(real(case, st - d["state"])).max() <= 1e-14 * np.abs(d["state"]).max()
    else:
        assert np.array_equal(real(case, st), real(case, d["state"]))


@pytest.mark.skipif(not ref_available(5, 3), reason="oracle/_ref not built in this tree")
@pytest.mark.parametrize("seed", [21, 22])
def test_oracle_matches_reference_live(seed):
    """Fresh random cases straight against the reference build, when present."""
    rng = np.random.default_rng(seed)
    dim = int(rng.integers(2, 4))
    order = int(rng.choice([5, 9]))
    n = tuple(int(x) for x in rng.integers(10, 14, size=3))
    n = (n[0], min(n[1], n[2]), max(n[1], n[2]))
    c = cases.smooth_random(dim, order, n, seed=seed, stretch=0.05,
                            inviscid=bool(rng.integers(0, 2)), time_order=int(rng.choice([3, 4])))
    r = RefSolver(c)
    o = Oracle(c)
    assert np.array_equal(o.rhs(), r.rhs())
    r.steps(2)
    o.steps(2)
    assert np.array_equal(o.state()[:5], r.state()[:5])
