"""C-grid divisions with their wake cut on the device (shock_multi_*):
geometry bit for bit, one right-hand side and 10 steps against SHOCK's own
multi-rank run of the same division, as the other divisions are checked
(1e-12 per right-hand side, 1e-10 relative L2 after the steps, or twice
SHOCK's own FP64-vs-80-bit distance where that is larger).  (Named to
run after the other GPU tests.)"""
import numpy as np
import pytest

import shock_b200
from _util import l2_rel, rel_err
from refbind import multirank_available, run_multirank
from test_gpu_multiblock import _assemble
from test_multiblock_host import CGRIDS, cgrid_division

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(CGRIDS))
def test_cgrid_division_on_gpu(name):
    case, d, full = cgrid_division(name)
    if not multirank_available(case.order, case.dim, full=full):
        pytest.skip("multi-rank reference build absent (make -C oracle with the reference sources)")
    nsteps = 10
    ref = run_multirank(d, nsteps, rhs=True, full=full)
    m = shock_b200.Multi(d, full_metric=full)
    try:
        for b in range(len(d.blocks)):
            assert np.array_equal(m.geometry(b), ref[b]["geometry"]), (name, b)
        q = _assemble(d, [m.rhs(b) for b in range(len(d.blocks))])
        m.steps(nsteps)
        st = _assemble(d, [m.state(b) for b in range(len(d.blocks))])
    finally:
        m.close()
    idx = [0, 1, 2, 3, 4] if case.dim == 3 else [0, 1, 2, 4]
    qr = _assemble(d, [r["rhs"] for r in ref])
    sr = _assemble(d, [r["state"][:5] for r in ref])
    tol_rhs, tol_l2 = np.full(len(idx), 1e-12), np.full(len(idx), 1e-10)
    # where SHOCK's own FP64 build is further than that from its 80-bit
    # build, twice that distance (as for the other divisions)
    if multirank_available(case.order, case.dim, True, full=full):
        ref80 = run_multirank(d, nsteps, rhs=True, extended=True, full=full)
        tol_rhs = np.maximum(tol_rhs, 2.0 * rel_err(qr, _assemble(d, [r["rhs"] for r in ref80]))[idx])
        tol_l2 = np.maximum(tol_l2, 2.0 * l2_rel(sr, _assemble(d, [r["state"][:5] for r in ref80]))[idx])
    e_rhs = rel_err(q, qr)[idx]
    assert (e_rhs <= tol_rhs).all(), (name, e_rhs, tol_rhs)
    e = l2_rel(st, sr)[idx]
    assert (e <= tol_l2).all(), (name, e, tol_l2)
