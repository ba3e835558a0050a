"""Serving loop (shock_server_*): continuous batching inside an HBM budget.

Each request's result must be the same alone and in a mix (bitwise: a
request runs the same kernels with its class's fixed launch configuration
whatever else is on the device), FP64 requests must agree with a solo
shock_ctx solve at the one-RHS parity tolerance, and requests that do not
fit in the budget together are admitted in arrival order as memory frees.
"""
import time

import numpy as np
import pytest

import shock_b200
from _util import real, reference_floor, rel_err
from shock_b200 import cases

pytestmark = pytest.mark.gpu

FP64, MIXED = shock_b200.SHOCK_FP64, shock_b200.SHOCK_MIXED




def _err(a, b):
    """Normwise relative error per variable; velocity components relative to
    the largest velocity component (w of a vortex column is rounding noise
    around zero, so max|w| is no scale)."""
    err = rel_err(a, b)
    vs = max(np.abs(b[k]).max() for k in (1, 2, 3))
    for k in (1, 2, 3):
        err[k] = np.abs(a[k] - b[k]).max() / vs
    return err


def _mix():
    return [
        (cases.isentropic_vortex(48, 3.0, 0.5), 7, FP64),
        (cases.smooth_random(2, 9, (40, 36, 1), seed=11), 4, FP64),
        (cases.taylor_green(16, order=5, perturb=0.0, reynolds=800.0), 5, FP64),
        (cases.isentropic_vortex(40, 2.0, 0.3, order=9, inviscid=False, reynolds=2000.0), 4, FP64),
        (cases.taylor_green_2d(64, 5, 0.3, 500.0), 6, MIXED),
        (cases.vortex_column(20, 20, 4.0, 0.6, order=5, reynolds=3000.0), 3, FP64),
        (cases.isentropic_vortex(32, 1.5, 0.7), 9, FP64),
    ]


def _run(server, reqs, gap=0.0):
    ids = []
    for case, n, prec in reqs:
        ids.append(server.submit(case, n, prec))
        if gap:
            time.sleep(gap)
    out = []
    for rid in ids:
        server.wait(rid, 120.0)
        out.append(server.result(rid))
    return out


def test_serve_result_same_alone_and_in_mix():
    reqs = _mix()
    srv = shock_b200.Server(hbm_budget=2 << 30)
    mixed = _run(srv, reqs, gap=0.002)
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    for (case, n, prec), (state, info) in zip(reqs, mixed):
        assert info["status"] == 0 and info["done_s"] >= info["admit_s"] >= info["submit_s"]
        alone = shock_b200.Server(hbm_budget=1 << 30)
        (a_state, _), = _run(alone, [(case, n, prec)])
        alone.close()
        assert np.array_equal(real(case, state), real(case, a_state)), case.name
        if prec == FP64:
            s = shock_b200.Solver(case)
            s.steps(n)
            err = _err(real(case, state), real(case, s.state()))
            s.close()
            # 1e-12, or twice SHOCK's own FP64-vs-80-bit distance where the
            # case is ill-conditioned (the WENO9 vortex's nearly uniform far
            # field makes its smoothness indicators so)
            floor = reference_floor(case, n)
            tol = 1e-12 if floor is None else np.maximum(1e-12, 2.0 * floor)
            assert (err <= tol).all(), (case.name, err, tol)


def test_serve_admits_within_budget_in_arrival_order():
    reqs = [(cases.isentropic_vortex(64, 1.0 + i, 0.4), 5 + i, FP64) for i in range(5)]
    srv = shock_b200.Server(hbm_budget=64 << 20, max_requests=2)
    res = _run(srv, reqs)
    st = srv.stats()
    srv.close()
    assert st["completed"] == 5
    admits = [info["admit_s"] for _, info in res]
    assert admits == sorted(admits)
    # at most two on the device at once: the third waits for a finish
    dones = sorted(info["done_s"] for _, info in res)
    assert admits[2] >= dones[0] - 1e-6


def test_serve_rejects_request_larger_than_budget():
    srv = shock_b200.Server(hbm_budget=64 << 20)
    big = cases.taylor_green(64, order=5)
    with pytest.raises(shock_b200.ShockError) as e:
        srv.submit(big, 1)
    assert e.value.code == -2
    srv.close()
