"""shock_rhs_static (the entry point that allocates nothing) against shock_rhs.

Both run the same stage kernels on the same geometry and state, so the
right-hand sides must agree within the one-RHS tolerance of the parity
tests (they are in fact expected to be identical).  Two different blocks
are evaluated back to back, so the second call runs on scratch that the
first call left behind.  The file is named to be collected last: it must
pass in a fresh process and after every other test.
"""
import ctypes as C

import numpy as np
import pytest

import shock_b200
from _util import real, rel_err
from shock_b200 import cases

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-12
SHOCK_EINVAL = -1


def _fn():
    f = shock_b200.lib().shock_rhs_static
    f.restype = C.c_int
    f.argtypes = [C.POINTER(shock_b200.Params), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return f


def _static_rhs(case, state, precision):
    """RHS through shock_rhs_static on device copies of geometry and state."""
    import torch

    p = shock_b200.params_from_case(case, precision)
    geom = torch.from_numpy(shock_b200.host_geometry(case)).cuda()
    st = torch.from_numpy(np.ascontiguousarray(state)).cuda()
    q = torch.zeros_like(st)
    stream = torch.cuda.current_stream().cuda_stream
    rc = _fn()(C.byref(p), geom.data_ptr(), st.data_ptr(), q.data_ptr(), stream)
    assert rc == 0, shock_b200.lib().shock_last_error().decode()
    torch.cuda.synchronize()
    return q.cpu().numpy()


def _check(case, precision):
    s = shock_b200.Solver(case, precision=precision)
    state = s.state()
    ref = real(case, s.rhs())
    s.close()
    got = real(case, _static_rhs(case, state, precision))
    err = rel_err(got, ref)
    assert (err <= RHS_TOL).all(), err


def test_static_rhs_matches_context_rhs_twice():
    a = cases.taylor_green(n=16, order=5)
    b = cases.smooth_random(2, 9, (24, 20, 1), seed=7)
    _check(a, shock_b200.SHOCK_FP64)
    _check(b, shock_b200.SHOCK_MIXED)


def test_static_rhs_rejects_large_block():
    import torch

    case = cases.taylor_green(n=80, order=5)   # 86^3 ghosted points > 524288
    p = shock_b200.params_from_case(case)
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    rc = _fn()(C.byref(p), buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), None)
    assert rc == SHOCK_EINVAL
    assert "at most 524288" in shock_b200.lib().shock_last_error().decode()
