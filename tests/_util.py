"""Shared helpers for the test suite: golden fixtures and error norms."""
import glob
import os

import numpy as np

from shock_b200 import cases

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name):
    d = dict(np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False))
    c = cases.Case(dim=int(d["dim"]), order=int(d["order"]), ni=int(d["ni"]), nj=int(d["nj"]),
                   nk=int(d["nk"]), x=d["in_x"], y=d["in_y"], z=d["in_z"], rho=d["in_rho"],
                   u=d["in_u"], v=d["in_v"], w=d["in_w"], p=d["in_p"],
                   time_order=int(d["time_order"]), tau=float(d["tau"]), mach=float(d["mach"]),
                   reynolds=float(d["reynolds"]), prandtl=float(d["prandtl"]),
                   gamma=float(d["gamma"]), gas_r=float(d["gas_r"]), t0=float(d["t0"]),
                   l0=float(d["l0"]), inviscid=bool(d["inviscid"]), mms=str(d["mms"]),
                   mms_case=int(d["mms_case"]), periodic=tuple(bool(x) for x in d["periodic"]),
                   period=tuple(float(x) for x in d["period"]), name=name)
    return c, d


def real(case, a, g=None):
    g = case.ghosts if g is None else g
    if case.dim == 3:
        return a[..., g:g + case.ni, g:g + case.nj, g:g + case.nk]
    return a[..., g:g + case.ni, g:g + case.nj, :]


def rel_err(a, b):
    """Per-variable normwise relative error: max|a-b| / max|b| over real points."""
    out = []
    for k in range(a.shape[0]):
        s = np.abs(b[k]).max()
        d = np.abs(a[k] - b[k]).max()
        out.append(0.0 if s == 0 and d == 0 else d / (s if s > 0 else 1.0))
    return np.array(out)


def l2_rel(a, b):
    """Per-variable relative L2 error over real points."""
    out = []
    for k in range(a.shape[0]):
        s = np.sqrt(np.mean(b[k] ** 2))
        d = np.sqrt(np.mean((a[k] - b[k]) ** 2))
        out.append(0.0 if s == 0 and d == 0 else d / (s if s > 0 else 1.0))
    return np.array(out)


def conserved(prim5):
    """rho, rho u, rho v, rho w, rho e from SHOCK's state variables."""
    r = prim5[0]
    return np.stack([r, r * prim5[1], r * prim5[2], r * prim5[3], r * prim5[4]])


def reference_floor(case, nsteps):
    """Per-variable distance (normwise, as rel_err) between SHOCK's FP64 and
    80-bit builds after nsteps steps of `case`: the reference's own rounding
    error on it, or None when the reference builds are absent."""
    from refbind import RefSolver, ref_available
    if not (ref_available(case.order, case.dim) and ref_available(case.order, case.dim, extended=True)):
        return None
    a, b = RefSolver(case), RefSolver(case, extended=True)
    a.steps(nsteps)
    b.steps(nsteps)
    return rel_err(real(case, a.state()[:5]), real(case, b.state()[:5]))
