"""Generate the golden fixtures in tests/golden/ from SHOCK's own code.

Runs the reference translation units (oracle/_ref, built by
``make -C oracle ref`` from the unmodified sources in the reference tree)
on small seeded cases and stores, per case, the inputs (grid, initial
primitives, parameters, manufactured-solution data) and the outputs
(geometry, one right-hand side, the state after a few full RK steps).
The fixtures pin the CPU restatement in oracle/ (tests/test_oracle_pin.py)
and, through it, the GPU kernels.  The same reference sources built at
PRECISION=3 (80-bit long double) give rhs80/state80: the distance between
the FP64 and the 80-bit results is SHOCK's own FP64 rounding floor, which
sets the parity tolerance on ill-conditioned cases (low Mach, WENO9).

Usage: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from shock_b200 import cases  # noqa: E402
from refbind import RefSolver  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def golden_cases():
    yield "w5_2d_visc_stretch", cases.smooth_random(2, 5, (14, 12, 1), seed=11, stretch=0.1), 3
    yield "w9_2d_inviscid_rk3", cases.smooth_random(2, 9, (14, 13, 1), seed=12, inviscid=True, time_order=3), 3
    yield "w5_3d_visc", cases.smooth_random(3, 5, (10, 9, 9), seed=13), 2
    yield "w9_3d_visc", cases.smooth_random(3, 9, (12, 11, 11), seed=14), 1
    yield "w5_3d_tgv_curvilinear", cases.taylor_green(12, order=5), 2
    yield "w5_3d_inviscid_stretch", cases.smooth_random(3, 5, (9, 8, 10), seed=15, inviscid=True, stretch=0.1), 2
    yield "w5_2d_mms_reference", cases.mms_square(16, 5, family="reference", mms_case=0), 3
    yield "w9_2d_mms_reference_supersonic", cases.mms_square(20, 9, family="reference", mms_case=1), 2
    yield "w5_2d_mms_baseline", cases.mms_square(32, 5, family="baseline"), 3


def case_arrays(c):
    d = dict(dim=c.dim, order=c.order, ni=c.ni, nj=c.nj, nk=c.nk, time_order=c.time_order,
             tau=c.tau, mach=c.mach, reynolds=c.reynolds, prandtl=c.prandtl, gamma=c.gamma,
             gas_r=c.gas_r, t0=c.t0, l0=c.l0, inviscid=int(c.inviscid), mms=c.mms,
             mms_case=c.mms_case, periodic=np.array(c.periodic, dtype=np.int32),
             period=np.array(c.period, dtype=np.float64))
    for k in ("x", "y", "z", "rho", "u", "v", "w", "p"):
        d["in_" + k] = getattr(c, k)
    return d


def main():
    import shock_b200
    for name, c, nsteps in golden_cases():
        d = case_arrays(c)
        ext = None
        if c.mms == "baseline":
            # the product-form manufactured solution, evaluated by the library's
            # host code, drives the reference through ref_harness/mms_external.c
            ext = shock_b200.host_mms_baseline(c)
            d["dirichlet9"], d["source5"] = ext
        r = RefSolver(c, external=ext)
        if c.mms == "reference":
            d["dirichlet9"] = r.mms_exact()
            d["source5"] = r.mms_source()
        d["geometry"] = r.geometry()
        d["rhs"] = r.rhs()
        r.steps(nsteps)
        d["nsteps"] = nsteps
        d["state"] = r.state(0)[:5]
        if ext is None:
            r80 = RefSolver(c, extended=True)
            d["rhs80"] = r80.rhs()
            r80.steps(nsteps)
            d["state80"] = r80.state(0)[:5]
        else:   # no extended-precision build of the external-data variant
            d["rhs80"] = d["rhs"]
            d["state80"] = d["state"]
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **d)
        print("wrote", name)


if __name__ == "__main__":
    main()
