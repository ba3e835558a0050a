import os
import subprocess
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(__file__))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def pytest_sessionstart(session):
    # The oracle is a plain-C checker; build it if this tree has no copy yet.
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=True)


# Achieved parity errors, recorded by the GPU parity tests and printed at the
# end of the run (and written as JSON to $SHOCK_PARITY_REPORT when it is set),
# so that a run records the errors reached, not only that they were in bounds.
_REPORT = []


def record_parity(test, case, kind, err, tol, floor=None):
    import numpy as np
    e = np.atleast_1d(np.asarray(err, dtype=float))
    t = np.atleast_1d(np.asarray(tol, dtype=float))
    row = {"test": test, "case": case, "kind": kind, "max_err": float(e.max()),
           "err": [float(x) for x in e], "tol": [float(x) for x in np.broadcast_to(t, e.shape)]}
    if floor is not None:
        row["reference_floor"] = [float(x) for x in np.atleast_1d(floor)]
    _REPORT.append(row)


@pytest.fixture
def parity():
    return record_parity


def pytest_terminal_summary(terminalreporter):
    if not _REPORT:
        return
    tr = terminalreporter
    tr.write_sep("-", "achieved parity errors (max over variables; tolerance)")
    for r in _REPORT:
        fl = f" floor {max(r['reference_floor']):.1e}" if "reference_floor" in r else ""
        if r["kind"].startswith("observed order"):
            tr.write_line(f"{r['case']:<34} {r['kind']:<26} {min(r['err']):.2f} >= {max(r['tol']):.1f}")
        else:
            tr.write_line(f"{r['case']:<34} {r['kind']:<26} {r['max_err']:.2e} <= {max(r['tol']):.1e}{fl}")
    path = os.environ.get("SHOCK_PARITY_REPORT")
    if path:
        import json
        with open(path, "w") as f:
            json.dump(_REPORT, f, indent=1)
