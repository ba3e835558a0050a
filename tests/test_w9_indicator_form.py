"""The WENO9 smoothness indicators of the kernels (FP32 and FP64) are
SHOCK's integer quadratic forms (src/WENO.c:25-53) rewritten on first
differences as sums of squares.

The tables are read from the kernel source.  On random stencils the
factorised form must give SHOCK's value exactly (the tables hold exact
rationals, the FP32 and FP64 tables the same ones), and in FP32 / FP64 it
must stay within a few units of rounding, where the integer form loses up
to about 1e-3 (FP32) to cancellation.
"""
import os
import re
from fractions import Fraction

import numpy as np

SRC = os.path.join(os.path.dirname(__file__), "..", "shock_b200", "csrc", "stage_bodies.cuh")


def _table(name):
    text = open(SRC).read()
    body = text[text.index(name):]
    body = body[body.index("{") + 1:body.index("};")]
    rows = re.findall(r"\{([^{}]*)\}", body)
    out = []
    for row in rows:
        vals = []
        for item in (x.strip() for x in row.split(",")):
            if not item:
                continue
            m = re.fullmatch(r"(?:float|double)\((-?\d+)\. / (\d+)\.\)", item)
            if m:
                vals.append(Fraction(int(m.group(1)), int(m.group(2))))
            else:
                vals.append(Fraction(item.rstrip("f").rstrip(".")))
        out.append(vals)
    return out


def _shock_form(c, f):
    """SHOCK's indicator: the upper-triangle integer form on 5 values."""
    acc, i = Fraction(0), 0
    for a in range(5):
        for b in range(a, 5):
            acc += c[i] * f[a] * f[b]
            i += 1
    return acc


def _ldl_form(t, d):
    L10, L20, L21, L30, L31, L32, D0, D1, D2, D3 = t
    y0 = d[0] + L10 * d[1] + L20 * d[2] + L30 * d[3]
    y1 = d[1] + L21 * d[2] + L31 * d[3]
    y2 = d[2] + L32 * d[3]
    return D0 * y0 * y0 + D1 * y1 * y1 + D2 * y2 * y2 + D3 * d[3] * d[3]


def test_factorised_indicators_equal_shock_forms():
    ints, ldl = _table("c_w9is[5][15]"), _table("c_w9ldl[5][10]")
    assert len(ints) == 5 and len(ldl) == 5
    rng = np.random.default_rng(7)
    for k in range(5):
        assert all(x > 0 for x in ldl[k][6:]), "pivots of a positive-definite form"
        for trial in range(300):
            f = [Fraction(float(v)) for v in np.cumsum(rng.normal(size=5))]
            d = [f[j + 1] - f[j] for j in range(4)]
            exact = _shock_form(ints[k], f)
            # the table holds exact rationals: the identity holds exactly
            assert _ldl_form(ldl[k], d) == exact


def test_factorised_indicators_fp32_accuracy():
    ints, ldl = _table("c_w9is[5][15]"), _table("c_w9ldl[5][10]")
    rng = np.random.default_rng(11)
    worst_new = worst_old = 0.0
    for k in range(5):
        t32 = [np.float32(float(x)) for x in ldl[k]]
        c32 = [np.float32(float(x)) for x in ints[k]]
        for trial in range(400):
            # a random walk, a gentle slope on an offset, a jump with small noise
            kind = trial % 3
            if kind == 0:
                x = np.cumsum(rng.normal(size=5))
            elif kind == 1:
                x = rng.normal() + rng.normal() * np.linspace(0, 1, 5) + 1e-3 * rng.normal(size=5)
            else:
                x = np.where(np.arange(5) < 1 + trial % 4, 1.0, -1.0) + 1e-4 * rng.normal(size=5)
            exact = float(_shock_form(ints[k], [Fraction(float(v)) for v in x]))
            d = np.diff(x).astype(np.float32)
            new = np.float32(_ldl_form(t32, d))
            f = (x - x[0]).astype(np.float32)
            old, i = np.float32(0), 0
            for a in range(5):
                inner = np.float32(0)
                for b in range(a, 5):
                    inner = np.float32(inner + c32[i] * f[b])
                    i += 1
                old = np.float32(old + f[a] * inner)
            worst_new = max(worst_new, abs(float(new) - exact) / exact)
            worst_old = max(worst_old, abs(float(old) - exact) / exact)
    print(f"FP32 relative error: factorised {worst_new:.2e}, integer form {worst_old:.2e}")
    assert worst_new < 1e-5, worst_new
    assert worst_old > 20 * worst_new, (worst_old, worst_new)


def test_fp64_table_is_the_fp32_one():
    assert _table("c_w9ldl64[5][10]") == _table("c_w9ldl[5][10]")


def test_factorised_indicators_fp64_accuracy():
    """In FP64 the factorised form is at least as accurate as the integer form
    SHOCK evaluates, to a few units of FP64 rounding."""
    ints, ldl = _table("c_w9is[5][15]"), _table("c_w9ldl64[5][10]")
    rng = np.random.default_rng(13)
    worst_new = worst_old = 0.0
    for k in range(5):
        t64 = [float(x) for x in ldl[k]]
        c64 = [float(x) for x in ints[k]]
        for trial in range(300):
            kind = trial % 3
            if kind == 0:
                x = np.cumsum(rng.normal(size=5))
            elif kind == 1:
                x = rng.normal() + rng.normal() * np.linspace(0, 1, 5) + 1e-6 * rng.normal(size=5)
            else:
                x = np.where(np.arange(5) < 1 + trial % 4, 1.0, -1.0) + 1e-8 * rng.normal(size=5)
            exact = float(_shock_form(ints[k], [Fraction(float(v)) for v in x]))
            d = np.diff(x)
            new = _ldl_form(t64, d)
            old, i = 0.0, 0
            for a in range(5):
                inner = 0.0
                for b in range(a, 5):
                    inner = inner + c64[i] * x[b]
                    i += 1
                old = old + x[a] * inner
            worst_new = max(worst_new, abs(float(new) - exact) / exact)
            worst_old = max(worst_old, abs(float(old) - exact) / exact)
    print(f"FP64 relative error: factorised {worst_new:.2e}, integer form {worst_old:.2e}")
    assert worst_new < 1e-14, worst_new
    assert worst_old >= worst_new, (worst_old, worst_new)
