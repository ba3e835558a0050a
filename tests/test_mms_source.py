"""Independent check of the built-in product-form manufactured solution's
source term J*S (shock_host_mms_baseline), without the symbolic generator
that wrote it.

The source is the residual of SHOCK's non-dimensional Navier-Stokes
equations at the exact steady solution (docs/goveq.tex; the discrete terms
are src/WENO.c and src/ZD.c, mu = 1 in manufactured-solution mode,
src/Functions.c:2473-2476):

    S = div F_inviscid(U) - div F_viscous(U)
    F_inviscid,x = (rho u, rho u^2 + Ups p, rho u v, u (rho e + Ups p))
    tau_ij = u_i,j + u_j,i - 2/3 delta_ij div u
    F_viscous,x = (0, Psi tau_xx, Psi tau_xy, Psi (u tau_xx + v tau_xy) + Gam T_x)
    e = |u|^2/2 + Ups/(gamma-1) p/rho,  T = p/rho

Here every derivative is taken numerically: eighth-order central
differences in 80-bit long double of the fields and fluxes written out
below, nested for the viscous terms.  The truncation error of the
differences is below 1e-14 of the terms and their rounding about 1e-12, so
the library's long-double closed forms must agree to 1e-9.
"""
import numpy as np
import pytest

import shock_b200
from shock_b200 import cases

LD = np.longdouble
H = LD(1) / LD(512)
# eighth-order central first derivative: sum_k c_k (f(x+kh) - f(x-kh)) / h
C8 = [LD(4) / LD(5), LD(-1) / LD(5), LD(4) / LD(105), LD(-1) / LD(280)]


def d_dx(f, x, y):
    return sum(c * (f(x + (k + 1) * H, y) - f(x - (k + 1) * H, y)) for k, c in enumerate(C8)) / H


def d_dy(f, x, y):
    return sum(c * (f(x, y + (k + 1) * H) - f(x, y - (k + 1) * H)) for k, c in enumerate(C8)) / H


def _fields(gamma):
    tp = LD(2) * np.arccos(LD(-1))      # 2 pi in long double
    rho = lambda x, y: LD(1) + LD("0.1") * np.sin(tp * x) * np.sin(tp * y)
    u = lambda x, y: LD("0.3") * np.cos(tp * x) * np.sin(tp * y)
    v = lambda x, y: LD("0.3") * np.sin(tp * x) * np.cos(tp * y)
    # SHOCK units at Ma = 1: p_S = gamma * p
    p = lambda x, y: LD(gamma) * (LD(1) / LD(gamma) + LD("0.05") * np.cos(tp * x) * np.cos(tp * y))
    return rho, u, v, p


def source(x, y, gamma, mach, reynolds, prandtl):
    g = LD(gamma)
    ups = LD(1) / (g * LD(mach) ** 2)
    psi = LD(1) / LD(reynolds)
    gam = LD(1) / ((g - 1) * LD(mach) ** 2 * LD(reynolds) * LD(prandtl))
    rho, u, v, p = _fields(gamma)
    e = lambda x, y: (u(x, y) ** 2 + v(x, y) ** 2) / 2 + ups / (g - 1) * p(x, y) / rho(x, y)
    T = lambda x, y: p(x, y) / rho(x, y)
    Hs = lambda x, y: rho(x, y) * e(x, y) + ups * p(x, y)

    def div(fx, fy):
        return d_dx(fx, x, y) + d_dy(fy, x, y)

    # stresses from numerical velocity gradients
    ux = lambda a, b: d_dx(u, a, b)
    uy = lambda a, b: d_dy(u, a, b)
    vx = lambda a, b: d_dx(v, a, b)
    vy = lambda a, b: d_dy(v, a, b)
    txx = lambda a, b: 2 * ux(a, b) - LD(2) / 3 * (ux(a, b) + vy(a, b))
    tyy = lambda a, b: 2 * vy(a, b) - LD(2) / 3 * (ux(a, b) + vy(a, b))
    txy = lambda a, b: uy(a, b) + vx(a, b)
    Tx = lambda a, b: d_dx(T, a, b)
    Ty = lambda a, b: d_dy(T, a, b)

    s_rho = div(lambda a, b: rho(a, b) * u(a, b), lambda a, b: rho(a, b) * v(a, b))
    s_ru = (div(lambda a, b: rho(a, b) * u(a, b) ** 2 + ups * p(a, b), lambda a, b: rho(a, b) * u(a, b) * v(a, b))
            - psi * div(txx, txy))
    s_rv = (div(lambda a, b: rho(a, b) * u(a, b) * v(a, b), lambda a, b: rho(a, b) * v(a, b) ** 2 + ups * p(a, b))
            - psi * div(txy, tyy))
    s_re = (div(lambda a, b: u(a, b) * Hs(a, b), lambda a, b: v(a, b) * Hs(a, b))
            - gam * div(Tx, Ty)
            - psi * div(lambda a, b: u(a, b) * txx(a, b) + v(a, b) * txy(a, b),
                        lambda a, b: u(a, b) * txy(a, b) + v(a, b) * tyy(a, b)))
    return s_rho, s_ru, s_rv, s_re


@pytest.mark.parametrize("n,reynolds", [(64, 100.0), (20, 37.0)])
def test_mms_baseline_source_against_numerical_derivatives(n, reynolds):
    c = cases.mms_square(n, 5, family="baseline", reynolds=reynolds)
    geo = shock_b200.host_geometry(c)
    ex, js = shock_b200.host_mms_baseline(c)
    x = geo[0, :, :, 0].astype(LD)
    y = geo[1, :, :, 0].astype(LD)
    J = geo[3, :, :, 0].astype(LD)
    s = source(x, y, c.gamma, c.mach, c.reynolds, c.prandtl)
    g = c.ghosts
    real = (slice(g, g + c.ni), slice(g, g + c.nj))
    for k, sk in zip((0, 1, 2, 4), s):
        ref = (J * sk)[real]
        got = js[k, :, :, 0][real].astype(LD)
        err = float(np.abs(got - ref).max() / np.abs(ref).max())
        assert err < 1e-9, (k, err)
    assert not js[3].any()


def test_mms_baseline_exact_fields():
    """The exact state of the Dirichlet ghosts: rho, u, v, e, p, T, c, mu."""
    c = cases.mms_square(24, 5, family="baseline")
    geo = shock_b200.host_geometry(c)
    ex, _ = shock_b200.host_mms_baseline(c)
    rho, u, v, p = _fields(c.gamma)
    x = geo[0, :, :, 0].astype(LD)
    y = geo[1, :, :, 0].astype(LD)
    ups = 1.0 / (c.gamma * c.mach ** 2)
    r, uu, vv, pp = (f(x, y).astype(np.float64) for f in (rho, u, v, p))
    e = 0.5 * (uu * uu + vv * vv) + pp / r / (c.gamma - 1) * ups
    for k, ref in ((0, r), (1, uu), (2, vv), (4, e), (5, pp), (6, pp / r), (7, np.sqrt(ups * c.gamma * pp / r))):
        err = np.abs(ex[k, :, :, 0] - ref).max() / np.abs(ref).max()
        assert err < 1e-14, (k, err)
    assert np.all(ex[8] == 1.0) and not ex[3].any()
