"""Problem set-ups: grids, initial states and SHOCK parameters.

A ``Case`` carries everything SHOCK reads from its CGNS grid/solution and
``config.ini`` for one run of the per-RK-stage path: the real-point
coordinates and primitive fields (the arrays ``loadFile`` returns,
src/Load.c:252-744), the ``[Numerics]``/``[FluidProperties]``/``[Options]``
keys the hot path consumes (src/Import.c:36-238), and which faces are
periodic (SHOCK encodes periodicity as self-interfaces in the ``.sddc``
division file, src/Load.c:191-250).

Non-dimensionalisation follows SHOCK (src/Functions.c:2012-2013,
docs/goveq.tex:158-162): Upsilon = 1/(gamma Ma^2), p = rho T,
e = |u|^2/2 + Upsilon/(gamma-1) p/rho, velocities in units of
u_ref = Ma c_0.  States given with rho_0 = 1, c_0 = 1 map to SHOCK units
at Ma = 1 as rho_S = rho, u_S = u, p_S = gamma p.

The generators here build the benchmark workloads from their definitions
with seeded synthetic data (no dataset is involved):
  * ``mms_square``       -- 2D manufactured solution on the unit square
  * ``taylor_green``     -- 3D Taylor-Green vortex on a perturbed periodic cube
  * ``decaying_turbulence`` -- random-phase solenoidal field, periodic cube
  * ``isentropic_vortex``-- 2D periodic isentropic vortex (ensemble members)
  * ``smooth_random``    -- smooth random periodic states for parity tests
  * ``channel``          -- wall-bounded blocks (wall / farfield y faces) for the
                            boundary-condition parity tests
  * ``duct``             -- through-flow blocks (inflow / outflow x faces)
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional, Tuple

import numpy as np


@dataclasses.dataclass
class Case:
    dim: int
    order: int                      # WENO order: 5 or 9 (SPACEORDER)
    ni: int
    nj: int
    nk: int
    x: np.ndarray                   # real-point coordinates, shape (ni,nj,nk)
    y: np.ndarray
    z: np.ndarray
    rho: np.ndarray                 # real-point primitives, shape (ni,nj,nk)
    u: np.ndarray
    v: np.ndarray
    w: np.ndarray
    p: np.ndarray
    time_order: int = 4             # [Numerics] TimeOrder: 3 (RK3-TVD) or 4 (RK4)
    tau: float = 1e-3               # [Numerics] Tau
    mach: float = 1.0               # [FluidProperties] Mach
    reynolds: float = 1000.0        # Reynolds
    prandtl: float = 0.72           # Prandtl
    gamma: float = 1.4              # Gamma
    gas_r: float = 287.0            # R
    t0: float = 300.0               # T
    l0: float = 1.0                 # L
    inviscid: bool = False          # [Options] Inviscid
    mms: str = "none"               # "none" | "reference" (ManufacturedSolution.c family) | "baseline"
    mms_case: int = 0               # [ManufacturedSolution] case
    periodic: Tuple[bool, bool, bool] = (True, True, True)
    period: Tuple[float, float, float] = (1.0, 1.0, 1.0)
    bc: Tuple[int, int, int, int, int, int] = (0, 0, 0, 0, 0, 0)   # SHOCK_BC_* per face (Left..InFront)
    t_wall: float = 1.0             # [BoundaryConditions] T_wall (isothermal walls)
    rho_inflow: float = 1.0         # [BoundaryConditions] rho_inflow, p_inflow, p_outflow
    p_inflow: float = 1.0
    p_outflow: float = 1.0
    u_inflow: Tuple[float, float, float] = (0.0, 0.0, 0.0)   # cos/sin(AoA)*u0, 0: also SHOCK's Initialize velocity
    name: str = "case"

    @property
    def ghosts(self) -> int:
        return (self.order + 1) // 2

    @property
    def real_points(self) -> int:
        return self.ni * self.nj * (self.nk if self.dim == 3 else 1)

    def real_fields(self):
        return (self.x, self.y, self.z, self.u, self.v, self.w, self.p, self.rho)

    def replace(self, **kw) -> "Case":
        return dataclasses.replace(self, **kw)

    def energy(self) -> np.ndarray:
        """e from (rho,u,v,w,p) exactly as src/Functions.c:872-874 forms it."""
        ups = 1.0 / (self.gamma * (self.mach * self.mach))
        return (0.5 * ((self.u * self.u) + (self.v * self.v) + (self.w * self.w))
                + self.p / self.rho / (self.gamma - 1.0) * ups)


def _mesh(dim, n, lo, length, endpoint):
    axes = []
    for a in range(3):
        if a < dim:
            if endpoint:
                axes.append(lo[a] + length[a] * np.arange(n[a]) / (n[a] - 1))
            else:
                axes.append(lo[a] + length[a] * np.arange(n[a]) / n[a])
        else:
            axes.append(np.zeros(1))
    return np.meshgrid(*axes, indexing="ij")


def cfl_tau(case: Case, cfl: float = 0.5) -> float:
    """tau = cfl / max over cells of sum_d (|theta_d| + c |grad xi_d| +
    2 nu |grad xi_d|^2) on the initial state, with |grad xi_d| = 1/spacing
    of the Cartesian skeleton and nu = max(4/3, gamma/Pr) mu / (rho Re) the
    largest diffusivity of SHOCK's viscous terms (momentum, and heat: in
    SHOCK's units T diffuses at gamma mu / (rho Re Pr) whatever the Mach
    number), mu taken as 1.  The viscous part matters only on fine grids at
    low Reynolds number: on the 64^2 unit-square manufactured solution at
    Re = 100 the convective estimate alone gives a step about three times
    RK4's stability limit of the sixth-order viscous stencils (SHOCK's own
    build diverges after some 25 steps there)."""
    ups = 1.0 / (case.gamma * case.mach ** 2)
    c = np.sqrt(ups * case.gamma * case.p / case.rho)
    vel = (case.u, case.v, case.w)
    n = (case.ni, case.nj, case.nk)
    nu = 0.0 if case.inviscid else max(4.0 / 3.0, case.gamma / case.prandtl) / (case.rho * case.reynolds)
    s = np.zeros_like(case.rho)
    for a in range(case.dim):
        h = case.period[a] / n[a] if case.periodic[a] else case.period[a] / (n[a] - 1)
        s = s + (np.abs(vel[a]) + c) / h + 2.0 * nu / (h * h)
    return float(cfl / s.max())


def smooth_random(dim: int, order: int, n: Tuple[int, int, int], seed: int = 0,
                  amp: float = 0.05, mach: float = 1.0, inviscid: bool = False,
                  reynolds: float = 200.0, time_order: int = 4, stretch: float = 0.0,
                  length: float = 1.0) -> Case:
    """Smooth random periodic state: a few low Fourier modes per field on a
    periodic box, optionally with a smooth coordinate stretch per axis."""
    rng = np.random.default_rng(seed)
    ni, nj, nk = n[0], n[1], (n[2] if dim == 3 else 1)
    L = (length, length, length if dim == 3 else 1.0)
    x, y, z = _mesh(dim, (ni, nj, nk), (0.0, 0.0, 0.0), L, endpoint=False)
    if stretch:
        x = x + stretch * L[0] / (2 * math.pi) * np.sin(2 * math.pi * x / L[0])
        y = y + stretch * L[1] / (2 * math.pi) * np.sin(2 * math.pi * y / L[1])
        if dim == 3:
            z = z + stretch * L[2] / (2 * math.pi) * np.sin(2 * math.pi * z / L[2])
    X = [2 * math.pi * x / L[0], 2 * math.pi * y / L[1], 2 * math.pi * z / L[2]]

    def field():
        f = np.zeros_like(x)
        for _ in range(3):
            kv = rng.integers(0, 3, size=3)
            if dim == 2:
                kv[2] = 0
            ph = rng.uniform(0, 2 * math.pi)
            f = f + rng.normal() * np.sin(kv[0] * X[0] + kv[1] * X[1] + kv[2] * X[2] + ph)
        return f

    rho = 1.0 + amp * field()
    u = 0.3 + amp * field()
    v = -0.2 + amp * field()
    w = (0.1 + amp * field()) if dim == 3 else np.zeros_like(x)
    p = 1.0 + amp * field()
    c = Case(dim=dim, order=order, ni=ni, nj=nj, nk=nk, x=x, y=y, z=z, rho=rho, u=u, v=v,
             w=w, p=p, time_order=time_order, mach=mach, reynolds=reynolds,
             inviscid=inviscid, periodic=(True, True, dim == 3), period=L,
             name=f"smooth{dim}d_w{order}")
    c.tau = cfl_tau(c)
    return c


def parabolic_cgrid(dim: int, order: int, n: Tuple[int, int, int], half_width: float = 1.5, height: float = 1.2,
                    span: float = 0.4, seed: int = 0, mach: float = 0.5, reynolds: float = 500.0,
                    inviscid: bool = False) -> Case:
    """A C-grid in parabolic coordinates, x = (xi^2 - eta^2)/2, y = xi eta
    (z = the span in 3D, periodic): xi runs over ni points across
    (-half_width, half_width), eta over nj points in (0, height), both at
    half-cell offsets, so the grid wraps around the focus and the row below
    j = 0 is the row j = 0 read from the other end of i (the ghost point
    (xi, -eta) is the point (-xi, eta)).  That cut is the wake cut of a
    C-grid (division_file generators join it bottom to bottom with
    Transform (-1,-2,3), see wake_cut); the other faces are farfield.  A
    seeded smooth state on a uniform stream along x."""
    rng = np.random.default_rng(seed)
    ni, nj, nk = n[0], n[1], (n[2] if dim == 3 else 1)
    xi = -half_width + (np.arange(ni) + 0.5) * (2 * half_width / ni)
    eta = (np.arange(nj) + 0.5) * (height / nj)
    zs = span * np.arange(nk) / nk if dim == 3 else np.zeros(1)
    X, E, Z = np.meshgrid(xi, eta, zs, indexing="ij")
    x = 0.5 * (X * X - E * E)
    y = X * E
    z = Z

    def smooth():
        return sum(rng.normal() * np.sin(rng.integers(1, 3) * x + rng.uniform(0, 2 * math.pi))
                   * np.cos(rng.integers(1, 3) * y) for _ in range(2))

    amp = 0.02
    u = 1.0 + amp * smooth()
    v = amp * smooth()
    w = amp * smooth() if dim == 3 else np.zeros_like(x)
    rho = 1.0 + amp * smooth()
    p = 1.0 / (1.4 * mach * mach) * (1.0 + amp * smooth())
    far = 3   # BC_NAMES["farfield"]
    c = Case(dim=dim, order=order, ni=ni, nj=nj, nk=nk, x=x, y=y, z=z, rho=rho, u=u, v=v, w=w, p=p,
             mach=mach, reynolds=reynolds, inviscid=inviscid, periodic=(False, False, dim == 3),
             period=(1.0, 1.0, span), bc=(far, far, 0, far, 0, 0), u_inflow=(1.0, 0.0, 0.0),
             name=f"cgrid{dim}d_w{order}")
    # the cells around the focus are small and skewed: SHOCK's own run of a
    # 24 x 12 grid blows up within 10 steps at CFL 0.5 of this estimate
    c.tau = cfl_tau(c, cfl=0.125)
    return c


def wake_cut(division: "Division") -> "Division":
    """The division of a C-grid (parabolic_cgrid) with its wake cut: the
    bottom face of block (i, 0, k) joins the bottom face of block
    (parts[0]-1-i, 0, k) with Transform (-1,-2,3) -- i runs the other way
    across the cut, and both normals point out of the zone -- as SHOCK's own
    division generator writes it (TOOLS/generatedivfile/generatedivfile_3.c,
    its case 2).  The blocks along i must mirror one another in size."""
    P = division.parts
    nb = division.neighbour.copy()
    tf = division.transform.copy()
    blocks = list(division.blocks)
    for k in range(P[2]):
        for i in range(P[0]):
            r = (k * P[1]) * P[0] + i
            m = (k * P[1]) * P[0] + (P[0] - 1 - i)
            if blocks[r].ni != blocks[m].ni:
                raise ValueError("the blocks along i do not mirror one another")
            nb[r, 2] = m
            tf[r, 2] = (-1, -2, 3)
            bc = list(blocks[r].bc)
            bc[2] = 0
            blocks[r] = blocks[r].replace(bc=tuple(bc))
    return Division(case=division.case, parts=division.parts, blocks=blocks, neighbour=nb,
                    translation=division.translation.copy(), lo=division.lo, transform=tf,
                    axes=division.axes, flips=division.flips)


BC_NAMES = {"wall_viscous": 1, "wall_inviscid": 2, "farfield": 3, "wall_isothermal": 4,
            "inflow_subsonic": 5, "inflow_supersonic": 6, "outflow_subsonic": 7,
            "inflow_riemann": 8, "inflow_isentropic": 9, "outflow_riemann": 10, "outflow_rudy": 11}


def channel(dim: int, order: int, n: Tuple[int, int, int], bc: str = "wall_viscous", seed: int = 0,
            mach: float = 0.3, reynolds: float = 500.0, inviscid: bool = False, time_order: int = 4,
            stretch: float = 0.0, walls_i: bool = False, prandtl: float = 0.72, t_wall: float = 1.0) -> Case:
    """Wall-bounded block: periodic in x (and z in 3D), the two y faces of
    type ``bc`` (SHOCK's BCWallViscous / BCWallInviscid / BCFarfield /
    BCWallViscousIsothermal at t_wall).  The
    wall-normal grid spans [0, 1] with both end points on the walls and an
    optional tanh clustering towards them.  Initial state: a parabolic
    streamwise profile plus smooth seeded perturbations.  walls_i=True also
    closes the x faces (a box with walls on two axes)."""
    rng = np.random.default_rng(seed)
    ni, nj, nk = n[0], n[1], (n[2] if dim == 3 else 1)
    Lx, Lz = 2.0, 1.0
    xa = Lx * np.arange(ni) / (ni - 1 if walls_i else ni)
    eta = np.arange(nj) / (nj - 1)
    ya = 0.5 * (1.0 + np.tanh(stretch * (2 * eta - 1)) / math.tanh(stretch)) if stretch else eta
    za = Lz * np.arange(nk) / nk if dim == 3 else np.zeros(1)
    x, y, z = np.meshgrid(xa, ya, za, indexing="ij")
    X, Z = 2 * math.pi * x / Lx, 2 * math.pi * z / Lz

    def pert():
        f = np.zeros_like(x)
        for _ in range(2):
            kx, kz = rng.integers(1, 3), (rng.integers(0, 3) if dim == 3 else 0)
            f = f + rng.normal() * np.sin(math.pi * y) * np.sin(kx * X + kz * Z + rng.uniform(0, 2 * math.pi))
        return f

    amp = 0.05
    u = 4.0 * y * (1.0 - y) + amp * pert()
    v = amp * pert()
    w = amp * pert() if dim == 3 else np.zeros_like(x)
    rho = 1.0 + 0.02 * pert()
    p = 1.0 + 0.02 * pert()
    t = BC_NAMES[bc]
    faces = [0, 0, t, t, 0, 0]
    if walls_i:
        faces[0] = faces[1] = t
    c = Case(dim=dim, order=order, ni=ni, nj=nj, nk=nk, x=x, y=y, z=z, rho=rho, u=u, v=v, w=w, p=p,
             time_order=time_order, mach=mach, reynolds=reynolds, inviscid=inviscid, prandtl=prandtl,
             periodic=(not walls_i, False, dim == 3), period=(Lx, 1.0, Lz), bc=tuple(faces), t_wall=t_wall,
             name=f"channel{dim}d_w{order}_{bc}")
    c.tau = cfl_tau(c)
    return c


def duct(dim: int, order: int, n: Tuple[int, int, int], inflow: str = "inflow_subsonic", seed: int = 0,
         mach: float = 0.5, reynolds: float = 500.0, inviscid: bool = False, time_order: int = 4,
         walls: str = "", outflow: str = "outflow_subsonic") -> Case:
    """Through-flow block: inflow of kind ``inflow`` on the x-lower face,
    outflow of kind ``outflow`` on the x-upper face, periodic in y (and z),
    or ``walls`` ("wall_viscous", ...) on the y faces.  The inflow state is rho_inflow = p_inflow = 1 moving at
    u_inflow = (1, 0, 0) (in SHOCK's velocity units, Ma = mach); the initial
    field is that state with smooth seeded perturbations; p_outflow is 0.98
    of the inflow pressure."""
    rng = np.random.default_rng(seed)
    ni, nj, nk = n[0], n[1], (n[2] if dim == 3 else 1)
    Lx, Ly, Lz = 2.0, 1.0, 1.0
    xa = Lx * np.arange(ni) / (ni - 1)
    ya = Ly * np.arange(nj) / (nj - 1 if walls else nj)
    za = Lz * np.arange(nk) / nk if dim == 3 else np.zeros(1)
    x, y, z = np.meshgrid(xa, ya, za, indexing="ij")
    X, Y, Z = 2 * math.pi * x / Lx, 2 * math.pi * y / Ly, 2 * math.pi * z / Lz

    def pert():
        f = np.zeros_like(x)
        for _ in range(2):
            ky, kz = rng.integers(1, 3), (rng.integers(0, 3) if dim == 3 else 0)
            f = f + rng.normal() * np.sin(math.pi * x / Lx) * np.sin(ky * Y + kz * Z + rng.uniform(0, 2 * math.pi))
        return f

    amp = 0.03
    u = 1.0 + amp * pert()
    v = amp * pert()
    w = amp * pert() if dim == 3 else np.zeros_like(x)
    rho = 1.0 + amp * pert()
    p = 1.0 + amp * pert()
    faces = [BC_NAMES[inflow], BC_NAMES[outflow], 0, 0, 0, 0]
    if walls:
        faces[2] = faces[3] = BC_NAMES[walls]
    c = Case(dim=dim, order=order, ni=ni, nj=nj, nk=nk, x=x, y=y, z=z, rho=rho, u=u, v=v, w=w, p=p,
             time_order=time_order, mach=mach, reynolds=reynolds, inviscid=inviscid,
             periodic=(False, not walls, dim == 3), period=(Lx, Ly, Lz), bc=tuple(faces),
             rho_inflow=1.0, p_inflow=1.0, p_outflow=0.98, u_inflow=(1.0, 0.0, 0.0),
             name=f"duct{dim}d_w{order}_{inflow}_{outflow}")
    c.tau = cfl_tau(c)
    return c


def taylor_green(n: int = 64, order: int = 5, mach: float = 0.1, reynolds: float = 1600.0,
                 perturb: float = 0.05, time_order: int = 4) -> Case:
    """3D Taylor-Green vortex on [0,2pi)^3 with every coordinate perturbed by
    x_i += perturb*sin(x_j)*sin(x_k).  u = sin x cos y cos z,
    v = -cos x sin y cos z, w = 0, p = p0 + (cos2x+cos2y)(cos2z+2)/16 at Ma,
    isothermal rho (T = 1).  In SHOCK units p_S = 1 + gamma Ma^2 (...)/16."""
    L = 2 * math.pi
    X, Y, Z = _mesh(3, (n, n, n), (0.0, 0.0, 0.0), (L, L, L), endpoint=False)
    x = X + perturb * np.sin(Y) * np.sin(Z)
    y = Y + perturb * np.sin(X) * np.sin(Z)
    z = Z + perturb * np.sin(X) * np.sin(Y)
    gamma = 1.4
    u = np.sin(X) * np.cos(Y) * np.cos(Z)
    v = -np.cos(X) * np.sin(Y) * np.cos(Z)
    w = np.zeros_like(X)
    p = 1.0 + gamma * mach ** 2 * (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0) / 16.0
    rho = p.copy()
    c = Case(dim=3, order=order, ni=n, nj=n, nk=n, x=x, y=y, z=z, rho=rho, u=u, v=v, w=w,
             p=p, time_order=time_order, mach=mach, reynolds=reynolds, gamma=gamma,
             periodic=(True, True, True), period=(L, L, L), name=f"tgv{n}_w{order}")
    c.tau = cfl_tau(c)
    return c


def mms_square(n: int = 64, order: int = 5, family: str = "baseline", reynolds: float = 100.0,
               mms_case: int = 0, inviscid: bool = False, time_order: int = 4) -> Case:
    """2D unit square with n x n points on [0,1]^2 (x_i = i/(n-1), the
    2d_cube layout), manufactured-solution mode: every face is a Dirichlet
    ghost face holding the exact solution (src/ManufacturedSolution.c:340-388).

    family "baseline": rho = 1+0.1 sin(2pi x)sin(2pi y), u = 0.3 cos(2pi x)sin(2pi y),
      v = 0.3 sin(2pi x)cos(2pi y), p = 1/gamma + 0.05 cos(2pi x)cos(2pi y), at
      Ma = 1 (so p_S = gamma p), Re = 100, Pr = 0.72.
    family "reference": SHOCK's own sum-of-separable family; the initial state
      is overwritten by InitializeManufacturedSolution, so the fields here are
      placeholders."""
    X, Y, Z = _mesh(2, (n, n, 1), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), endpoint=True)
    gamma = 1.4
    tp = 2 * math.pi
    rho = 1.0 + 0.1 * np.sin(tp * X) * np.sin(tp * Y)
    u = 0.3 * np.cos(tp * X) * np.sin(tp * Y)
    v = 0.3 * np.sin(tp * X) * np.cos(tp * Y)
    w = np.zeros_like(X)
    p = gamma * (1.0 / gamma + 0.05 * np.cos(tp * X) * np.cos(tp * Y))
    mach = 1.0
    if family == "reference":
        mach = 0.5
        rho = np.ones_like(X)
        u = np.zeros_like(X)
        v = np.zeros_like(X)
        p = np.ones_like(X)
    c = Case(dim=2, order=order, ni=n, nj=n, nk=1, x=X, y=Y, z=Z, rho=rho, u=u, v=v, w=w, p=p,
             time_order=time_order, mach=mach, reynolds=reynolds, gamma=gamma,
             inviscid=inviscid, mms=family, mms_case=mms_case,
             periodic=(False, False, False), period=(1.0, 1.0, 1.0),
             name=f"mms_{family}{n}_w{order}")
    c.tau = cfl_tau(c)
    return c


def isentropic_vortex(n: int, beta: float, mach_inf: float, order: int = 5,
                      length: float = 10.0, inviscid: bool = True, reynolds: float = 1e4,
                      time_order: int = 4) -> Case:
    """2D isentropic vortex (Shu's form) centred in a periodic [0,L)^2 box,
    free stream along x at Mach mach_inf, with rho_0 = 1, c_0 = 1, p_0 = 1/gamma:
      du = -beta/(2pi) (y-yc) e^{(1-r^2)/2}, dv = beta/(2pi) (x-xc) e^{(1-r^2)/2},
      T = 1 - (gamma-1) beta^2/(8 gamma pi^2) e^{1-r^2}, rho = T^{1/(gamma-1)},
      p = rho T / gamma.  Mapped to SHOCK units at Ma = 1."""
    gamma = 1.4
    X, Y, Z = _mesh(2, (n, n, 1), (0.0, 0.0, 0.0), (length, length, 1.0), endpoint=False)
    xc = yc = length / 2
    r2 = (X - xc) ** 2 + (Y - yc) ** 2
    ex = np.exp(0.5 * (1.0 - r2))
    u = mach_inf + (-beta / (2 * math.pi)) * (Y - yc) * ex
    v = (beta / (2 * math.pi)) * (X - xc) * ex
    T = 1.0 - (gamma - 1.0) * beta ** 2 / (8 * gamma * math.pi ** 2) * ex * ex
    rho = T ** (1.0 / (gamma - 1.0))
    p_b = rho * T / gamma
    c = Case(dim=2, order=order, ni=n, nj=n, nk=1, x=X, y=Y, z=Z, rho=rho, u=u, v=v,
             w=np.zeros_like(X), p=gamma * p_b, time_order=time_order, mach=1.0,
             reynolds=reynolds, gamma=gamma, inviscid=inviscid,
             periodic=(True, True, False), period=(length, length, 1.0),
             name=f"vortex{n}")
    c.tau = cfl_tau(c)
    return c


def decaying_turbulence(n: int = 512, order: int = 9, seed: int = 3, mach_t: float = 0.6,
                        re_lambda: float = 100.0, k0: float = 4.0,
                        time_order: int = 4) -> Case:
    """Random-phase solenoidal velocity on [0,2pi)^3 with E(k) ~ k^4 exp(-2(k/k0)^2),
    scaled to turbulent Mach sqrt(<u.u>)/c = mach_t; rho = 1, p = 1/gamma
    (p_S = 1 at Ma = 1).  Re chosen so Re_lambda = u' lambda / nu = re_lambda
    with lambda^2 = 15 u'^2 / <omega^2> and u' = sqrt(<u.u>/3)."""
    L = 2 * math.pi
    rng = np.random.default_rng(seed)
    kk = np.fft.fftfreq(n, d=1.0 / n)
    kz = np.fft.rfftfreq(n, d=1.0 / n)
    KX, KY, KZ = np.meshgrid(kk, kk, kz, indexing="ij")
    K2 = KX ** 2 + KY ** 2 + KZ ** 2
    K = np.sqrt(K2)
    Ksafe = np.where(K == 0, 1.0, K)
    E = Ksafe ** 4 * np.exp(-2.0 * (Ksafe / k0) ** 2)
    amp = np.sqrt(E / (4 * math.pi * Ksafe ** 2))
    amp[K == 0] = 0.0
    uh = []
    for _ in range(3):
        ph = rng.uniform(0, 2 * math.pi, size=K.shape)
        uh.append(amp * np.exp(1j * ph))
    # project onto divergence-free
    dot = (KX * uh[0] + KY * uh[1] + KZ * uh[2]) / np.where(K2 == 0, 1.0, K2)
    uh = [uh[0] - KX * dot, uh[1] - KY * dot, uh[2] - KZ * dot]
    vel = [np.fft.irfftn(h, s=(n, n, n), axes=(0, 1, 2)) for h in uh]
    gamma = 1.4
    c0 = 1.0  # rho = 1, p = 1/gamma
    urms = math.sqrt(float(np.mean(vel[0] ** 2 + vel[1] ** 2 + vel[2] ** 2)))
    scale = mach_t * c0 / urms
    vel = [v * scale for v in vel]
    # vorticity magnitude from spectral derivatives
    om2 = 0.0
    wh = [np.fft.rfftn(v) for v in vel]
    cx = 1j * KY * wh[2] - 1j * KZ * wh[1]
    cy = 1j * KZ * wh[0] - 1j * KX * wh[2]
    cz = 1j * KX * wh[1] - 1j * KY * wh[0]
    for cc in (cx, cy, cz):
        om2 += float(np.mean(np.fft.irfftn(cc, s=(n, n, n)) ** 2))
    uprime = math.sqrt(float(np.mean(vel[0] ** 2 + vel[1] ** 2 + vel[2] ** 2)) / 3.0)
    lam = math.sqrt(15.0 * uprime ** 2 / om2)
    nu = uprime * lam / re_lambda
    reynolds = 1.0 / nu        # rho = 1, u_ref = c_0 = 1, L_ref = 1
    X, Y, Z = _mesh(3, (n, n, n), (0.0, 0.0, 0.0), (L, L, L), endpoint=False)
    rho = np.ones_like(X)
    p = np.ones_like(X)  # p_S = gamma * (1/gamma)
    c = Case(dim=3, order=order, ni=n, nj=n, nk=n, x=X, y=Y, z=Z, rho=rho, u=vel[0], v=vel[1],
             w=vel[2], p=p, time_order=time_order, mach=1.0, reynolds=reynolds, gamma=gamma,
             periodic=(True, True, True), period=(L, L, L), name=f"turb{n}_w{order}")
    c.tau = cfl_tau(c)
    return c


def taylor_green_2d(n: int = 64, order: int = 5, mach: float = 0.1, reynolds: float = 1600.0,
                    time_order: int = 4) -> Case:
    """2D Taylor-Green vortex on the uniform periodic [0,2pi)^2: u = sin x cos y,
    v = -cos x sin y, p_S = 1 + gamma Ma^2 (cos 2x + cos 2y)/4, isothermal rho."""
    L = 2 * math.pi
    X, Y, Z = _mesh(2, (n, n, 1), (0.0, 0.0, 0.0), (L, L, 1.0), endpoint=False)
    gamma = 1.4
    u = np.sin(X) * np.cos(Y)
    v = -np.cos(X) * np.sin(Y)
    p = 1.0 + gamma * mach ** 2 * (np.cos(2 * X) + np.cos(2 * Y)) / 4.0
    c = Case(dim=2, order=order, ni=n, nj=n, nk=1, x=X, y=Y, z=Z, rho=p.copy(), u=u, v=v,
             w=np.zeros_like(X), p=p, time_order=time_order, mach=mach, reynolds=reynolds, gamma=gamma,
             periodic=(True, True, False), period=(L, L, 1.0), name=f"tgv2d{n}_w{order}")
    c.tau = cfl_tau(c)
    return c


def vortex_column(n: int, nz: int, beta: float, mach_inf: float, order: int = 5, length: float = 10.0,
                  inviscid: bool = False, reynolds: float = 1e4, time_order: int = 4) -> Case:
    """The 2D isentropic vortex extruded along z (w = 0) on a periodic
    [0,L)^2 x [0,L nz/n) box with n x n x nz points."""
    v2 = isentropic_vortex(n, beta, mach_inf, order=order, length=length, inviscid=inviscid,
                           reynolds=reynolds, time_order=time_order)
    h = length / n
    X, Y, Z = _mesh(3, (n, n, nz), (0.0, 0.0, 0.0), (length, length, h * nz), endpoint=False)
    rep = lambda a: np.repeat(a[:, :, :1], nz, axis=2)
    c = Case(dim=3, order=order, ni=n, nj=n, nk=nz, x=X, y=Y, z=Z, rho=rep(v2.rho), u=rep(v2.u),
             v=rep(v2.v), w=np.zeros_like(X), p=rep(v2.p), time_order=time_order, mach=1.0,
             reynolds=reynolds, gamma=v2.gamma, inviscid=inviscid, periodic=(True, True, True),
             period=(length, length, h * nz), name=f"vcol{n}x{nz}")
    c.tau = cfl_tau(c)
    return c


def serving_stream(count: int, seed: int = 5, rate: float = 200.0, min_points: int = 32 ** 2,
                   max_points: int = 128 ** 3):
    """Seeded solve requests for the serving workload: Poisson arrivals at
    `rate` per second; total points log-uniform in [min_points, max_points],
    half 2D (n x n) and half 3D (n^3); Taylor-Green or isentropic vortex;
    Mach U[0.1, 0.6], Re U[100, 5000], WENO5 or WENO9, 20..500 steps.
    Returns a list of (arrival time s, case, nsteps)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for _ in range(count):
        t += float(rng.exponential(1.0 / rate))
        pts = math.exp(rng.uniform(math.log(min_points), math.log(max_points)))
        dim = 2 if rng.uniform() < 0.5 else 3
        order = 5 if rng.uniform() < 0.5 else 9
        tgv = rng.uniform() < 0.5
        mach = float(rng.uniform(0.1, 0.6))
        re = float(rng.uniform(100.0, 5000.0))
        nsteps = int(rng.integers(20, 501))
        beta = float(rng.uniform(1.0, 5.0))
        if dim == 2:
            n = max(order + 3, int(round(math.sqrt(pts))))
            case = taylor_green_2d(n, order, mach, re) if tgv else \
                isentropic_vortex(n, beta, mach, order=order, inviscid=False, reynolds=re)
        else:
            n = max(order + 3, int(round(pts ** (1.0 / 3.0))))
            case = taylor_green(n, order, mach, re, perturb=0.0) if tgv else \
                vortex_column(n, n, beta, mach, order=order, reynolds=re)
        out.append((t, case, nsteps))
    return out


@dataclasses.dataclass
class Division:
    """A Cartesian division of one block into parts[0] x parts[1] (x parts[2])
    blocks, as SHOCK's .sddc division files describe one (the layout
    TOOLS/generatedivfile/generatedivfile_3.c writes): block rank
    r = (k * parts[1] + j) * parts[0] + i, each with its real-point slice of
    the case, the block across each face (Left, Right, Bottom, Top, Behind,
    InFront; -1 at a face of the whole block that is not periodic, which
    keeps the case's face type) and the float32 Translation the face adds to
    coordinates it receives (minus / plus the period where a periodic axis
    wraps around)."""
    case: Case
    parts: Tuple[int, int, int]
    blocks: list                    # Case per block (sizes, fields; periodic False; bc on outer faces)
    neighbour: np.ndarray           # (nblocks, 6) int
    translation: np.ndarray         # (nblocks, 6, 3) float32
    lo: np.ndarray                  # (nblocks, 3) first real index of each block in the whole block
    transform: Optional[np.ndarray] = None   # (nblocks, 6, 3) int: the .sddc Transform per face (1,2,3)
    axes: Optional[np.ndarray] = None        # (nblocks, 3) int: the whole block's axis each block axis runs along
    flips: Optional[np.ndarray] = None       # (nblocks, 3) bool: ... and whether it runs the other way

    def __post_init__(self):
        nb = len(self.blocks)
        if self.axes is None:
            self.axes = np.tile(np.arange(3), (nb, 1))
            self.flips = np.zeros((nb, 3), dtype=bool)
        if self.transform is None:
            self.transform = _transforms(self.neighbour, self.axes, self.flips, self.case.dim)

    def to_block(self, b, a):
        """Array a of the whole block's shape (..., ni, nj, nk) seen from
        block b's index order (its slice, then its axes as it holds them)."""
        bl = self.blocks[b]
        n = (bl.ni, bl.nj, bl.nk if self.case.dim == 3 else 1)
        sl = [slice(None)] * (a.ndim - 3)
        whole = [None, None, None]
        for c in range(3):
            ax = self.axes[b, c]
            whole[ax] = slice(int(self.lo[b, ax]), int(self.lo[b, ax]) + n[c])
        s = a[tuple(sl + whole)]
        lead = a.ndim - 3
        s = np.transpose(s, list(range(lead)) + [lead + int(x) for x in self.axes[b]])
        for c in range(3):
            if self.flips[b, c]:
                s = np.flip(s, axis=lead + c)
        return s

    def from_block(self, b, a):
        """Block b's real-point array (..., its own index order) in the whole
        block's axis order (the inverse of to_block's reordering)."""
        lead = a.ndim - 3
        for c in range(3):
            if self.flips[b, c]:
                a = np.flip(a, axis=lead + c)
        inv = [int(np.nonzero(self.axes[b] == w)[0][0]) for w in range(3)]
        return np.transpose(a, list(range(lead)) + [lead + c for c in inv])


def write_division(division: "Division", path: str, zone: str = "zone"):
    """Write the division as a SHOCK .sddc file (the layout loadDivision
    reads, src/Load.c:191-250, little-endian, which SHOCK reads unswapped on
    x86): per rank the zone name, the block's first and last point in the
    whole block, and per face
    the neighbour (1-based, 0 for none), the Transform, this side's and the
    donor's point ranges (block-local, 1-based), rotation centre and angle
    (zero) and the Translation."""
    import struct
    dim = division.case.dim
    rows = []
    for b, bl in enumerate(division.blocks):
        n = (bl.ni, bl.nj, bl.nk)[:dim]
        lo = [int(division.lo[b, int(division.axes[b, c])]) for c in range(dim)]
        row = zone.encode()[:32].ljust(32, b"\0")
        row += struct.pack(f"<{2 * dim}q", *[lo[c] + 1 for c in range(dim)], *[lo[c] + n[c] for c in range(dim)])
        for f in range(2 * dim):
            nb = int(division.neighbour[b, f])
            t = [int(x) for x in division.transform[b, f][:dim]]
            rng = [1] * dim + list(n)
            drng = [0] * (2 * dim)
            if nb >= 0:
                a, hi = f // 2, f % 2
                rng[a] = rng[dim + a] = n[a] if hi else 1
                dn = (division.blocks[nb].ni, division.blocks[nb].nj, division.blocks[nb].nk)[:dim]
                da, dhi = abs(t[a]) - 1, hi ^ (1 if t[a] > 0 else 0)
                drng = [1] * dim + list(dn)
                drng[da] = drng[dim + da] = dn[da] if dhi else 1
            else:
                t = [0] * dim
                rng = [0] * (2 * dim)
            row += struct.pack(f"<i{dim}i{2 * dim}q{2 * dim}q9f", nb + 1 if nb >= 0 else 0, *t, *rng, *drng,
                               0.0, 0.0, 0.0, 0.0, 0.0, 0.0, *[float(x) for x in division.translation[b, f]])
        rows.append(row)
    with open(path, "wb") as fh:
        fh.write(b"".join(rows))


def load_division(case: Case, path: str, nranks: int, swap: bool = False) -> "Division":
    """The division a SHOCK .sddc file describes over the one zone ``case``
    holds (its grid and fields, all rows naming that zone), as SHOCK's ranks
    take it (src/Load.c:191-250, 355-400): rank r's block is the case's real
    points between the row's corners, its neighbours, Translations and
    Transforms are the row's (read by the library's shock_read_division), and
    a face without a neighbour keeps the case's face type.  The zone's axes
    must be every block's axes (Transforms of +-1, +-2, +-3 in place, as
    TOOLS/generatedivfile writes them)."""
    from . import read_division
    nb, tr, tf, co, sz = read_division(path, case.dim, nranks, swap=swap)
    n = (case.ni, case.nj, case.nk if case.dim == 3 else 1)
    lo = co[:, :3] - 1
    blocks = []
    for r in range(nranks):
        sl = tuple(slice(int(lo[r, a]), int(co[r, 3 + a])) for a in range(3))
        if any(sl[a].start < 0 or sl[a].stop > n[a] for a in range(3)):
            raise ValueError(f"rank {r}: corners {co[r].tolist()} outside the {n} zone")
        bc = [0] * 6
        for f in range(2 * case.dim):
            if nb[r, f] < 0:
                bc[f] = case.bc[f]
            elif any(abs(int(tf[r, f, c])) != c + 1 for c in range(case.dim)):
                raise ValueError(f"rank {r} face {f}: Transform {tf[r, f, :case.dim].tolist()} re-orders the "
                                 "zone's axes; a rotated block needs its own orientation (rotate_block)")
        blocks.append(case.replace(ni=int(sz[r, 0]), nj=int(sz[r, 1]), nk=int(sz[r, 2]) if case.dim == 3 else 1,
                                   x=case.x[sl], y=case.y[sl], z=case.z[sl], rho=case.rho[sl], u=case.u[sl],
                                   v=case.v[sl], w=case.w[sl], p=case.p[sl], periodic=(False, False, False),
                                   bc=tuple(bc), name=f"{case.name}_b{r}"))
    parts = tuple(len(np.unique(lo[:, a])) for a in range(3))
    return Division(case=case, parts=parts, blocks=blocks, neighbour=nb, translation=tr, lo=lo, transform=tf)


def _transforms(neigh, axes, flips, dim):
    """The .sddc Transform of every interface from the blocks' orientations:
    entry c of face f of block b is +-(1 + the axis of the neighbour that b's
    axis c runs along), negative where the two run opposite ways."""
    nb = neigh.shape[0]
    t = np.zeros((nb, 6, 3), dtype=np.int32)
    for b in range(nb):
        for f in range(2 * dim):
            n = neigh[b, f]
            if n < 0:
                continue
            for c in range(3):
                d = int(np.nonzero(axes[n] == axes[b, c])[0][0])
                s = -1 if flips[b, c] != flips[n, d] else 1
                t[b, f, c] = s * (d + 1)
    return t


def rotate_block(division: "Division", b: int, axes: Tuple[int, int, int], flips: Tuple[bool, bool, bool]):
    """The same division with block b holding its points in another index
    order: its new axis c runs along its old axis axes[c], reversed where
    flips[c] (a zone meshed in another orientation, as a .sddc file with
    non-identity Transforms describes one).  Faces, neighbours, face types,
    translations and every interface's Transform follow."""
    import copy
    d = copy.copy(division)
    dim = d.case.dim
    axes = tuple(int(a) for a in axes)
    flips = tuple(bool(x) for x in flips)
    old = d.blocks[b]
    nold = (old.ni, old.nj, old.nk if dim == 3 else 1)

    def re(a):
        s = np.transpose(np.asarray(a), axes)
        for c in range(3):
            if flips[c]:
                s = np.flip(s, axis=c)
        return np.ascontiguousarray(s)

    neigh = d.neighbour.copy()
    trans = d.translation.copy()
    bc = list(old.bc)
    for c in range(3):
        for side in (0, 1):
            of = 2 * axes[c] + (side ^ int(flips[c]))
            neigh[b, 2 * c + side] = division.neighbour[b, of]
            trans[b, 2 * c + side] = division.translation[b, of]
            bc[2 * c + side] = old.bc[of]
    new = old.replace(ni=nold[axes[0]], nj=nold[axes[1]], nk=nold[axes[2]] if dim == 3 else 1,
                      x=re(old.x), y=re(old.y), z=re(old.z), rho=re(old.rho), u=re(old.u), v=re(old.v),
                      w=re(old.w), p=re(old.p), bc=tuple(bc))
    blocks = list(d.blocks)
    blocks[b] = new
    ax = d.axes.copy()
    fl = d.flips.copy()
    ax[b] = [division.axes[b, axes[c]] for c in range(3)]
    fl[b] = [bool(division.flips[b, axes[c]]) ^ flips[c] for c in range(3)]
    return Division(case=d.case, parts=d.parts, blocks=blocks, neighbour=neigh, translation=trans, lo=d.lo,
                    axes=ax, flips=fl)


def split(case: Case, parts: Tuple[int, ...]) -> Division:
    parts = tuple(parts) + (1,) * (3 - len(parts))
    if case.dim == 2:
        parts = (parts[0], parts[1], 1)
    n = (case.ni, case.nj, case.nk if case.dim == 3 else 1)
    cuts = []
    for a in range(3):
        q, r = divmod(n[a], parts[a])
        sizes = [q + (1 if i < r else 0) for i in range(parts[a])]
        cuts.append(np.concatenate([[0], np.cumsum(sizes)]).astype(int))
    nb = parts[0] * parts[1] * parts[2]
    neigh = -np.ones((nb, 6), dtype=np.int32)
    trans = np.zeros((nb, 6, 3), dtype=np.float32)
    lo = np.zeros((nb, 3), dtype=np.int64)
    blocks = []
    for k in range(parts[2]):
        for j in range(parts[1]):
            for i in range(parts[0]):
                r = (k * parts[1] + j) * parts[0] + i
                idx = (i, j, k)
                sl = tuple(slice(cuts[a][idx[a]], cuts[a][idx[a] + 1]) for a in range(3))
                lo[r] = [cuts[a][idx[a]] for a in range(3)]
                bc = [0] * 6
                for a in range(case.dim):
                    for side in (0, 1):
                        f = 2 * a + side
                        m = list(idx)
                        m[a] += 1 if side else -1
                        if 0 <= m[a] < parts[a]:
                            neigh[r, f] = (m[2] * parts[1] + m[1]) * parts[0] + m[0]
                        elif case.periodic[a]:
                            m[a] %= parts[a]
                            neigh[r, f] = (m[2] * parts[1] + m[1]) * parts[0] + m[0]
                            trans[r, f, a] = np.float32(case.period[a] if side else -case.period[a])
                        else:
                            bc[f] = case.bc[f]
                sub = case.replace(ni=int(sl[0].stop - sl[0].start), nj=int(sl[1].stop - sl[1].start),
                                   nk=int(sl[2].stop - sl[2].start) if case.dim == 3 else 1,
                                   x=case.x[sl], y=case.y[sl], z=case.z[sl], rho=case.rho[sl], u=case.u[sl],
                                   v=case.v[sl], w=case.w[sl], p=case.p[sl], periodic=(False, False, False),
                                   bc=tuple(bc), name=f"{case.name}_b{r}")
                blocks.append(sub)
    return Division(case=case, parts=parts, blocks=blocks, neighbour=neigh, translation=trans, lo=lo)
