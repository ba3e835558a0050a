"""ctypes bindings for the oracle libraries (test infrastructure only).

* ``RefSolver`` drives SHOCK's own CPU code (oracle/_ref/libshockref_*.so,
  built by oracle/Makefile from the unmodified reference sources) through
  ref_harness.c.
* ``Oracle`` drives the CPU restatement (oracle/liboracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module, as the checker.  The shipped library never imports it.

Array conventions (both bindings): ghosted SoA fields, C order with k
fastest, index ijk = i*NJg*NKg + j*NKg + k (src/Functions.c:2306); 2D uses
NKg = 1.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_dp = C.POINTER(C.c_double)


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


class RefParams(C.Structure):
    _fields_ = [
        ("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int),
        ("time_order", C.c_int),
        ("tau", C.c_double), ("mach", C.c_double), ("reynolds", C.c_double),
        ("prandtl", C.c_double), ("gamma", C.c_double), ("gas_r", C.c_double),
        ("t0", C.c_double), ("l0", C.c_double),
        ("inviscid", C.c_int), ("mms", C.c_int), ("mms_case", C.c_int),
        ("periodic", C.c_int * 3), ("period", C.c_double * 3),
        ("bc", C.c_int * 6), ("t_wall", C.c_double),
        ("rho_inflow", C.c_double), ("p_inflow", C.c_double), ("p_outflow", C.c_double),
        ("u_inflow", C.c_double * 3),
    ]


def ref_available(order: int, dim: int, extended: bool = False, full: bool = False) -> bool:
    tag = "80" if extended else ""
    name = "libshockreffull" if full else "libshockref"
    return os.path.exists(os.path.join(HERE, "_ref", f"{name}{tag}_w{order}_{dim}d.so"))


def dropin_available(order: int, dim: int) -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", f"libshockdropin_w{order}_{dim}d.so"))


class RefSolver:
    """One block of SHOCK's reference solver (one library per order/dim)."""

    _libs: dict = {}

    def __init__(self, case, extended=False, external=None, _lib="libshockref", full=False):
        """extended=True loads the PRECISION=3 (80-bit long double) build.
        external=(exact9, js5): manufactured solution given as arrays on the
        ghosted block (the build with ref_harness/mms_external.c).
        full=True: the build that keeps the 3D metric's cross derivatives
        (src/Functions.c:6479-6484 left out, 3D only)."""
        self.case = case
        if full:
            _lib = "libshockreffull"
        tag = "80" if extended else ("x" if external is not None else "")
        key = (case.order, case.dim, _lib + tag)
        if key not in RefSolver._libs:
            path = os.path.join(HERE, "_ref", f"{_lib}{tag}_w{case.order}_{case.dim}d.so")
            if not os.path.exists(path):
                raise FileNotFoundError(path + " (run make -C oracle ref)")
            lib = C.CDLL(path, mode=os.RTLD_LOCAL)
            lib.ref_init.restype = C.c_int
            lib.ref_time_steps.restype = C.c_double
            RefSolver._libs[key] = lib
        self.lib = RefSolver._libs[key]
        p = RefParams()
        p.ni, p.nj, p.nk = case.ni, case.nj, (case.nk if case.dim == 3 else 1)
        p.time_order = case.time_order
        p.tau, p.mach, p.reynolds = case.tau, case.mach, case.reynolds
        p.prandtl, p.gamma, p.gas_r, p.t0, p.l0 = case.prandtl, case.gamma, case.gas_r, case.t0, case.l0
        p.inviscid = int(case.inviscid)
        p.mms = 1 if (case.mms == "reference" or external is not None) else 0
        p.mms_case = case.mms_case
        for a in range(3):
            p.periodic[a] = int(case.periodic[a])
            p.period[a] = case.period[a]
        for f in range(6):
            p.bc[f] = int(getattr(case, "bc", (0,) * 6)[f])
        p.t_wall = float(getattr(case, "t_wall", 1.0))
        p.rho_inflow = float(getattr(case, "rho_inflow", 1.0))
        p.p_inflow = float(getattr(case, "p_inflow", 1.0))
        p.p_outflow = float(getattr(case, "p_outflow", 1.0))
        for a in range(3):
            p.u_inflow[a] = float(getattr(case, "u_inflow", (0.0, 0.0, 0.0))[a])
        self.params = p
        f = lambda a: np.ascontiguousarray(np.asarray(a, np.float64).transpose(2, 1, 0)).ravel()
        x, y, z, u, v, w, pr, rho = (f(a) for a in case.real_fields())
        self._keep = (x, y, z, u, v, w, pr, rho)
        if external is not None:
            ex = np.ascontiguousarray(external[0], np.float64).ravel()
            js = np.ascontiguousarray(external[1], np.float64).ravel()
            self.lib.ref_set_external(_ptr(ex), _ptr(js), C.c_size_t(ex.size // 9))
        rc = self.lib.ref_init(C.byref(p), _ptr(x), _ptr(y), _ptr(z), _ptr(u), _ptr(v),
                               _ptr(w), _ptr(pr), _ptr(rho))
        assert rc == 0
        d = (C.c_int * 6)()
        self.lib.ref_dims(d)
        self.shape = (d[0], d[1], d[2])
        self.start = (d[3], d[4], d[5])
        self.n = d[0] * d[1] * d[2]

    def rhs(self) -> np.ndarray:
        q = np.zeros(5 * self.n)
        self.lib.ref_rhs(_ptr(q))
        return q.reshape((5,) + self.shape)

    def steps(self, n: int):
        self.lib.ref_steps(C.c_int(n))

    def time_steps(self, n: int) -> float:
        return self.lib.ref_time_steps(C.c_int(n))

    def control_loop(self, nsteps, nan_at=0, decel=0.7, accel_every=0, accel=1.1, backup_every=5) -> int:
        """startSimulation's control around the step (ref_harness.c
        control_loop): NaN check and reset from the last backup with
        tau *= decel, tau *= accel every accel_every iterations, a NaN
        planted at iteration nan_at.  Returns the number of resets."""
        f = getattr(self.lib, self._loop_fn)
        f.restype = C.c_int
        f.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int, C.c_double, C.c_int]
        return f(nsteps, nan_at, decel, accel_every, accel, backup_every)

    _loop_fn = "ref_control_loop"

    def tau(self) -> float:
        self.lib.ref_tau.restype = C.c_double
        return self.lib.ref_tau()

    def state(self, which: int = 0) -> np.ndarray:
        """rho,u,v,w,e,p,T,c,mue of U_RK (0) or U_lastStep (1)."""
        s = np.zeros(9 * self.n)
        self.lib.ref_get_state(_ptr(s), C.c_int(which))
        return s.reshape((9,) + self.shape)

    def set_state(self, prim5: np.ndarray):
        a = np.ascontiguousarray(prim5, dtype=np.float64).ravel()
        assert a.size == 5 * self.n
        self.lib.ref_set_state(_ptr(a))

    def set_last_pressure(self, p: np.ndarray):
        """p of U_lastStep (ghosted)."""
        a = np.ascontiguousarray(p, dtype=np.float64).ravel()
        assert a.size == self.n
        self.lib.ref_set_last_p(_ptr(a))

    def geometry(self) -> np.ndarray:
        """x,y,z,J,xi_x,xi_y,xi_z,eta_x,eta_y,eta_z,zeta_x,zeta_y,zeta_z."""
        g = np.zeros(13 * self.n)
        self.lib.ref_get_geom(_ptr(g))
        return g.reshape((13,) + self.shape)

    def post(self) -> np.ndarray:
        """SHOCK's CalcValuesForPost on U_lastStep: Mach number, |grad rho|,
        lambda2 (3 fields, ghosted)."""
        q = np.zeros(3 * self.n)
        self.lib.ref_post(_ptr(q))
        return q.reshape((3,) + self.shape)

    def probe_points(self, xyz):
        """SHOCK's placement of PressureHistory probes at the n x 3
        locations xyz (preparePressureHistoryValues): (ghosted linear index
        of the chosen point, whether this block records the probe) each."""
        xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
        n = len(xyz)
        ijk = np.zeros(n, np.int32)
        flag = np.zeros(n, np.int32)
        self.lib.ref_probe_points(C.c_int(n), _ptr(xyz), ijk.ctypes.data_as(C.POINTER(C.c_int)),
                                  flag.ctypes.data_as(C.POINTER(C.c_int)))
        return ijk, flag

    def mms_source(self) -> np.ndarray:
        """J*S of the reference manufactured-solution source (5 fields)."""
        q = np.zeros(5 * self.n)
        self.lib.ref_mms_source(_ptr(q))
        return q.reshape((5,) + self.shape)

    def mms_exact(self) -> np.ndarray:
        """Exact solution at every ghosted point after set-up (9 fields)."""
        return self.state(1)


class DropinSolver(RefSolver):
    """SHOCK's own set-up and time loop (ref_harness.c) running its time
    steps on the GPU through the SHOCK-side binding shock_b200/dropin/GPU.c:
    GPU_Create after the set-up, GPU_CalcRungeKutta in place of
    CalcRungeKutta, GPU_SyncHost before the host reads U_RK
    (oracle/_ref/libshockdropin_*.so, linked with libshock_b200.so)."""

    _loop_fn = "ref_dropin_control_loop"

    def __init__(self, case, device: int = 0):
        super().__init__(case, _lib="libshockdropin")
        rc = self.lib.ref_dropin_create(C.c_int(device))
        if rc != 0:
            raise RuntimeError(f"GPU_Create returned {rc}")

    def steps(self, n: int):
        self.lib.ref_dropin_steps(C.c_int(n))

    def sync(self):
        self.lib.ref_dropin_sync()

    def close(self):
        self.lib.ref_dropin_destroy()


class OcParams(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("order", C.c_int),
        ("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int),
        ("time_order", C.c_int),
        ("tau", C.c_double), ("mach", C.c_double), ("reynolds", C.c_double),
        ("prandtl", C.c_double), ("gamma", C.c_double), ("gas_r", C.c_double),
        ("t0", C.c_double), ("l0", C.c_double),
        ("inviscid", C.c_int), ("mms", C.c_int),
        ("periodic", C.c_int * 3), ("period", C.c_double * 3),
    ]


_oclib = None


def _oracle_lib():
    global _oclib
    if _oclib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (run make -C oracle)")
        lib = C.CDLL(path)
        lib.oc_create.restype = C.c_void_p
        for name in ("oc_dims", "oc_set_dirichlet", "oc_set_source", "oc_set_state",
                     "oc_get_state", "oc_get_geom", "oc_rhs", "oc_steps", "oc_free"):
            getattr(lib, name).argtypes = None
        lib.oc_set_weno_eps.argtypes = [C.c_void_p, C.c_double]
        _oclib = lib
    return _oclib


class Oracle:
    """The CPU restatement, same calling convention as RefSolver."""

    def __init__(self, case, dirichlet9=None, source5=None, weno_eps=0.0):
        if any(getattr(case, "bc", (0,) * 6)):
            raise ValueError("the CPU restatement covers periodic and manufactured-solution faces only")
        lib = self.lib = _oracle_lib()
        p = OcParams()
        p.dim, p.order = case.dim, case.order
        p.ni, p.nj, p.nk = case.ni, case.nj, (case.nk if case.dim == 3 else 1)
        p.time_order = case.time_order
        p.tau, p.mach, p.reynolds = case.tau, case.mach, case.reynolds
        p.prandtl, p.gamma, p.gas_r, p.t0, p.l0 = case.prandtl, case.gamma, case.gas_r, case.t0, case.l0
        p.inviscid = int(case.inviscid)
        p.mms = 0 if case.mms == "none" else 1
        for a in range(3):
            p.periodic[a] = int(case.periodic[a])
            p.period[a] = case.period[a]
        f = lambda a: np.ascontiguousarray(np.asarray(a, np.float64).transpose(2, 1, 0)).ravel()
        arrs = [f(a) for a in case.real_fields()]
        self.h = C.c_void_p(lib.oc_create(C.byref(p), *[_ptr(a) for a in arrs]))
        d = (C.c_int * 6)()
        lib.oc_dims(self.h, d)
        self.shape = (d[0], d[1], d[2])
        self.start = (d[3], d[4], d[5])
        self.n = d[0] * d[1] * d[2]
        if dirichlet9 is not None:
            a = np.ascontiguousarray(dirichlet9, np.float64).ravel()
            lib.oc_set_dirichlet(self.h, _ptr(a))
        if source5 is not None:
            a = np.ascontiguousarray(source5, np.float64).ravel()
            lib.oc_set_source(self.h, _ptr(a))
        if weno_eps > 0:
            lib.oc_set_weno_eps(self.h, C.c_double(weno_eps))

    def __del__(self):
        try:
            self.lib.oc_free(self.h)
        except Exception:
            pass

    def rhs(self):
        q = np.zeros(5 * self.n)
        self.lib.oc_rhs(self.h, _ptr(q))
        return q.reshape((5,) + self.shape)

    def steps(self, n):
        self.lib.oc_steps(self.h, C.c_int(n))

    def state(self, which=0):
        s = np.zeros(9 * self.n)
        self.lib.oc_get_state(self.h, _ptr(s), C.c_int(which))
        return s.reshape((9,) + self.shape)

    def set_state(self, prim5):
        a = np.ascontiguousarray(prim5, np.float64).ravel()
        self.lib.oc_set_state(self.h, _ptr(a))

    def geometry(self):
        g = np.zeros(13 * self.n)
        self.lib.oc_get_geom(self.h, _ptr(g))
        return g.reshape((13,) + self.shape)


# ---------------------------------------------------------------------------
# SHOCK's own code on several ranks (oracle/_ref/libshockmpi_*): the blocks of
# a division (shock_b200.cases.split) as the ranks of one run, exchanging
# their interfaces with SHOCK's TransferMeshParameter and
# TransferFlowParameterWithGhosts over the forked shared-memory stand-in for
# MPI (ref_harness/mpi_shm.c).  The ranks are forked from a fresh process
# started with multiprocessing's "spawn" method, so no GPU context is ever
# forked.
# ---------------------------------------------------------------------------
def multirank_available(order: int, dim: int, extended: bool = False, full: bool = False) -> bool:
    tag = ("full" if full else "") + ("80" if extended else "")
    return os.path.exists(os.path.join(HERE, "_ref", f"libshockmpi{tag}_w{order}_{dim}d.so"))


def _ref_params(case) -> "RefParams":
    p = RefParams()
    p.ni, p.nj, p.nk = case.ni, case.nj, (case.nk if case.dim == 3 else 1)
    p.time_order = case.time_order
    p.tau, p.mach, p.reynolds = case.tau, case.mach, case.reynolds
    p.prandtl, p.gamma, p.gas_r, p.t0, p.l0 = case.prandtl, case.gamma, case.gas_r, case.t0, case.l0
    p.inviscid = int(case.inviscid)
    p.mms = 0
    p.mms_case = 0
    for a in range(3):
        p.periodic[a] = 0
        p.period[a] = 0.0
    for f in range(6):
        p.bc[f] = int(case.bc[f])
    p.t_wall = float(case.t_wall)
    p.rho_inflow, p.p_inflow, p.p_outflow = float(case.rho_inflow), float(case.p_inflow), float(case.p_outflow)
    for a in range(3):
        p.u_inflow[a] = float(case.u_inflow[a])
    return p


def _multirank_worker(division, nsteps, rhs, extended, full=False, division_file=None, swap=0):
    case = division.case
    tag = ("full" if full else "") + ("80" if extended else "")
    lib = C.CDLL(os.path.join(HERE, "_ref", f"libshockmpi{tag}_w{case.order}_{case.dim}d.so"), mode=os.RTLD_LOCAL)
    lib.refmpi_run.restype = C.c_int
    lib.refmpi_run_file.restype = C.c_int
    nb = len(division.blocks)
    g2 = case.order + 1
    shapes = [(b.ni + g2, b.nj + g2, (b.nk + g2) if case.dim == 3 else 1) for b in division.blocks]
    ng = [s[0] * s[1] * s[2] for s in shapes]
    off = np.zeros(nb, dtype=np.uint64)
    for b in range(1, nb):
        off[b] = off[b - 1] + 27 * ng[b - 1]
    total = int(off[-1]) + 27 * ng[-1]
    params = (RefParams * nb)(*[_ref_params(b) for b in division.blocks])
    f = lambda a: np.ascontiguousarray(np.asarray(a, np.float64).transpose(2, 1, 0)).ravel()
    keep = [[f(a) for a in b.real_fields()] for b in division.blocks]
    ptrs = (C.POINTER(C.c_double) * (8 * nb))(*[_ptr(a) for fl in keep for a in fl])
    neigh = np.ascontiguousarray(division.neighbour, dtype=np.int32)
    trans = np.ascontiguousarray(division.translation, dtype=np.float32)
    tfm = np.ascontiguousarray(division.transform, dtype=np.int32)
    out = np.zeros(total)
    face = max(max(s[0] * s[1], s[1] * s[2], s[0] * s[2]) for s in shapes)
    slot = 13 * (g2 // 2) * face * 16       # long double in the 80-bit build
    path = None if division_file is None else os.fsencode(str(division_file))
    comm = np.zeros(nb)
    rc = lib.refmpi_run_file(C.c_int(nb), params, neigh.ctypes.data_as(C.POINTER(C.c_int)),
                             trans.ctypes.data_as(C.POINTER(C.c_float)), tfm.ctypes.data_as(C.POINTER(C.c_int)), ptrs,
                             C.c_int(int(rhs)), C.c_int(nsteps),
                             _ptr(out), off.ctypes.data_as(C.POINTER(C.c_size_t)), C.c_size_t(total),
                             C.c_size_t(slot), C.c_char_p(path), C.c_int(swap), _ptr(comm))
    if rc != 0:
        raise RuntimeError(f"multi-rank reference run failed ({rc})")
    res = []
    for b in range(nb):
        o, n = int(off[b]), ng[b]
        res.append({"geometry": out[o:o + 13 * n].reshape((13,) + shapes[b]),
                    "rhs": out[o + 13 * n:o + 18 * n].reshape((5,) + shapes[b]),
                    "state": out[o + 18 * n:o + 27 * n].reshape((9,) + shapes[b]),
                    "comm_time": float(comm[b])})
    return res


def run_multirank(division, nsteps: int, rhs: bool = False, extended: bool = False, full: bool = False,
                  division_file=None, swap: int = 0):
    """Per block: geometry (13, ghosted), one right-hand side at the initial
    state (5, when rhs) and the state after nsteps steps (9: rho,u,v,w,e,p,
    T,c,mue) of SHOCK's own multi-rank run of the division, and the seconds
    SHOCK counted in its halo exchange during the steps (comm_time, waits
    for the neighbours included) (extended: the
    80-bit build; full: the build with the full 3D metric).  With
    division_file, each rank reads its interfaces from that .sddc file with
    SHOCK's own loadDivision (src/Load.c:191-250; swap: its SwapDivFile
    option, 0 auto, 1 never, 2 always) instead of from the division's
    neighbour, translation and transform tables; the blocks' sizes and
    fields still come from the division."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        return pool.apply(_multirank_worker, (division, nsteps, rhs, extended, full, division_file, swap))


class RefIface(C.Structure):
    """One face's interface as SHOCK's loadDivision reads it
    (ref_harness/load_division.c)."""
    _fields_ = [("neighbour", C.c_int), ("transform", C.c_int * 3), ("range", C.c_longlong * 6),
                ("drange", C.c_longlong * 6), ("rc", C.c_float * 3), ("ra", C.c_float * 3), ("tr", C.c_float * 3)]


_ROW_READERS = {}


def _row_reader(dim):
    if dim not in _ROW_READERS:
        lib = C.CDLL(os.path.join(HERE, "_ref", f"libshockmpi_w5_{dim}d.so"), mode=os.RTLD_LOCAL)
        lib.ref_load_division_row.restype = C.c_int
        _ROW_READERS[dim] = lib
    return _ROW_READERS[dim]


def generator_path():
    """SHOCK's division-file generator built from its sources, or None."""
    p = os.path.join(HERE, "_ref", "generatedivfile_3")
    return p if os.path.exists(p) else None


def load_division_row(path, dim: int, rank: int, nranks: int, swap: int = 0):
    """One rank's row of a .sddc file as SHOCK's own loadDivision reads it
    (src/Load.c:191-250; swap: its SwapDivFile option): (corners (6,),
    per face (neighbour 1-based or 0, transform (3,), range (2*dim,), drange
    (2*dim,), translation (3,))).  In process: the file's size must be nranks rows,
    which the caller checks first (loadDivision ends the process otherwise)."""
    lib = _row_reader(dim)
    corners = (C.c_longlong * 6)()
    faces = (RefIface * 6)()
    ni = lib.ref_load_division_row(os.fsencode(str(path)), C.c_int(rank), C.c_int(nranks), C.c_int(swap), corners,
                                   faces)
    if ni < 0:
        raise RuntimeError("ref_load_division_row failed")
    out = []
    for f in range(2 * dim):
        x = faces[f]
        # ranges as SHOCK holds them: the first point per axis, then the last
        rng = np.array(x.range[:dim] + x.range[3:3 + dim])
        drng = np.array(x.drange[:dim] + x.drange[3:3 + dim])
        out.append((x.neighbour, np.array(x.transform[:]), rng, drng, np.array(x.tr[:], dtype=np.float32)))
    return np.array(corners[:]), out


CONFIG_DOUBLES = ("time_order", "tau", "mach", "reynolds", "prandtl", "gamma", "gas_r", "t0", "l0", "t_wall",
                  "rho_inflow", "p_inflow", "p_outflow", "u_inflow", "v_inflow", "w_inflow")
CONFIG_FLAGS = ("inviscid", "mms", "swap_div_file", "inflow_normal_subsonic", "inflow_riemann_subsonic",
                "inflow_isentrop_subsonic", "inflow_normal_supersonic", "outflow_normal_subsonic",
                "outflow_riemann_subsonic", "outflow_rudy_subsonic")


def config_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libshockini_3d.so"))


def _config_import_child(path):
    lib = C.CDLL(os.path.join(HERE, "_ref", "libshockini_3d.so"), mode=os.RTLD_LOCAL)
    d = (C.c_double * 16)()
    i = (C.c_int * 10)()
    if lib.ref_config_import(os.fsencode(str(path)), d, i) != 0:
        raise RuntimeError("ref_config_import failed")
    out = dict(zip(CONFIG_DOUBLES, d[:]))
    out.update(zip(CONFIG_FLAGS, i[:]))
    return out


def config_import(path) -> dict:
    """SHOCK's own reading of a config.ini (ConfigImport, src/Import.c:17-275,
    with its iniparser): the fields the library's shock_params_from_ini
    fills, and SHOCK's inflow/outflow option flags.  Runs in a child process,
    since SHOCK ends the process on a file iniparser rejects or on an
    inflow/outflow choice that does not name exactly one option each; then
    RuntimeError carries the end of its output."""
    import json
    import subprocess
    import sys
    code = ("import json, sys; sys.path.insert(0, sys.argv[1]); import refbind; "
            "print('CONFIG ' + json.dumps(refbind._config_import_child(sys.argv[2])))")
    r = subprocess.run([sys.executable, "-c", code, HERE, str(path)], capture_output=True, text=True, timeout=120)
    for line in r.stdout.splitlines():
        if r.returncode == 0 and line.startswith("CONFIG "):
            return json.loads(line[7:])
    raise RuntimeError(f"SHOCK's ConfigImport ended with {r.returncode}: {(r.stdout + r.stderr)[-400:]}")


def dropin_multirank_available(order: int, dim: int, real: bool = False) -> bool:
    tag = "real" if real else ""
    return os.path.exists(os.path.join(HERE, "_ref", f"libshockdropinmpi{tag}_w{order}_{dim}d.so"))


def _dropin_multirank_worker(division, nsteps, tau_at, tau_factor, nan, real=False):
    case = division.case
    os.environ["SHOCK_B200_LIB"] = os.path.join(os.path.dirname(HERE), "shock_b200", "libshock_b200.so")
    if nan is not None:
        os.environ["SHOCK_MOCK_NAN"] = f"{nan[0]} {nan[1]}"
    tag = "real" if real else ""
    lib = C.CDLL(os.path.join(HERE, "_ref", f"libshockdropinmpi{tag}_w{case.order}_{case.dim}d.so"),
                 mode=os.RTLD_LOCAL)
    lib.refmpi_dropin_run.restype = C.c_int
    nb = len(division.blocks)
    g2 = case.order + 1
    shapes = [(b.ni + g2, b.nj + g2, (b.nk + g2) if case.dim == 3 else 1) for b in division.blocks]
    ng = np.array([s[0] * s[1] * s[2] for s in shapes], dtype=np.uint64)
    off = np.zeros(nb, dtype=np.uint64)
    for b in range(1, nb):
        off[b] = off[b - 1] + 44 * ng[b - 1]
    total = int(off[-1] + 44 * ng[-1])
    params = (RefParams * nb)(*[_ref_params(b) for b in division.blocks])
    f = lambda a: np.ascontiguousarray(np.asarray(a, np.float64).transpose(2, 1, 0)).ravel()
    keep = [[f(a) for a in b.real_fields()] for b in division.blocks]
    ptrs = (C.POINTER(C.c_double) * (8 * nb))(*[_ptr(a) for fl in keep for a in fl])
    neigh = np.ascontiguousarray(division.neighbour, dtype=np.int32)
    trans = np.ascontiguousarray(division.translation, dtype=np.float32)
    tfm = np.ascontiguousarray(division.transform, dtype=np.int32)
    out = np.zeros(total)
    extra = np.zeros(nb + 17)
    face = max(max(s[0] * s[1], s[1] * s[2], s[0] * s[2]) for s in shapes)
    nr = [b.real_points for b in division.blocks]
    slot = max(13 * (g2 // 2) * face * 8, max(8 * (8 * r + 6 * int(n)) for r, n in zip(nr, ng)))
    rc = lib.refmpi_dropin_run(C.c_int(nb), params, neigh.ctypes.data_as(C.POINTER(C.c_int)),
                               trans.ctypes.data_as(C.POINTER(C.c_float)), tfm.ctypes.data_as(C.POINTER(C.c_int)),
                               ptrs, C.c_int(nsteps), C.c_int(tau_at), C.c_double(tau_factor), _ptr(out),
                               off.ctypes.data_as(C.POINTER(C.c_size_t)), ng.ctypes.data_as(C.POINTER(C.c_size_t)),
                               C.c_size_t(total), _ptr(extra), C.c_size_t(slot))
    if rc != 0:
        raise RuntimeError(f"drop-in multi-rank run failed ({rc})")
    res = []
    for b in range(nb):
        o, n = int(off[b]), int(ng[b])
        blk = out[o:o + 44 * n]
        res.append({"shock_geometry": blk[:13 * n].reshape((13,) + shapes[b]),
                    "initial": blk[13 * n:19 * n].reshape((6,) + shapes[b]),
                    "after_steps": blk[19 * n:25 * n].reshape((6,) + shapes[b]),
                    "after_upload_step": blk[25 * n:31 * n].reshape((6,) + shapes[b]),
                    "library_geometry": blk[31 * n:44 * n].reshape((13,) + shapes[b]),
                    "nan_steps": int(extra[b])})
    steps = int(extra[nb])
    taus = [float(t) for t in extra[nb + 1:nb + 17] if t != 0.0]
    return res, steps, taus


def run_dropin_multirank(division, nsteps: int, tau_at: int = -1, tau_factor: float = 1.0, nan=None,
                         real: bool = False):
    """The drop-in binding (shock_b200/dropin/GPU.c) in its division mode,
    inside SHOCK's own multi-rank set-up of the division, over the library's
    host test double (ref_harness/mock_shock.c), or with real=True over the
    library itself on rank 0's GPU; see refmpi_dropin_run.  nan = (step,
    block) plants a non-finite density in the double.  Returns (per block
    dict, the double's step count, the time steps it was given)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        return pool.apply(_dropin_multirank_worker, (division, nsteps, tau_at, tau_factor, nan, real))


def _dropin_multirank_histories_worker(division, np_, nv, xyz, nsteps, real=False, cpu=False):
    case = division.case
    os.environ["SHOCK_B200_LIB"] = os.path.join(os.path.dirname(HERE), "shock_b200", "libshock_b200.so")
    tag = "real" if real else ""
    lib = C.CDLL(os.path.join(HERE, "_ref", f"libshockdropinmpi{tag}_w{case.order}_{case.dim}d.so"),
                 mode=os.RTLD_LOCAL)
    lib.refmpi_dropin_histories.restype = C.c_int
    nb = len(division.blocks)
    per = np_ * (2 + nsteps) + nv * (2 + 3 * nsteps) + nsteps
    off = np.arange(nb, dtype=np.uint64) * np.uint64(per)
    params = (RefParams * nb)(*[_ref_params(b) for b in division.blocks])
    f = lambda a: np.ascontiguousarray(np.asarray(a, np.float64).transpose(2, 1, 0)).ravel()
    keep = [[f(a) for a in b.real_fields()] for b in division.blocks]
    ptrs = (C.POINTER(C.c_double) * (8 * nb))(*[_ptr(a) for fl in keep for a in fl])
    neigh = np.ascontiguousarray(division.neighbour, dtype=np.int32)
    trans = np.ascontiguousarray(division.translation, dtype=np.float32)
    tfm = np.ascontiguousarray(division.transform, dtype=np.int32)
    xyz = np.ascontiguousarray(xyz, np.float64)
    out = np.zeros(nb * per)
    g2 = case.order + 1
    shapes = [(b.ni + g2, b.nj + g2, (b.nk + g2) if case.dim == 3 else 1) for b in division.blocks]
    face = max(max(s[0] * s[1], s[1] * s[2], s[0] * s[2]) for s in shapes)
    ng = [s[0] * s[1] * s[2] for s in shapes]
    slot = max(13 * (g2 // 2) * face * 8, max(8 * (8 * b.real_points + 6 * n) for b, n in zip(division.blocks, ng)))
    rc = lib.refmpi_dropin_histories(C.c_int(nb), params, neigh.ctypes.data_as(C.POINTER(C.c_int)),
                                     trans.ctypes.data_as(C.POINTER(C.c_float)),
                                     tfm.ctypes.data_as(C.POINTER(C.c_int)), ptrs, C.c_int(np_), C.c_int(nv),
                                     _ptr(xyz), C.c_int(nsteps), _ptr(out),
                                     off.ctypes.data_as(C.POINTER(C.c_size_t)), C.c_size_t(out.size),
                                     C.c_size_t(slot), C.c_int(int(cpu)))
    if rc != 0:
        raise RuntimeError(f"drop-in multi-rank histories failed ({rc})")
    return out.reshape(nb, per)


def run_dropin_multirank_histories(division, np_: int, nv: int, xyz, nsteps: int, real: bool = False,
                                   cpu: bool = False):
    """The drop-in's division mode with device probe histories (over the
    test double, or with real=True over the library on rank 0's GPU; cpu=True:
    the same loop with SHOCK's own steps and writers): every rank places the
    locations xyz ((np_ + nv) x 3) with SHOCK's own prepare*HistoryValues and
    runs nsteps steps writing its histories.  Per rank: per pressure point
    its ijk, flag and nsteps pressures; per velocity point ijk, flag, 3 x
    nsteps velocities; then the nsteps times."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        return pool.apply(_dropin_multirank_histories_worker, (division, np_, nv, xyz, nsteps, real, cpu))


def mock_div_probe_value(b, f, o, s):
    """The test double's probe value of block b, field f (p, u, v, w) at
    ghosted point o after step s (ref_harness/mock_shock.c)."""
    return 100.0 * b + 1.0 + f + 0.01 * s + 1e-7 * float(o)


def _dropin_multirank_film_worker(division, nsamples, again, real, cpu):
    case = division.case
    os.environ["SHOCK_B200_LIB"] = os.path.join(os.path.dirname(HERE), "shock_b200", "libshock_b200.so")
    tag = "real" if real else ""
    lib = C.CDLL(os.path.join(HERE, "_ref", f"libshockdropinmpi{tag}_w{case.order}_{case.dim}d.so"),
                 mode=os.RTLD_LOCAL)
    lib.refmpi_dropin_film.restype = C.c_int
    nb = len(division.blocks)
    nr = [b.real_points for b in division.blocks]
    per = [8 * nsamples * n + nsamples for n in nr]
    off = np.zeros(nb, dtype=np.uint64)
    for b in range(1, nb):
        off[b] = off[b - 1] + per[b - 1]
    params = (RefParams * nb)(*[_ref_params(b) for b in division.blocks])
    f = lambda a: np.ascontiguousarray(np.asarray(a, np.float64).transpose(2, 1, 0)).ravel()
    keep = [[f(a) for a in b.real_fields()] for b in division.blocks]
    ptrs = (C.POINTER(C.c_double) * (8 * nb))(*[_ptr(a) for fl in keep for a in fl])
    neigh = np.ascontiguousarray(division.neighbour, dtype=np.int32)
    trans = np.ascontiguousarray(division.translation, dtype=np.float32)
    tfm = np.ascontiguousarray(division.transform, dtype=np.int32)
    out = np.zeros(int(off[-1]) + per[-1])
    g2 = case.order + 1
    shapes = [(b.ni + g2, b.nj + g2, (b.nk + g2) if case.dim == 3 else 1) for b in division.blocks]
    face = max(max(s[0] * s[1], s[1] * s[2], s[0] * s[2]) for s in shapes)
    ng = [s[0] * s[1] * s[2] for s in shapes]
    slot = max(13 * (g2 // 2) * face * 8, max(8 * (8 * r + 6 * n) for r, n in zip(nr, ng)),
               max(8 * 8 * r * (2 * nsamples + 4) for r in nr))
    rc = lib.refmpi_dropin_film(C.c_int(nb), params, neigh.ctypes.data_as(C.POINTER(C.c_int)),
                                trans.ctypes.data_as(C.POINTER(C.c_float)), tfm.ctypes.data_as(C.POINTER(C.c_int)),
                                ptrs, C.c_int(nsamples), C.c_int(again), _ptr(out),
                                off.ctypes.data_as(C.POINTER(C.c_size_t)), C.c_size_t(out.size), C.c_size_t(slot),
                                C.c_int(int(cpu)))
    if rc != 0:
        raise RuntimeError(f"drop-in multi-rank film failed ({rc})")
    return [out[int(off[b]):int(off[b]) + per[b]] for b in range(nb)]


def run_dropin_multirank_film(division, nsamples: int, again: int, real: bool = False, cpu: bool = False):
    """The drop-in's division mode with device Film (over the test double,
    or with real=True over the library on rank 0's GPU; cpu=True: SHOCK's
    own steps and sampling on every rank): per rank the eight Film arrays
    (nsamples x its real points each) and the sample times; after sample
    `again` the sample index goes back one (a NaN reset)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        return pool.apply(_dropin_multirank_film_worker, (division, nsamples, again, real, cpu))
