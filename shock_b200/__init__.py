"""shock_b200: SHOCK's per-RK-stage right-hand side on a B200.

Python host side over the C ABI in include/shock_b200.h
(shock_b200/libshock_b200.so, built from shock_b200/csrc for sm_100a).

``Solver`` mirrors SHOCK's solver entry points for one block:
set-up from a grid and initial state (SHOCK.c:main up to startSimulation),
``rhs()`` (one stage right-hand side, the pieces CalcRungeKutta calls),
``steps(n)`` (n calls of CalcRungeKutta, src/Functions.c:2034-2390, with
the state kept on the device) and state download (the U_RK arrays).

There is no CPU fallback: constructing a Solver without the compiled
library or without a CUDA device raises.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

from . import cases  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("SHOCK_B200_LIB", os.path.join(HERE, "libshock_b200.so"))

SHOCK_FP64 = 0
SHOCK_MIXED = 1
SHOCK_EINVAL = -1
# face boundary conditions (shock_params.bc), SHOCK's BC.c types
SHOCK_BC_AUTO = 0
SHOCK_BC_WALL_VISCOUS = 1
SHOCK_BC_WALL_INVISCID = 2
SHOCK_BC_FARFIELD = 3
SHOCK_BC_WALL_ISOTHERMAL = 4
SHOCK_BC_INFLOW_SUBSONIC = 5
SHOCK_BC_INFLOW_SUPERSONIC = 6
SHOCK_BC_OUTFLOW_SUBSONIC = 7
SHOCK_BC_INFLOW_RIEMANN = 8
SHOCK_BC_INFLOW_ISENTROPIC = 9
SHOCK_BC_OUTFLOW_RIEMANN = 10
SHOCK_BC_OUTFLOW_RUDY = 11

_lib = None
_lock = threading.Lock()

_dp = C.POINTER(C.c_double)


class ShockError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"shock_b200 error {code}: {msg}")
        self.code = code


class Params(C.Structure):
    """Mirror of struct shock_params (include/shock_b200.h)."""
    _fields_ = [
        ("dim", C.c_int), ("order", C.c_int),
        ("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int),
        ("time_order", C.c_int),
        ("tau", C.c_double), ("mach", C.c_double), ("reynolds", C.c_double),
        ("prandtl", C.c_double), ("gamma", C.c_double), ("gas_r", C.c_double),
        ("t0", C.c_double), ("l0", C.c_double),
        ("inviscid", C.c_int), ("mms", C.c_int),
        ("periodic", C.c_int * 3), ("period", C.c_double * 3),
        ("precision", C.c_int), ("zeta_fix", C.c_int),
        ("bc", C.c_int * 6), ("t_wall", C.c_double),
        ("rho_inflow", C.c_double), ("p_inflow", C.c_double), ("p_outflow", C.c_double),
        ("u_inflow", C.c_double * 3), ("weno_eps", C.c_double), ("full_metric", C.c_int),
    ]


def params_from_ini(path: str, base: Params = None) -> Params:
    """shock_params with the config.ini keys of SHOCK's hot path read from path
    (other fields taken from base, or zero)."""
    p = Params() if base is None else base
    _check(lib().shock_params_from_ini(os.fsencode(path), C.byref(p)))
    return p


def build_library(force: bool = False) -> str:
    """Compile shock_b200/csrc into libshock_b200.so (nvcc, sm_100a)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-j8", "-C", os.path.join(HERE, "csrc")], check=True)
    return LIB_PATH


def lib():
    """Load the compiled library (building it if it is missing)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                build_library()
            L = C.CDLL(LIB_PATH)
            L.shock_last_error.restype = C.c_char_p
            L.shock_create.argtypes = [C.POINTER(Params)] + [_dp] * 8 + [C.c_int, C.POINTER(C.c_void_p)]
            for name in ("shock_destroy", "shock_dims", "shock_set_dirichlet", "shock_set_source",
                         "shock_upload_state", "shock_upload_last_pressure", "shock_download_state", "shock_rhs",
                         "shock_step",
                         "shock_step_async", "shock_sync", "shock_check_nan", "shock_geometry",
                         "shock_device_bytes", "shock_last_step_ms", "shock_kernels_per_step",
                         "shock_mms_baseline", "shock_set_kernel_timing", "shock_kernel_times", "shock_measure_fma_peak",
                         "shock_set_tau", "shock_get_tau", "shock_download_pressure",
                         "shock_multi_create", "shock_multi_destroy", "shock_multi_dims", "shock_multi_geometry",
                         "shock_multi_step", "shock_multi_rhs", "shock_multi_download_state",
                         "shock_multi_upload_state", "shock_multi_set_tau", "shock_multi_check_nan",
                         "shock_multi_info", "shock_host_multi_geometry", "shock_set_probes",
                         "shock_probe_history", "shock_film_reserve", "shock_film_sample", "shock_film_download",
                         "shock_host_geometry", "shock_host_mms_baseline", "shock_rhs_static",
                         "shock_batch_create", "shock_batch_destroy", "shock_batch_member_bytes",
                         "shock_batch_add", "shock_batch_remove", "shock_batch_step", "shock_batch_step_async",
                         "shock_batch_sync", "shock_batch_last_ms", "shock_batch_steps_left",
                         "shock_batch_dims", "shock_batch_download_state", "shock_batch_set_tuning",
                         "shock_batch_get_tuning", "shock_batch_info", "shock_batch_check_barrier_timeout",
                         "shock_params_from_ini", "shock_post", "shock_server_create",
                         "shock_server_set_tuning", "shock_server_submit", "shock_server_wait",
                         "shock_server_result", "shock_server_get_stats", "shock_server_destroy"):
                getattr(L, name).restype = C.c_int
            L.shock_batch_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_size_t, C.c_int,
                                             C.POINTER(C.c_void_p)]
            L.shock_batch_add.argtypes = [C.c_void_p, C.POINTER(Params)] + [_dp] * 8 + [C.c_int,
                                                                                      C.POINTER(C.c_int)]
            L.shock_server_submit.argtypes = [C.c_void_p, C.POINTER(Params)] + [_dp] * 8 + [
                C.c_int, C.POINTER(C.c_longlong)]
            L.shock_server_wait.argtypes = [C.c_void_p, C.c_longlong, C.c_double]
            L.shock_multi_create.argtypes = [C.POINTER(Params), C.c_int, C.c_void_p, C.c_int,
                                             C.POINTER(C.c_void_p)]
            L.shock_host_multi_geometry.argtypes = [C.POINTER(Params), C.c_int, C.c_void_p, C.c_void_p]
            L.shock_server_result.argtypes = [C.c_void_p, C.c_longlong, _dp, C.c_size_t, C.c_void_p]
            _lib = L
        return _lib


def _check(rc):
    if rc != 0:
        raise ShockError(rc, lib().shock_last_error().decode())


def _ptr(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def params_from_case(case, precision=SHOCK_FP64, zeta_fix=False, weno_eps=0.0, full_metric=False) -> Params:
    p = Params()
    p.dim, p.order = case.dim, case.order
    p.ni, p.nj, p.nk = case.ni, case.nj, (case.nk if case.dim == 3 else 1)
    p.time_order = case.time_order
    p.tau, p.mach, p.reynolds = case.tau, case.mach, case.reynolds
    p.prandtl, p.gamma, p.gas_r, p.t0, p.l0 = case.prandtl, case.gamma, case.gas_r, case.t0, case.l0
    p.inviscid = int(case.inviscid)
    p.mms = 0 if case.mms == "none" else 1
    for a in range(3):
        p.periodic[a] = int(case.periodic[a])
        p.period[a] = float(case.period[a])
    p.precision = int(precision)
    p.zeta_fix = int(bool(zeta_fix))
    for f in range(6):
        p.bc[f] = int(case.bc[f])
    p.t_wall = float(case.t_wall)
    p.rho_inflow, p.p_inflow, p.p_outflow = float(case.rho_inflow), float(case.p_inflow), float(case.p_outflow)
    for a in range(3):
        p.u_inflow[a] = float(case.u_inflow[a])
    p.weno_eps = float(weno_eps)
    p.full_metric = int(bool(full_metric))
    return p


def _ghosted_shape(case):
    g = case.order + 1
    return (case.ni + g, case.nj + g, (case.nk + g) if case.dim == 3 else 1)


def _fortran_coords(case):
    f = lambda a: np.ascontiguousarray(np.asarray(a, np.float64).transpose(2, 1, 0)).ravel()
    return f(case.x), f(case.y), f(case.z)


def host_geometry(case, full_metric=False) -> np.ndarray:
    """Block geometry (x,y,z,J, 9 metrics; ghosted) built on the host, no device."""
    shp = _ghosted_shape(case)
    out = np.zeros((13,) + shp)
    x, y, z = _fortran_coords(case)
    p = params_from_case(case, full_metric=full_metric)
    _check(lib().shock_host_geometry(C.byref(p), _ptr(x), _ptr(y), _ptr(z), _ptr(out)))
    return out


def host_mms_baseline(case):
    """(exact9, js5) of the built-in 2D manufactured solution, computed on the host."""
    shp = _ghosted_shape(case)
    ex = np.zeros((9,) + shp)
    js = np.zeros((5,) + shp)
    x, y, z = _fortran_coords(case)
    p = params_from_case(case)
    _check(lib().shock_host_mms_baseline(C.byref(p), _ptr(x), _ptr(y), _ptr(z), _ptr(ex), _ptr(js)))
    return ex, js


class Solver:
    """One block of SHOCK's stage right-hand side on a CUDA device."""

    def __init__(self, case, precision=SHOCK_FP64, device: int = 0, zeta_fix: bool = False,
                 dirichlet9=None, source5=None, weno_eps: float = 0.0, full_metric: bool = False):
        self.case = case
        self.lib = lib()
        self.params = params_from_case(case, precision, zeta_fix, weno_eps, full_metric)
        f = lambda a: np.ascontiguousarray(np.asarray(a, np.float64).transpose(2, 1, 0)).ravel()
        arrs = [f(a) for a in case.real_fields()]
        h = C.c_void_p()
        _check(self.lib.shock_create(C.byref(self.params), *[_ptr(a) for a in arrs], int(device), C.byref(h)))
        self.h = h
        d = (C.c_int * 6)()
        _check(self.lib.shock_dims(self.h, d))
        self.shape = (d[0], d[1], d[2])
        self.start = (d[3], d[4], d[5])
        self.n = d[0] * d[1] * d[2]
        if case.mms == "baseline" and dirichlet9 is None and source5 is None:
            dirichlet9, source5 = self.mms_baseline()
        if dirichlet9 is not None:
            a = np.ascontiguousarray(dirichlet9, np.float64).ravel()
            assert a.size == 9 * self.n
            _check(self.lib.shock_set_dirichlet(self.h, _ptr(a)))
        if source5 is not None:
            a = np.ascontiguousarray(source5, np.float64).ravel()
            assert a.size == 5 * self.n
            _check(self.lib.shock_set_source(self.h, _ptr(a)))

    def mms_baseline(self):
        """(exact9, js5) of the built-in 2D manufactured solution on this block."""
        ex = np.zeros(9 * self.n)
        js = np.zeros(5 * self.n)
        _check(self.lib.shock_mms_baseline(self.h, _ptr(ex), _ptr(js)))
        return ex.reshape((9,) + self.shape), js.reshape((5,) + self.shape)

    def close(self):
        if getattr(self, "h", None):
            self.lib.shock_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def rhs(self) -> np.ndarray:
        q = np.zeros(5 * self.n)
        _check(self.lib.shock_rhs(self.h, _ptr(q)))
        return q.reshape((5,) + self.shape)

    def steps(self, n: int):
        _check(self.lib.shock_step(self.h, C.c_int(n)))

    def set_tau(self, tau: float):
        """The time step of the following steps (SHOCK's numericalTau)."""
        _check(self.lib.shock_set_tau(self.h, C.c_double(tau)))

    def tau(self) -> float:
        t = C.c_double()
        _check(self.lib.shock_get_tau(self.h, C.byref(t)))
        return t.value

    def steps_async(self, n: int):
        _check(self.lib.shock_step_async(self.h, C.c_int(n)))

    def sync(self):
        _check(self.lib.shock_sync(self.h))

    def last_ms(self) -> float:
        v = C.c_float()
        _check(self.lib.shock_last_step_ms(self.h, C.byref(v)))
        return v.value

    def state(self, out: np.ndarray = None) -> np.ndarray:
        """rho,u,v,w,e (ghosted).  out: a C-contiguous float64 array of 5*NG
        values to download into (pinned host memory makes this a direct DMA)."""
        s = np.zeros(5 * self.n) if out is None else out
        assert s.dtype == np.float64 and s.flags["C_CONTIGUOUS"] and s.size == 5 * self.n
        _check(self.lib.shock_download_state(self.h, _ptr(s), 0))
        return s.reshape((5,) + self.shape)

    def set_probes(self, ijk, capacity: int = 1024):
        """Record p, u, v, w of U_lastStep at ghosted points ijk (a list of
        (i, j, k)) after every step, on the device."""
        a = np.ascontiguousarray(np.asarray(ijk, dtype=np.int32).reshape(-1, 3))
        self._nprobes = a.shape[0]
        _check(self.lib.shock_set_probes(self.h, C.c_int(a.shape[0]), a.ctypes.data_as(C.POINTER(C.c_int)),
                                         C.c_int(capacity)))

    def probe_history(self, max_steps: int = 1024) -> np.ndarray:
        """(steps, probes, 4): p, u, v, w after each step since the last call."""
        n = getattr(self, "_nprobes", 0)
        out = np.zeros(max(1, max_steps * n * 4))
        steps = C.c_int()
        _check(self.lib.shock_probe_history(self.h, _ptr(out), C.c_int(max_steps), C.byref(steps)))
        return out[:steps.value * n * 4].reshape(steps.value, n, 4)

    def film_reserve(self, frames: int):
        _check(self.lib.shock_film_reserve(self.h, C.c_int(frames)))
        self._film_cap = frames

    def film_sample(self):
        _check(self.lib.shock_film_sample(self.h))

    def film(self) -> np.ndarray:
        """(frames, 8, ni, nj, nk): rho, u, v, w, p, |grad rho|, Mach, lambda2."""
        c = self.case
        nk = c.nk if c.dim == 3 else 1
        cap = getattr(self, "_film_cap", 0)
        out = np.zeros(max(1, cap * 8 * c.ni * c.nj * nk))
        frames = C.c_int()
        _check(self.lib.shock_film_download(self.h, _ptr(out), C.c_int(cap), C.byref(frames)))
        return out[:frames.value * 8 * c.ni * c.nj * nk].reshape(frames.value, 8, c.ni, c.nj, nk)

    def pressure(self) -> np.ndarray:
        """U_RK's p after the last step (ghosted)."""
        s = np.zeros(self.n)
        _check(self.lib.shock_download_pressure(self.h, _ptr(s)))
        return s.reshape(self.shape)

    def set_state(self, prim5):
        a = np.ascontiguousarray(prim5, np.float64).ravel()
        assert a.size == 5 * self.n
        _check(self.lib.shock_upload_state(self.h, _ptr(a)))

    def set_last_pressure(self, p):
        """U_lastStep's pressure (ghosted) for the state set_state loaded:
        Rudy outflow faces start from it."""
        a = np.ascontiguousarray(p, np.float64).ravel()
        assert a.size == self.n
        _check(self.lib.shock_upload_last_pressure(self.h, _ptr(a)))

    def post(self) -> np.ndarray:
        """Mach number, |grad rho| and lambda2 of the current state (3 fields,
        ghosted; real points set), computed on the device as SHOCK's
        CalcValuesForPost does for sampling."""
        q = np.zeros(3 * self.n)
        _check(self.lib.shock_post(self.h, _ptr(q)))
        return q.reshape((3,) + self.shape)

    def geometry(self) -> np.ndarray:
        g = np.zeros(13 * self.n)
        _check(self.lib.shock_geometry(self.h, _ptr(g)))
        return g.reshape((13,) + self.shape)

    def check_nan(self) -> int:
        bad = C.c_int()
        rc = self.lib.shock_check_nan(self.h, C.byref(bad))
        if rc not in (0, -4):
            _check(rc)
        return bad.value

    def device_bytes(self) -> int:
        b = C.c_size_t()
        _check(self.lib.shock_device_bytes(self.h, C.byref(b)))
        return b.value

    def kernels_per_step(self) -> int:
        n = C.c_int()
        _check(self.lib.shock_kernels_per_step(self.h, C.byref(n)))
        return n.value

    def set_kernel_timing(self, on: bool = True):
        """Time every launch inside the step graph (event nodes between
        launches) from now on; clears the accumulated times."""
        _check(self.lib.shock_set_kernel_timing(self.h, int(bool(on))))

    def kernel_times(self):
        """({name: (total ms, launches)}, steps timed) since timing was switched on."""
        names = C.create_string_buffer(48 * 64)
        ms = (C.c_double * 64)()
        nl = (C.c_longlong * 64)()
        cnt, steps = C.c_int(), C.c_longlong()
        _check(self.lib.shock_kernel_times(self.h, 64, names, ms, nl, C.byref(cnt), C.byref(steps)))
        out = {}
        for i in range(cnt.value):
            nm = names.raw[48 * i:48 * i + 48].split(b"\0")[0].decode()
            out[nm] = (ms[i], nl[i])
        return out, steps.value

    def real(self, a: np.ndarray) -> np.ndarray:
        """Real-point view of a ghosted field array (..., NIg, NJg, NKg)."""
        g = self.start
        c = self.case
        if c.dim == 3:
            return a[..., g[0]:g[0] + c.ni, g[1]:g[1] + c.nj, g[2]:g[2] + c.nk]
        return a[..., g[0]:g[0] + c.ni, g[1]:g[1] + c.nj, :]


class Block(C.Structure):
    """Mirror of struct shock_block (include/shock_b200.h)."""
    _fields_ = [("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int), ("bc", C.c_int * 6),
                ("neighbour", C.c_int * 6), ("translation", (C.c_float * 3) * 6)] + \
               [(n, _dp) for n in ("x", "y", "z", "u", "v", "w", "p", "rho")] + \
               [("transform", (C.c_int * 3) * 6)]


def _division_blocks(division):
    """(Block array, kept field arrays) of a division for the C ABI."""
    case = division.case
    f = lambda a: np.ascontiguousarray(np.asarray(a, np.float64).transpose(2, 1, 0)).ravel()
    nb = len(division.blocks)
    arr = (Block * nb)()
    keep = []
    for b, bc in enumerate(division.blocks):
        B = arr[b]
        B.ni, B.nj, B.nk = bc.ni, bc.nj, (bc.nk if case.dim == 3 else 1)
        for q in range(6):
            B.bc[q] = int(bc.bc[q])
            B.neighbour[q] = int(division.neighbour[b, q])
            for c in range(3):
                B.translation[q][c] = float(division.translation[b, q, c])
                B.transform[q][c] = int(division.transform[b, q, c])
        fields = [f(a) for a in bc.real_fields()]
        keep.append(fields)
        for name, a in zip(("x", "y", "z", "u", "v", "w", "p", "rho"), fields):
            setattr(B, name, _ptr(a))
    return arr, keep


def locate_probes(case, geometry13, xyz):
    """The grid points SHOCK records probes at (shock_locate_probes): for
    the n x 3 locations xyz on the block of case with ghosted geometry
    geometry13 (13 x ghosted shape, as Solver.geometry or host_geometry give
    it), the ghosted (i, j, k) of each probe's point and whether the block
    records it."""
    g = np.ascontiguousarray(geometry13, np.float64)
    xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
    n = len(xyz)
    ijk = np.zeros((n, 3), np.int32)
    found = np.zeros(n, np.int32)
    x, y, z = (np.ascontiguousarray(g[a]) for a in range(3))
    ip = C.POINTER(C.c_int)
    _check(lib().shock_locate_probes(case.dim, case.ni, case.nj, case.nk if case.dim == 3 else 1, case.ghosts,
                                     _ptr(x), _ptr(y), _ptr(z), n, _ptr(xyz), ijk.ctypes.data_as(ip),
                                     found.ctypes.data_as(ip)))
    return ijk, found.astype(bool)


def read_division(path, dim, nranks, swap=False):
    """Every rank's row of a SHOCK .sddc division file (shock_read_division):
    (neighbour (n,6), translation (n,6,3), transform (n,6,3), corners (n,6),
    sizes (n,3))."""
    nb = np.zeros((nranks, 6), np.int32)
    tr = np.zeros((nranks, 6, 3), np.float32)
    tf = np.zeros((nranks, 6, 3), np.int32)
    co = np.zeros((nranks, 6), np.int64)
    sz = np.zeros((nranks, 3), np.int64)
    for r in range(nranks):
        B = Block()
        c6 = (C.c_longlong * 6)()
        _check(lib().shock_read_division(str(path).encode(), int(dim), int(nranks), r, int(bool(swap)),
                                         C.byref(B), c6))
        nb[r] = list(B.neighbour)
        tr[r] = [list(B.translation[f]) for f in range(6)]
        tf[r] = [list(B.transform[f]) for f in range(6)]
        co[r] = list(c6)
        sz[r] = (B.ni, B.nj, B.nk)
    return nb, tr, tf, co, sz


def host_multi_geometry(division, full_metric=False):
    """Per block geometry (13, ghosted) of a division, built on the host with
    the interfaces exchanged as SHOCK's ranks exchange them (no device)."""
    case = division.case
    arr, keep = _division_blocks(division)
    g2 = case.order + 1
    outs = [np.zeros((13, b.ni + g2, b.nj + g2, (b.nk + g2) if case.dim == 3 else 1)) for b in division.blocks]
    ptrs = (_dp * len(outs))(*[_ptr(o) for o in outs])
    p = params_from_case(case, full_metric=full_metric)
    _check(lib().shock_host_multi_geometry(C.byref(p), len(outs), arr, ptrs))
    return outs


class Multi:
    """The blocks of a division (shock_b200.cases.split) on one device,
    their interfaces exchanged on the device before every stage, as SHOCK's
    ranks exchange them (shock_multi_*)."""

    def __init__(self, division, precision=SHOCK_FP64, device: int = 0, zeta_fix: bool = False,
                 weno_eps: float = 0.0, full_metric: bool = False):
        self.division = division
        self.lib = lib()
        case = division.case
        self.params = params_from_case(case, precision, zeta_fix, weno_eps, full_metric)
        nb = len(division.blocks)
        arr, self._keep = _division_blocks(division)
        h = C.c_void_p()
        _check(self.lib.shock_multi_create(C.byref(self.params), nb, arr, int(device), C.byref(h)))
        self.h = h
        self._keep = None
        self.nblocks = nb
        self.shapes, self.starts = [], []
        for b in range(nb):
            d = (C.c_int * 6)()
            _check(self.lib.shock_multi_dims(self.h, b, d))
            self.shapes.append((d[0], d[1], d[2]))
            self.starts.append((d[3], d[4], d[5]))

    def close(self):
        if getattr(self, "h", None):
            self.lib.shock_multi_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _n(self, b):
        s = self.shapes[b]
        return s[0] * s[1] * s[2]

    def steps(self, n: int):
        _check(self.lib.shock_multi_step(self.h, C.c_int(n)))

    def rhs(self, b: int) -> np.ndarray:
        q = np.zeros(5 * self._n(b))
        _check(self.lib.shock_multi_rhs(self.h, int(b), _ptr(q)))
        return q.reshape((5,) + self.shapes[b])

    def state(self, b: int) -> np.ndarray:
        s = np.zeros(5 * self._n(b))
        _check(self.lib.shock_multi_download_state(self.h, int(b), _ptr(s)))
        return s.reshape((5,) + self.shapes[b])

    def geometry(self, b: int) -> np.ndarray:
        g = np.zeros(13 * self._n(b))
        _check(self.lib.shock_multi_geometry(self.h, int(b), _ptr(g)))
        return g.reshape((13,) + self.shapes[b])

    def set_tau(self, tau: float):
        _check(self.lib.shock_multi_set_tau(self.h, C.c_double(tau)))

    def info(self) -> dict:
        nb, nk, ms = C.c_int(), C.c_int(), C.c_float()
        _check(self.lib.shock_multi_info(self.h, C.byref(nb), C.byref(nk), C.byref(ms)))
        return {"blocks": nb.value, "kernels_per_step": nk.value, "last_ms": ms.value}

    def assemble(self, per_block):
        """The whole block's real points from per-block ghosted arrays
        (leading axis kept), for comparison with a single-block solve."""
        case = self.division.case
        g = case.ghosts
        lead = per_block[0].shape[0]
        out = np.zeros((lead, case.ni, case.nj, case.nk if case.dim == 3 else 1))
        for b, a in enumerate(per_block):
            bc, lo = self.division.blocks[b], self.division.lo[b]
            k0 = g if case.dim == 3 else 0
            r = self.division.from_block(b, a[:, g:g + bc.ni, g:g + bc.nj, k0:k0 + (bc.nk if case.dim == 3 else 1)])
            out[:, lo[0]:lo[0] + r.shape[1], lo[1]:lo[1] + r.shape[2], lo[2]:lo[2] + r.shape[3]] = r
        return out


class BatchTuning(C.Structure):
    """Mirror of struct shock_batch_tuning (include/shock_b200.h)."""
    _fields_ = [("persistent", C.c_int), ("blocks_per_sm", C.c_int), ("chunk", C.c_int),
                ("small_tile_max", C.c_int), ("max_blocks_per_sm", C.c_int)]


def member_bytes(case, precision=SHOCK_FP64) -> int:
    """Device bytes one batch member for this case takes from a batch arena."""
    b = C.c_size_t()
    p = params_from_case(case, precision)
    _check(lib().shock_batch_member_bytes(C.byref(p), C.byref(b)))
    return b.value


class Batch:
    """Many periodic blocks of one class (dim, order, precision, RK order)
    advanced together on one device (shock_batch_* in the C ABI).  Each
    member keeps its own size, physics, tau and step count; members can be
    added and removed between steps."""

    def __init__(self, dim: int, order: int, precision=SHOCK_FP64, time_order: int = 4,
                 arena_bytes: int = 1 << 30, device: int = 0):
        self.lib = lib()
        self.dim, self.order, self.precision, self.time_order = dim, order, precision, time_order
        h = C.c_void_p()
        _check(self.lib.shock_batch_create(dim, order, int(precision), time_order, int(arena_bytes),
                                           int(device), C.byref(h)))
        self.h = h
        self.cases = {}

    def close(self):
        if getattr(self, "h", None):
            self.lib.shock_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, case, nsteps: int) -> int:
        p = params_from_case(case, self.precision)
        f = lambda a: np.ascontiguousarray(np.asarray(a, np.float64).transpose(2, 1, 0)).ravel()
        arrs = [f(a) for a in case.real_fields()]
        m = C.c_int()
        _check(self.lib.shock_batch_add(self.h, C.byref(p), *[_ptr(a) for a in arrs], int(nsteps),
                                        C.byref(m)))
        self.cases[m.value] = case
        return m.value

    def remove(self, m: int):
        _check(self.lib.shock_batch_remove(self.h, int(m)))
        self.cases.pop(m, None)

    def step(self, n: int = 1):
        _check(self.lib.shock_batch_step(self.h, int(n)))

    def step_async(self, n: int = 1):
        _check(self.lib.shock_batch_step_async(self.h, int(n)))

    def sync(self):
        _check(self.lib.shock_batch_sync(self.h))

    def last_ms(self) -> float:
        v = C.c_float()
        _check(self.lib.shock_batch_last_ms(self.h, C.byref(v)))
        return v.value

    def steps_left(self, m: int) -> int:
        v = C.c_int()
        _check(self.lib.shock_batch_steps_left(self.h, int(m), C.byref(v)))
        return v.value

    def shape(self, m: int):
        d = (C.c_int * 6)()
        _check(self.lib.shock_batch_dims(self.h, int(m), d))
        return (d[0], d[1], d[2])

    def state(self, m: int) -> np.ndarray:
        shp = self.shape(m)
        s = np.zeros(5 * shp[0] * shp[1] * shp[2])
        _check(self.lib.shock_batch_download_state(self.h, int(m), _ptr(s)))
        return s.reshape((5,) + shp)

    def tuning(self) -> BatchTuning:
        t = BatchTuning()
        _check(self.lib.shock_batch_get_tuning(self.h, C.byref(t)))
        return t

    def set_tuning(self, persistent=None, blocks_per_sm=None, chunk=None, small_tile_max=None):
        t = self.tuning()
        if small_tile_max is not None:
            t.small_tile_max = int(small_tile_max)
        if persistent is not None:
            t.persistent = int(persistent)
        if blocks_per_sm is not None:
            t.blocks_per_sm = int(blocks_per_sm)
        if chunk is not None:
            t.chunk = int(chunk)
        _check(self.lib.shock_batch_set_tuning(self.h, C.byref(t)))

    def info(self) -> dict:
        n, k = C.c_int(), C.c_int()
        used, total = C.c_size_t(), C.c_size_t()
        _check(self.lib.shock_batch_info(self.h, C.byref(n), C.byref(used), C.byref(total), C.byref(k)))
        return {"members": n.value, "arena_used": used.value, "arena_total": total.value,
                "kernels_per_step": k.value}


class ServerConfig(C.Structure):
    """Mirror of struct shock_server_config."""
    _fields_ = [("device", C.c_int), ("hbm_budget", C.c_size_t), ("max_requests", C.c_int),
                ("setup_threads", C.c_int), ("round_ms", C.c_double)]


class RequestInfo(C.Structure):
    """Mirror of struct shock_request_info."""
    _fields_ = [("submit_s", C.c_double), ("admit_s", C.c_double), ("done_s", C.c_double),
                ("cell_stages", C.c_double), ("status", C.c_int), ("dims", C.c_int * 6)]


class ServerStats(C.Structure):
    """Mirror of struct shock_server_stats."""
    _fields_ = [("queued", C.c_longlong), ("running", C.c_longlong), ("completed", C.c_longlong),
                ("failed", C.c_longlong), ("rounds", C.c_longlong), ("steps_launched", C.c_longlong),
                ("cell_stages", C.c_double), ("busy_ms", C.c_double), ("arena_used", C.c_size_t),
                ("arena_total", C.c_size_t), ("uptime_s", C.c_double), ("loop_error", C.c_int)]


class Server:
    """The C request loop (shock_server_*): submit solve requests as they
    arrive; each runs on the device with continuous batching inside an HBM
    budget and is collected with wait()/result()."""

    def __init__(self, hbm_budget: int = 150 * 10 ** 9, device: int = 0, max_requests: int = 0,
                 setup_threads: int = 0, round_ms: float = 0.0):
        self.lib = lib()
        cfg = ServerConfig(int(device), int(hbm_budget), int(max_requests), int(setup_threads), float(round_ms))
        h = C.c_void_p()
        _check(self.lib.shock_server_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self.cases = {}

    def close(self):
        if getattr(self, "h", None):
            self.lib.shock_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_tuning(self, dim, order, precision, time_order=4, **kw):
        t = BatchTuning(kw.get("persistent", 1), kw.get("blocks_per_sm", 1), kw.get("chunk", 2048),
                        kw.get("small_tile_max", 0), 0)
        _check(self.lib.shock_server_set_tuning(self.h, int(dim), int(order), int(precision), int(time_order),
                                                C.byref(t)))

    def submit(self, case, nsteps: int, precision=SHOCK_FP64) -> int:
        p = params_from_case(case, precision)
        f = lambda a: np.ascontiguousarray(np.asarray(a, np.float64).transpose(2, 1, 0)).ravel()
        arrs = [f(a) for a in case.real_fields()]
        rid = C.c_longlong()
        _check(self.lib.shock_server_submit(self.h, C.byref(p), *[_ptr(a) for a in arrs], int(nsteps),
                                            C.byref(rid)))
        self.cases[rid.value] = case
        return rid.value

    def wait(self, rid: int, timeout: float = 600.0):
        _check(self.lib.shock_server_wait(self.h, C.c_longlong(rid), C.c_double(timeout)))

    def result(self, rid: int):
        """(rho,u,v,w,e ghosted, info dict) of a finished request; releases it."""
        case = self.cases.pop(rid)
        shp = _ghosted_shape(case)
        out = np.zeros(5 * shp[0] * shp[1] * shp[2])
        info = RequestInfo()
        _check(self.lib.shock_server_result(self.h, C.c_longlong(rid), _ptr(out), out.size, C.byref(info)))
        d = {"submit_s": info.submit_s, "admit_s": info.admit_s, "done_s": info.done_s,
             "tts_s": info.done_s - info.submit_s, "cell_stages": info.cell_stages, "status": info.status}
        return out.reshape((5,) + shp), d

    def stats(self) -> dict:
        st = ServerStats()
        _check(self.lib.shock_server_get_stats(self.h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}
