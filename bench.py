"""Benchmark: cell-stage updates/s of SHOCK's per-RK-stage right-hand side.

Default workload (N=1): 3D decaying compressible turbulence on a 512^3
uniform periodic cube, WENO9, viscous, RK4, FP64 (plain form): the largest
configuration that fits one GPU (about 58 GB of device memory).  The initial
velocity is a seeded random-phase solenoidal field, E(k) ~ k^4 exp(-2(k/4)^2),
at turbulent Mach 0.6, rho = 1, p = 1/gamma, Re_lambda = 100 (synthetic
inputs; no dataset is involved).  A step is one RK4 time step (4 stage
right-hand sides + updates) over the whole block.

Metric: cell-stage updates/s = real points x stages x steps x ranks / time.
  value  -- device time with the state resident in HBM (CUDA events on the
            solver's stream around each step's graph); the 512^3 state is
            far larger than L2 (small blocks get the L2 flushed by a 256 MiB
            write between timed steps).  The timed step graphs carry an event
            after every launch, so the per-kernel times (roofline.kernels_ms_
            per_step) are measured over the same timed steps and add up to
            the step time.
  e2e    -- the same steps through the public C ABI with host buffers:
            every step uploads the state from pinned host memory
            (shock_upload_state), runs it (shock_step) and reads the state
            back (shock_download_state); host wall clock around the three
            synchronous calls.
The mixed form (FP32 stencils, FP64 state) is timed the same way beside it,
and both forms are run on to 50 steps (the configuration's run length) from
the same initial state: "mixed.l2_vs_fp64" is the relative L2 of each
conserved variable of the mixed form against the FP64 form.

--impl reference: SHOCK's own CPU code (oracle/_ref, the unmodified
reference sources) on a bounded sample of the workload (REF_SAMPLES), one
single-block process per host core, each advancing its own copy by the same
--warmup and --steps RK4 steps; aggregate cell-stage/s over the slowest
process.  Under torchrun only rank 0 runs it.

Multi-GPU (torchrun, N>1): replicas only -- every rank advances its own
copy of the block (no data exchange on the path), value sums all ranks
over the max-over-ranks time ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (description, builder)
    "tgv64_w5": "3D curvilinear Taylor-Green vortex 64^3, WENO5, viscous, RK4, Ma=0.1, Re=1600",
    "tgv128_w5": "3D curvilinear Taylor-Green vortex 128^3, WENO5, viscous, RK4",
    "turb128_w9": "3D decaying turbulence 128^3, WENO9, viscous, RK4, Mt=0.6",
    "turb256_w9": "3D decaying turbulence 256^3, WENO9, viscous, RK4, Mt=0.6",
    "turb512_w9": "3D decaying turbulence 512^3, WENO9, viscous, RK4, Mt=0.6",
    "tgv512_w5": "3D Taylor-Green vortex 512^3, WENO5, viscous, RK4",
    "mms64_w5": "2D manufactured solution 64^2, WENO5, viscous, RK4",
    "batch_vortex256": "256 2D isentropic vortices, N in {32,48,...,256} (seeded), beta U[1,5], "
                       "Mach U[0.2,0.8], inviscid, WENO5, RK4, mixed precision, one batch",
    "serve_poisson": "Poisson arrivals (200/s, seeded) of 2D/3D Taylor-Green / vortex solve requests, "
                     "32^2..128^3 points log-uniform, WENO5/9, Mach U[0.1,0.6], Re U[100,5000], 20..500 steps",
}


def make_case(name):
    from shock_b200 import cases
    if name == "tgv64_w5":
        return cases.taylor_green(64, order=5)
    if name == "tgv128_w5":
        return cases.taylor_green(128, order=5)
    if name == "tgv512_w5":
        return cases.taylor_green(512, order=5)
    if name == "turb128_w9":
        return cases.decaying_turbulence(128, order=9)
    if name == "turb256_w9":
        return cases.decaying_turbulence(256, order=9)
    if name == "turb512_w9":
        return cases.decaying_turbulence(512, order=9)
    if name == "mms64_w5":
        return cases.mms_square(64, 5, family="baseline")
    raise SystemExit(f"unknown workload {name}")


def batch_cases(nmem=256, seed=4):
    """The batched-ensemble members: N from {32, 48, ..., 256}, beta U[1,5],
    Mach U[0.2,0.8], seeded."""
    import numpy as np
    from shock_b200 import cases
    rng = np.random.default_rng(seed)
    ns = rng.choice(np.arange(32, 257, 16), size=nmem)
    out = []
    for n in ns:
        out.append(cases.isentropic_vortex(int(n), beta=float(rng.uniform(1, 5)), mach_inf=float(rng.uniform(0.2, 0.8))))
    return out


def measured_traffic(workload, kernel, points, precision="fp64"):
    """DRAM bytes (read + write) of one launch of `kernel` on `workload`, from
    an ncu capture recorded in shock_b200/roofline.json: the workload's own,
    or that of a smaller block of the same flow and order scaled by the
    points one launch processes (None if neither is recorded)."""
    path = os.path.join(ROOT, "shock_b200", "roofline.json")
    with open(path) as f:
        t = json.load(f).get("traffic", {})
    e = t.get(workload, {}).get(precision, {}).get(kernel)
    if e is not None:
        return e["bytes"]
    for src in t.get(workload, {}).get("scaled_from", []):
        e = t.get(src, {}).get(precision, {}).get(kernel)
        if e is not None and e.get("points"):
            return e["bytes"] * points / e["points"]
    return None


def flops_per_cell_stage(case):
    path = os.path.join(ROOT, "shock_b200", "roofline.json")
    with open(path) as f:
        counts = json.load(f)["counts"]
    key = f"{case.dim}d_w{case.order}_{'inviscid' if case.inviscid else 'viscous'}"
    c = dict(counts[key])
    for a in ("xi", "eta", "zeta"):   # fused sweeps: WENO + viscous of a direction, the last one + RK
        if f"weno_{a}" in c and f"visc_{a}" in c:
            c[f"weno_visc_{a}"] = c[f"weno_{a}"] + c[f"visc_{a}"]
            c[f"weno_visc_rk_{a}"] = c[f"weno_visc_{a}"] + c["rk"]
            c[f"visc_rk_{a}"] = c[f"visc_{a}"] + c["rk"]
    return c


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() in ("active", "0x1", "1"):
                    reasons.add(nm)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def rank_helpers(world, device="cuda"):
    """barrier() (all ranks, then the device) and max_over_ranks(x) for the
    replicas run: every rank times its own copy of the work, the job's time is
    the slowest rank's (collectives on `device`: "cuda" under NCCL, "cpu"
    under gloo)."""
    import torch
    import torch.distributed as dist

    def barrier():
        if world > 1:
            dist.barrier()
        if device == "cuda":
            torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    return barrier, max_over_ranks


def replica_value(units_per_rank, world, seconds_max):
    """Whole-job throughput of the replicas run: every rank processed
    units_per_rank; the job took the slowest rank's time."""
    return units_per_rank * world / seconds_max


def flush_l2(torch, buf):
    buf.zero_()


# ---------------------------------------------------------------------------
# reference arm (CPU)
# ---------------------------------------------------------------------------
def _ref_worker(args):
    spec, nsteps, nwarm = args
    # SHOCK's own code reports its set-up on stdout; keep the bench's stdout
    # to the one JSON line
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from refbind import RefSolver
    from shock_b200 import cases
    case = getattr(cases, spec[0])(**spec[1])
    r = RefSolver(case)
    r.steps(nwarm)                  # warm-up (first touch)
    t = r.time_steps(nsteps)
    return t, case.real_points * case.time_order * nsteps


# SHOCK has no request loop: the serving stream's CPU counterpart solves a
# bounded sample of the same requests with SHOCK's own code, one process per
# request on a pool of one process per core, first come first served, all
# requests submitted at once; a request's time to solution is its wait for a
# core plus its solve.  The sample: the stream's requests in arrival order
# whose solve is estimated at most SERVE_REF_MAX_S on one core (SHOCK's CPU
# rates measured on the B200 box's cores, per core: WENO5 5.5e5, WENO9 3.3e5
# cell-stage updates/s), up to SERVE_REF_BUDGET_S of work per core.
SERVE_REF_MAX_S = 10.0
SERVE_REF_BUDGET_S = 30.0
SERVE_REF_RATE = {5: 5.5e5, 9: 3.3e5}


def _serve_ref_worker(args):
    case, nsteps = args
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from refbind import RefSolver
    t0 = time.time()
    r = RefSolver(case)
    r.steps(nsteps)
    return t0, time.time(), case.real_points * case.time_order * nsteps


def run_serve_reference(args):
    import numpy as np
    from shock_b200 import cases
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from refbind import ref_available
    stream = cases.serving_stream(args.requests, seed=5)
    cores = os.cpu_count() or 1
    sample, budget = [], cores * SERVE_REF_BUDGET_S
    for _, case, nsteps in stream:
        if not ref_available(case.order, case.dim):
            continue
        est = case.real_points * case.time_order * nsteps / SERVE_REF_RATE[case.order]
        if est <= SERVE_REF_MAX_S and est <= budget:
            sample.append((case, nsteps))
            budget -= est
    if not sample:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent)"}))
        return
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(cores, len(sample))) as pool:
        t_submit = time.time()
        res = pool.map(_serve_ref_worker, sample, chunksize=1)
    ends = np.array([e for _, e, _ in res])
    tts = ends - t_submit
    cells = sum(c for _, _, c in res)
    wall = float(ends.max() - t_submit)
    v = cells / wall
    what = (f"{len(sample)} of the stream's {len(stream)} requests (those whose SHOCK CPU solve is estimated at "
            f"<= {SERVE_REF_MAX_S:.0f} s on one core, in arrival order, up to {SERVE_REF_BUDGET_S:.0f} s of work "
            f"per core), each solved by SHOCK's own C code (oracle/_ref) in one process of a pool of "
            f"{min(cores, len(sample))}, first come first served, all submitted at once; {wall:.1f} s")
    print(json.dumps({
        "metric": "time to solution p50/p99 (s) and cell-stage updates/s", "value": v,
        "unit": "cell-stage updates/s", "impl": "reference", "n_gpus": args.gpus, "steps": len(sample),
        "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": args.workload, "description": WORKLOADS[args.workload], "requests": len(stream),
                   "hbm_budget_gb": args.hbm_gb, "parallelism": f"replicas x{args.gpus}"},
        "fp64": {"p50_s": float(np.percentile(tts, 50)), "p99_s": float(np.percentile(tts, 99)),
                 "throughput": v, "wall_s": wall},
        "cpu_baseline": {"value": v, "unit": "cell-stage updates/s", "cores": min(cores, len(sample)),
                         "kind": "reference", "sample": what},
        "e2e": {"value": v, "unit": "cell-stage updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def reference_throughput(spec, steps, warmup, procs):
    """procs processes, each advancing its own copy of the block `spec` (a
    shock_b200.cases builder and its arguments) by warmup untimed and steps
    timed RK steps; aggregate cell-stage/s over the slowest process."""
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker, [(spec, steps, warmup)] * procs)
    tmax = max(t for t, _ in res)
    cells = sum(c for _, c in res)
    return cells / tmax, tmax, res


# The CPU sample of each single-block workload: the block itself where one RK4
# step of SHOCK's CPU code takes a few seconds, else a 64^3 (WENO5) or 48^3
# (WENO9) block of the same flow and order, about 2 s per RK4 step on one
# core (a 512^3 block needs about 340 GB in SHOCK's CPU build, about 300
# doubles per ghosted point, and one RK4 step of a 128^3 WENO9 block takes
# about half a minute per core).
REF_SAMPLES = {
    "tgv64_w5": (("taylor_green", {"n": 64, "order": 5}), "the tgv64_w5 block"),
    "tgv128_w5": (("taylor_green", {"n": 64, "order": 5}), "a 64^3 block of the same flow and order"),
    "tgv512_w5": (("taylor_green", {"n": 64, "order": 5}), "a 64^3 block of the same flow and order"),
    "turb128_w9": (("decaying_turbulence", {"n": 48, "order": 9}), "a 48^3 block of the same flow and order"),
    "turb256_w9": (("decaying_turbulence", {"n": 48, "order": 9}), "a 48^3 block of the same flow and order"),
    "turb512_w9": (("decaying_turbulence", {"n": 48, "order": 9}), "a 48^3 block of the same flow and order"),
    "mms64_w5": (("mms_square", {"n": 64, "order": 5, "family": "baseline"}), "the mms64_w5 block"),
}


# SHOCK's MPI path on the host cores: a division of a sample block of the
# same flow and order, one rank per core, SHOCK's own set-up and
# TransferFlowParameterWithGhosts between the ranks over the forked
# shared-memory MPI stand-in (oracle/_ref/libshockmpi_*).  Every axis is
# split in two or more (SHOCK's self-periodic exchange takes one axis per
# rank at most) and each block keeps nj <= nk (its j-centred zeta stencil).
MPI_SAMPLES = {
    "w9": ("decaying_turbulence", {"n": 128, "order": 9}),
    "w5": ("taylor_green", {"n": 128, "order": 5}),
}
MPI_PARTS = {16: (4, 2, 2), 8: (2, 2, 2), 4: (2, 2, 1)}


def mpi_reference(workload, steps, warmup):
    """Cell-stage updates/s of SHOCK's MPI code path on a bounded sample:
    the division's steps timed as the difference between a run of
    warmup + steps and one of warmup steps (the same set-up in both).
    None where the sample does not apply or the build is absent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from refbind import multirank_available, run_multirank
    from shock_b200 import cases
    if workload not in WORKLOAD_INFO or "w" not in workload or workload.startswith("mms"):
        return None
    key = "w9" if "w9" in workload else "w5"
    spec = MPI_SAMPLES[key]
    order = spec[1]["order"]
    if not multirank_available(order, 3):
        return None
    n = spec[1]["n"]
    per = 300 * 8 * (n + order + 1) ** 3   # SHOCK's arrays for the whole sample, about 300 doubles a point
    cores = os.cpu_count() or 1
    procs = max([p for p in MPI_PARTS if p <= cores] or [0])
    if not procs or per > 0.5 * _host_avail_bytes():
        return None
    case = getattr(cases, spec[0])(**spec[1])
    d = cases.split(case, MPI_PARTS[procs])
    t0 = time.perf_counter()
    r1 = run_multirank(d, warmup)
    t1 = time.perf_counter()
    r2 = run_multirank(d, warmup + steps)
    t2 = time.perf_counter()
    dt = max((t2 - t1) - (t1 - t0), 1e-9)
    v = case.real_points * 4 * steps / dt
    # SHOCK's own comm_time over the timed steps, the slowest rank
    comm = max(b2["comm_time"] - b1["comm_time"] for b1, b2 in zip(r1, r2))
    parts = "x".join(str(x) for x in MPI_PARTS[procs])
    return {"value": v, "unit": "cell-stage updates/s", "cores": procs, "kind": "reference", "seconds": dt,
            "comm_seconds": comm, "comm_share": comm / dt,
            "sample": f"SHOCK's MPI code path (oracle/_ref/libshockmpi_*: its own set-up and halo exchange between "
                      f"ranks over the forked shared-memory MPI stand-in), a {n}^3 block of the same flow and order "
                      f"divided {parts} ({procs} ranks, one per core), {steps} RK4 steps timed as the difference "
                      f"of runs of {warmup + steps} and {warmup} steps ({dt:.1f} s)"}


def ref_sample(workload):
    spec, what = REF_SAMPLES[workload]
    kw = spec[1]
    pts = kw["n"] ** (2 if spec[0] == "mms_square" else 3)
    return spec, pts, what


def _host_avail_bytes():
    try:
        with open("/proc/meminfo") as f:
            for ln in f:
                if ln.startswith("MemAvailable:"):
                    return int(ln.split()[1]) * 1024
    except OSError:
        pass
    return 32 << 30


def ref_procs(points=64 ** 3, order=5):
    """One single-block SHOCK process per host core, capped so that the
    processes' arrays (about 300 doubles per ghosted point) use at most half
    of the available host memory."""
    g2 = order + 1
    side = round(points ** (1 / 3))
    per = 300 * 8 * (side + g2) ** 3
    return max(1, min(os.cpu_count() or 1, 32, int(0.5 * _host_avail_bytes() // per)))


def batch_reference_sample(procs, steps=1, warmup=1, seed=4):
    """SHOCK's own CPU code on a sample of the batch members: one member per
    process (the first `procs` members), `steps` timed RK4 steps each."""
    import numpy as np
    rng = np.random.default_rng(seed)
    ns = rng.choice(np.arange(32, 257, 16), size=256)
    specs = []
    for n in ns:
        specs.append(("isentropic_vortex", {"n": int(n), "beta": float(rng.uniform(1, 5)),
                                            "mach_inf": float(rng.uniform(0.2, 0.8))}))
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker, [(sp, steps, warmup) for sp in specs[:procs]])
    tmax = max(t for t, _ in res)
    cells = sum(c for _, c in res)
    return cells / tmax, tmax


def run_reference(args, rank, world):
    """SHOCK's own CPU implementation of the path (oracle/_ref) on the host
    cores: every process advances its own copy of the workload's CPU sample
    by --warmup untimed and --steps timed RK4 steps (each step a bounded
    sample of the workload); rank 0 only."""
    if rank != 0:
        return
    if args.workload == "batch_vortex256":
        procs = ref_procs(256 ** 2, 5)
        v, t = batch_reference_sample(procs, steps=args.steps, warmup=args.warmup)
        print(json.dumps({
            "metric": "cell-stage updates/s", "value": v, "unit": "cell-stage updates/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "description": WORKLOADS[args.workload]},
            "cpu_baseline": {"value": v, "unit": "cell-stage updates/s", "cores": procs, "kind": "reference",
                             "sample": f"first {procs} batch members, one SHOCK process each (oracle/_ref), "
                                       f"{args.steps} timed RK4 steps; {t:.1f} s"},
            "e2e": {"value": v, "unit": "cell-stage updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    if args.workload == "serve_poisson":
        run_serve_reference(args)
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from refbind import ref_available
    order, dim = (9, 3) if "w9" in args.workload else (5, 3 if args.workload != "mms64_w5" else 2)
    if not ref_available(order, dim):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent)"}))
        return
    spec, pts, what = ref_sample(args.workload)
    procs = ref_procs(pts, order)
    v, t, _ = reference_throughput(spec, args.steps, args.warmup, procs)
    replicas = {"value": v, "unit": "cell-stage updates/s", "cores": procs, "kind": "reference",
                "sample": f"{procs} single-block processes, each {args.warmup} warm-up and {args.steps} "
                          f"timed RK4 steps of {what}, SHOCK's own C code (oracle/_ref); slowest "
                          f"process {t:.1f} s; a step of the line = one RK4 step of every process"}
    # SHOCK's MPI path (a division with its halo exchange) where the sample
    # applies: the line's value; the single-block replicas beside it
    try:
        mpi = mpi_reference(args.workload, args.steps, args.warmup)
    except (OSError, RuntimeError) as e:
        print(f"bench: SHOCK's MPI-path sample skipped: {e}", file=sys.stderr)
        mpi = None
    base = mpi if mpi is not None else replicas
    v = base["value"]
    ms = (t if mpi is None else mpi["seconds"]) * 1e3 / args.steps
    line = {
        "metric": "cell-stage updates/s", "value": v, "unit": "cell-stage updates/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(args.workload, world),
        "cpu_baseline": base,
        "single_block_replicas": replicas if mpi is not None else None,
        "e2e": {"value": v, "unit": "cell-stage updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
L2_CACHE_BYTES = 126 * 2 ** 20
L2_STEPS = 50      # mixed-vs-FP64 comparison after this many steps (the 512^3 configuration's run length)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="turb512_w9", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-l2", action="store_true", help="skip the mixed-vs-FP64 L2 run")
    ap.add_argument("--tune-budget", type=float, default=60.0, help="seconds the batch autotuner may spend")
    ap.add_argument("--requests", type=int, default=48, help="serve_poisson: requests in the stream")
    ap.add_argument("--hbm-gb", type=float, default=150.0, help="serve_poisson: HBM budget")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import numpy as np
    import torch
    import torch.distributed as dist
    import shock_b200

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))

    barrier, max_over_ranks = rank_helpers(world, "cuda")

    if args.workload == "batch_vortex256":
        run_batch(args, world, rank, local, barrier, max_over_ranks)
        if world > 1:
            dist.destroy_process_group()
        return
    if args.workload == "serve_poisson":
        run_serve(args, world, rank, local, barrier, max_over_ranks)
        if world > 1:
            dist.destroy_process_group()
        return

    case = make_case(args.workload)
    stage_cells = case.real_points * case.time_order
    g2 = case.order + 1
    state_bytes = 5 * 8 * (case.ni + g2) * (case.nj + g2) * ((case.nk + g2) if case.dim == 3 else 1)
    # the stage streams the state and about 45 other fields: blocks whose
    # state alone is below the L2 size get the L2 flushed between steps
    flush = None
    if state_bytes < 4 * L2_CACHE_BYTES:
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    l2_steps = max(L2_STEPS, args.warmup + args.steps)

    def run_form(precision, sampler=None):
        """W warm-up steps, K timed steps (step graph with an event after every
        launch: per-kernel device times over the timed region), then untimed
        steps up to l2_steps; returns the solver and its figures."""
        s = shock_b200.Solver(case, precision=precision, device=local)
        s.set_kernel_timing(True)
        for _ in range(args.warmup):
            s.steps(1)
        s.set_kernel_timing(True)          # clear what the warm-up accumulated
        barrier()
        if sampler:
            sampler.start()
        total_ms = 0.0
        for _ in range(args.steps):
            if flush is not None:
                flush.zero_()
                torch.cuda.synchronize()
            s.steps(1)
            total_ms += s.last_ms()
        clocks = sampler.stop() if sampler else None
        barrier()
        kt, ksteps = s.kernel_times()
        s.set_kernel_timing(False)
        rest = l2_steps - args.warmup - args.steps
        if rest > 0 and not args.no_l2:
            s.steps(rest)
        return s, total_ms, kt, ksteps, clocks

    solver, ms64, kt64, ksteps, clocks = run_form(shock_b200.SHOCK_FP64, ClockSampler(local))
    ms64 = max_over_ranks(ms64)
    value = replica_value(stage_cells * args.steps, world, ms64 * 1e-3)
    state64 = None if args.no_l2 else solver.state()

    # end to end through the C ABI with pinned host buffers: every step
    # uploads that step's input state, runs the step and reads the result back
    n5 = 5 * solver.n
    host = torch.empty(n5, dtype=torch.float64, pin_memory=True).numpy()
    host[:] = solver.state().ravel()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        solver.set_state(host.reshape((5,) + solver.shape))
        solver.steps(1)
        solver.state(out=host)
    t1 = time.perf_counter()
    barrier()
    e2e_s = max_over_ranks(t1 - t0)
    e2e = {"value": stage_cells * args.steps * world / e2e_s, "unit": "cell-stage updates/s",
           "h2d_bytes_per_step": 8 * n5, "d2h_bytes_per_step": 8 * n5}
    launches = solver.kernels_per_step() * args.steps
    del host
    solver.close()

    mixed = None
    if not args.no_mixed:
        try:
            smix, msmix, ktmix, _, clocks_mix = run_form(shock_b200.SHOCK_MIXED, ClockSampler(local))
            msmix = max_over_ranks(msmix)
            mixed = {"value": stage_cells * args.steps * world / (msmix * 1e-3),
                     "ms_per_step": msmix / args.steps, "speedup_vs_fp64": ms64 / msmix,
                     "kernels_ms_per_step": {k: v[0] / args.steps for k, v in ktmix.items()},
                     "clocks": clocks_mix}
            if state64 is not None:
                l2 = l2_conserved(case, smix.state(), state64)
                mixed["l2_vs_fp64"] = {"steps": l2_steps, "rho": l2[0], "rho_u": l2[1], "rho_v": l2[2],
                                       "rho_w": l2[3], "rho_e": l2[4],
                                       "definition": "relative L2 over the real points of each conserved "
                                                     "variable, mixed form against the FP64 form after the "
                                                     "same steps from the same initial state"}
            smix.close()
        except shock_b200.ShockError as e:
            mixed = {"error": str(e)}

    # roofline of the dominant kernel: SHOCK's FP64 operations per launch over
    # its average launch time in the timed region
    fl = flops_per_cell_stage(case)
    peaks = measure_peaks(local)
    dom = max(kt64.items(), key=lambda kv: kv[1][0])
    dom_name, (dom_ms_total, dom_launches) = dom
    launch_ms = dom_ms_total / dom_launches
    dom_flops = fl.get(dom_name, 0.0) * case.real_points
    achieved = dom_flops / (launch_ms * 1e-3) / 1e12
    step_tf = fl["total"] * stage_cells * args.steps / (ms64 * 1e-3) / 1e12
    roofline = {"bound": "fp64", "kernel": dom_name, "achieved": achieved, "peak": peaks["fp64_tflops"],
                "unit": "TFLOP/s", "frac": achieved / peaks["fp64_tflops"],
                "traffic": measured_traffic(args.workload, dom_name, case.real_points),
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch "
                                  "(shock_b200/roofline.json records the capture and its scaling)",
                "peak_source": "measured on this GPU by shock_measure_fma_peak (register-only FP64 FMA loop); "
                               "MEASURED_PEAKS.json has HBM and bf16 figures only",
                "frac_of_nominal_40tf": achieved / 40.0,
                "flops_per_launch": dom_flops, "launch_ms": launch_ms, "launches_timed": dom_launches,
                "step_fp64_tflops": step_tf, "step_frac": step_tf / peaks["fp64_tflops"],
                "kernels_ms_per_step": {k: v[0] / args.steps for k, v in kt64.items()},
                "kernels_sum_ms_per_step": sum(v[0] for v in kt64.values()) / args.steps,
                "hbm": {"algorithmic_bytes_per_cell_stage": (200 if case.dim == 3 else 160),
                        "achieved_gbs": (200 if case.dim == 3 else 160) * stage_cells * args.steps
                        / (ms64 * 1e-3) / 1e9,
                        "peak_gbs": measured_hbm_gbs(),
                        "peak_source": "MEASURED_PEAKS.json (measured copy bandwidth)" if measured_hbm_gbs(False)
                        else "fallback: 6650 GB/s, an earlier copy-bandwidth measurement on this pool"}}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(args.workload, case)

    if rank == 0:
        line = {
            "metric": "cell-stage updates/s", "value": value, "unit": "cell-stage updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms64 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(args.workload, world),
            "mixed": mixed, "e2e": e2e, "gpu_launches": launches,
            "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
            "fp32_peak_tflops": peaks["fp32_tflops"],
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def bench_config(workload, world):
    """The config object of both arms' lines (same keys, same values)."""
    from shock_b200 import cases as _c  # noqa: F401
    info = WORKLOAD_INFO.get(workload, {})
    cfg = {"workload": workload, "description": WORKLOADS[workload], "parallelism": f"replicas x{world}"}
    cfg.update(info)
    return cfg


# points, stages per step and the L2 treatment of each single-block workload
WORKLOAD_INFO = {
    "tgv64_w5": {"points": 64 ** 3, "stages_per_step": 4, "l2": "flushed (256 MiB write) between timed steps"},
    "tgv128_w5": {"points": 128 ** 3, "stages_per_step": 4, "l2": "flushed (256 MiB write) between timed steps"},
    "turb128_w9": {"points": 128 ** 3, "stages_per_step": 4, "l2": "inputs (state 0.9 GB) larger than L2"},
    "turb256_w9": {"points": 256 ** 3, "stages_per_step": 4, "l2": "inputs (state 6.4 GB) larger than L2"},
    "turb512_w9": {"points": 512 ** 3, "stages_per_step": 4, "l2": "inputs (state 5.7 GB, 58 GB in all) larger than L2"},
    "tgv512_w5": {"points": 512 ** 3, "stages_per_step": 4, "l2": "inputs (state 5.5 GB, 56 GB in all) larger than L2"},
    "mms64_w5": {"points": 64 ** 2, "stages_per_step": 4, "l2": "flushed (256 MiB write) between timed steps"},
}


def measured_hbm_gbs(fallback=True):
    """The measured HBM copy bandwidth (MEASURED_PEAKS.json), else the
    earlier measurement of 6650 GB/s (fallback=False: None instead)."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            v = json.load(f).get("hbm_gbs")
            if v:
                return v
    except (OSError, ValueError):
        pass
    return 6650.0 if fallback else None


def cpu_baseline_sample(workload, case):
    """SHOCK's own CPU code (oracle/_ref) on a bounded sample of the workload:
    one single-block process per host core, a few RK4 steps each."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from refbind import ref_available
    if not ref_available(case.order, case.dim):
        return None
    try:
        mpi = mpi_reference(workload, CPU_BASELINE_STEPS, 1)
    except (OSError, RuntimeError) as e:      # the sample is reported, not required
        print(f"bench: SHOCK's MPI-path sample skipped: {e}", file=sys.stderr)
        mpi = None
    spec, pts, what = ref_sample(workload)
    procs = ref_procs(pts, case.order)
    v, tmax, _ = reference_throughput(spec, CPU_BASELINE_STEPS, 1, procs)
    replicas = {"value": v, "unit": "cell-stage updates/s", "cores": procs, "kind": "reference",
                "sample": f"{procs} single-block processes x {CPU_BASELINE_STEPS} timed RK4 steps (after 1 warm-up "
                          f"step) of {what}, SHOCK's own C code (oracle/_ref); {tmax:.1f} s"}
    if mpi is None:
        return replicas
    mpi["single_block_replicas"] = replicas
    return mpi


CPU_BASELINE_STEPS = 3


def l2_conserved(case, a, r):
    """Relative L2 of each conserved variable (rho, rho u, rho v, rho w, rho e)
    over the real points between two states of SHOCK's variables; one
    variable at a time, so a 512^3 block needs little extra host memory."""
    import numpy as np
    g = case.ghosts
    sl = (slice(g, g + case.ni), slice(g, g + case.nj), slice(g, g + case.nk) if case.dim == 3 else slice(None))
    ra, rr = a[0][sl], r[0][sl]
    out = np.zeros(5)
    for k in range(5):
        ca = ra if k == 0 else ra * a[k][sl]
        cr = rr if k == 0 else rr * r[k][sl]
        den = float(np.sqrt(np.mean(np.square(cr))))
        num = float(np.sqrt(np.mean(np.square(ca - cr))))
        out[k] = 0.0 if den == 0 and num == 0 else num / (den or 1.0)
    return out


def run_batch(args, world, rank, local, barrier, max_over_ranks):
    """Batched ensemble: all members advance together, one persistent launch
    (or one launch per phase, as tuned) per RK stage, one CUDA graph per step.
    value: mixed-precision batch, device time; FP64 batch beside it; every
    mixed member checked against its FP64 solve (relative L2 per conserved
    variable, max over members).  The batch state (about 2.3 GB) is larger
    than L2, so no flush is needed between steps."""
    import numpy as np
    import shock_b200
    from shock_b200 import autotune
    cs = batch_cases()
    pts = sum(c.real_points for c in cs)
    nstage = 4
    need = sum(shock_b200.member_bytes(c) for c in cs)
    arena = int(need * 1.05) + (256 << 20)
    out = {}
    for prec in (shock_b200.SHOCK_MIXED, shock_b200.SHOCK_FP64):
        entry = autotune.lookup(2, 5, prec, cs)
        tuned_now = entry is None
        if tuned_now:
            entry = autotune.tune(cs, 2, 5, prec, device=local, budget_s=args.tune_budget)
        b = shock_b200.Batch(2, 5, prec, arena_bytes=arena, device=local)
        ms = [b.add(c, args.warmup + args.steps) for c in cs]
        autotune.apply(b, entry)
        b.step(args.warmup)
        barrier()
        total = 0.0
        sampler = ClockSampler(local)
        sampler.start()
        for _ in range(args.steps):
            b.step(1)
            total += b.last_ms()
        clocks = sampler.stop()
        barrier()
        total = max_over_ranks(total)
        out[prec] = {"ms": total, "info": b.info(), "tuning": {k: entry[k] for k in
                                                               ("persistent", "blocks_per_sm", "chunk", "small_tile_max")},
                     "tuned_now": tuned_now, "clocks": clocks, "states": [b.state(m) for m in ms]}
        b.close()
    worst = np.zeros(5)
    for c, sm, s64 in zip(cs, out[shock_b200.SHOCK_MIXED]["states"], out[shock_b200.SHOCK_FP64]["states"]):
        worst = np.maximum(worst, l2_conserved(c, sm, s64))
    # the persistent form (one cooperative launch per RK stage) beside the
    # tuner's choice, mixed precision
    bp = shock_b200.Batch(2, 5, shock_b200.SHOCK_MIXED, arena_bytes=arena, device=local)
    for c in cs:
        bp.add(c, args.warmup + args.steps)
    bp.set_tuning(persistent=1, blocks_per_sm=1)
    occ = bp.tuning().max_blocks_per_sm
    bp.set_tuning(persistent=1, blocks_per_sm=occ, chunk=1024)
    bp.step(args.warmup)
    barrier()
    pers_ms = 0.0
    for _ in range(args.steps):
        bp.step(1)
        pers_ms += bp.last_ms()
    pers_launches = bp.info()["kernels_per_step"]
    bp.close()
    pers_ms = max_over_ranks(pers_ms)

    mixed_ms = out[shock_b200.SHOCK_MIXED]["ms"]
    fp64_ms = out[shock_b200.SHOCK_FP64]["ms"]
    value = pts * nstage * args.steps * world / (mixed_ms * 1e-3)
    fp64_value = pts * nstage * args.steps * world / (fp64_ms * 1e-3)

    # end to end through the C ABI: host arrays in, host results out
    barrier()
    t0 = time.perf_counter()
    b = shock_b200.Batch(2, 5, shock_b200.SHOCK_MIXED, arena_bytes=arena, device=local)
    autotune.apply(b, autotune.lookup(2, 5, shock_b200.SHOCK_MIXED, cs))
    ms = [b.add(c, args.steps) for c in cs]
    b.step(args.steps)
    h2d = d2h = 0
    for m, c in zip(ms, cs):
        st = b.state(m)
        d2h += st.nbytes
        h2d += 8 * 8 * c.real_points
    b.close()
    t1 = time.perf_counter()
    barrier()
    e2e_s = max_over_ranks(t1 - t0)

    fl = flops_per_cell_stage(cs[0])["total"]
    peaks = measure_peaks(local)
    ach64 = fl * pts * nstage * args.steps / (fp64_ms * 1e-3) / 1e12
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from refbind import ref_available
        if ref_available(5, 2):
            procs = ref_procs(256 ** 2, 5)
            v, t = batch_reference_sample(procs, steps=1, warmup=1)
            cpu = {"value": v, "unit": "cell-stage updates/s", "cores": procs, "kind": "reference",
                   "sample": f"first {procs} batch members, one SHOCK process each (oracle/_ref), 1 timed RK4 step; "
                             f"{t:.1f} s"}
    if rank == 0:
        mix = out[shock_b200.SHOCK_MIXED]
        print(json.dumps({
            "metric": "cell-stage updates/s", "value": value, "unit": "cell-stage updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": mixed_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64 mixed",
            "data": "synthetic",
            "config": {"workload": args.workload, "description": WORKLOADS[args.workload], "members": len(cs),
                       "points": pts, "stages_per_step": nstage, "l2": "state (2.3 GB) larger than L2",
                       "parallelism": f"replicas x{world}", "tuning": mix["tuning"],
                       "launches_per_step": mix["info"]["kernels_per_step"]},
            "fp64": {"value": fp64_value, "ms_per_step": fp64_ms / args.steps,
                     "tuning": out[shock_b200.SHOCK_FP64]["tuning"]},
            "persistent_form": {"value": pts * nstage * args.steps * world / (pers_ms * 1e-3),
                                "ms_per_step": pers_ms / args.steps, "launches_per_step": pers_launches,
                                "note": "one cooperative launch per RK stage with grid barriers, mixed"},
            "mixed_speedup": fp64_ms / mixed_ms,
            "mixed_vs_fp64_l2_max_over_members": {"rho": worst[0], "rho_u": worst[1], "rho_v": worst[2],
                                                  "rho_e": worst[4]},
            "e2e": {"value": pts * nstage * args.steps * world / e2e_s, "unit": "cell-stage updates/s",
                    "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                    "note": f"one full solve of all members: set-up from host arrays, {args.steps} steps, download"},
            "gpu_launches": mix["info"]["kernels_per_step"] * args.steps,
            "roofline": {"bound": "fp64", "kernel": "whole batched step (FP64 form)", "achieved": ach64,
                         "peak": peaks["fp64_tflops"], "unit": "TFLOP/s", "frac": ach64 / peaks["fp64_tflops"],
                         "traffic": None, "flops_per_cell_stage": fl},
            "cpu_baseline": cpu, "clocks": mix["clocks"],
        }))


def run_serve(args, world, rank, local, barrier, max_over_ranks):
    """Serving stream: requests submitted at their Poisson arrival times to
    the C request loop; time to solution per request (p50/p99) and aggregate
    cell-stage updates/s, FP64 and mixed; beside it the same requests
    submitted at once (the batched throughput the stream is compared with)."""
    import numpy as np
    import shock_b200
    from shock_b200 import cases
    stream = cases.serving_stream(args.requests, seed=5 + rank)
    res = {}
    for prec in (shock_b200.SHOCK_FP64, shock_b200.SHOCK_MIXED):
        for mode in ("poisson", "batched"):
            srv = shock_b200.Server(hbm_budget=int(args.hbm_gb * 1e9), device=local)
            barrier()
            t0 = time.perf_counter()
            ids = []
            for t_arr, case, n in stream:
                if mode == "poisson":
                    dt = t_arr - (time.perf_counter() - t0)
                    if dt > 0:
                        time.sleep(dt)
                ids.append(srv.submit(case, n, prec))
            infos = []
            for rid in ids:
                srv.wait(rid, 3600.0)
                infos.append(srv.result(rid)[1])
            t1 = time.perf_counter()
            st = srv.stats()
            srv.close()
            tts = np.array([i["tts_s"] for i in infos])
            cells = sum(i["cell_stages"] for i in infos)
            res[(prec, mode)] = {"p50_s": float(np.percentile(tts, 50)), "p99_s": float(np.percentile(tts, 99)),
                                 "throughput": cells / (t1 - t0), "wall_s": t1 - t0, "rounds": st["rounds"],
                                 "cell_stages": cells, "busy_ms": st["busy_ms"]}
    if rank == 0:
        f64, mix = res[(shock_b200.SHOCK_FP64, "poisson")], res[(shock_b200.SHOCK_MIXED, "poisson")]
        bf, bm = res[(shock_b200.SHOCK_FP64, "batched")], res[(shock_b200.SHOCK_MIXED, "batched")]
        print(json.dumps({
            "metric": "time to solution p50/p99 (s) and cell-stage updates/s", "value": f64["throughput"] * world,
            "unit": "cell-stage updates/s", "n_gpus": world, "steps": len(stream), "warmup": 0,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "description": WORKLOADS[args.workload],
                       "requests": len(stream), "hbm_budget_gb": args.hbm_gb, "parallelism": f"replicas x{world}"},
            "fp64": {k: f64[k] for k in ("p50_s", "p99_s", "throughput", "wall_s", "rounds")},
            "mixed": {k: mix[k] for k in ("p50_s", "p99_s", "throughput", "wall_s", "rounds")},
            "batched": {"fp64": bf["throughput"], "mixed": bm["throughput"]},
            "p99_over_p50": {"fp64": f64["p99_s"] / f64["p50_s"], "mixed": mix["p99_s"] / mix["p50_s"]},
            "stream_over_batched": {"fp64": f64["throughput"] / bf["throughput"],
                                    "mixed": mix["throughput"] / bm["throughput"]},
            "e2e": {"value": f64["throughput"] * world, "unit": "cell-stage updates/s",
                    "note": "requests enter as host arrays and results return to host memory"},
        }))


def measure_peaks(device):
    import ctypes as C
    import shock_b200
    a, b = C.c_double(), C.c_double()
    shock_b200.lib().shock_measure_fma_peak(device, C.byref(a), C.byref(b))
    return {"fp64_tflops": a.value, "fp32_tflops": b.value}


if __name__ == "__main__":
    main()
