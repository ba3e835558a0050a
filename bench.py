"""Benchmark: cell-stage updates/s of SHOCK's per-RK-stage right-hand side.

Default workload (N=1): the 3D curvilinear Taylor-Green vortex, 64^3
periodic points with every coordinate perturbed by x_i += 0.05 sin(x_j)
sin(x_k), Ma = 0.1, Re = 1600, WENO5, viscous, RK4, FP64 (plain form).
A step is one RK4 time step (4 stage right-hand sides + updates) over the
whole block.  Inputs are synthetic (seedless analytic initial state).

Metric: cell-stage updates/s = real points x stages x steps x ranks / time.
  value  -- device time with the state resident in HBM (CUDA events on the
            solver's stream around each step's graph), the L2 flushed
            (256 MiB write) between timed steps because the 64^3 state fits
            in the 126 MB L2.
  e2e    -- the same steps through the public C ABI with host buffers:
            every step uploads the state from pinned host memory
            (shock_upload_state), runs it (shock_step) and reads the state
            back (shock_download_state); host wall clock around the three
            synchronous calls.
The mixed form (FP32 stencils, FP64 state) is reported beside it.

--impl reference: SHOCK's own CPU code (oracle/_ref, the unmodified
reference sources) on the same workload, one single-block process per host
core, each advancing its own copy; aggregate cell-stage/s over a bounded
sample of steps.  Under torchrun only rank 0 runs it.

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


def measured_traffic(workload, kernel, precision="fp64"):
    """DRAM bytes (read + write) of one launch of `kernel` on `workload`, from
    the ncu capture recorded in shock_b200/roofline.json (None if absent)."""
    path = os.path.join(ROOT, "shock_b200", "roofline.json")
    with open(path) as f:
        t = json.load(f).get("traffic", {})
    e = t.get(workload, {}).get(precision, {}).get(kernel)
    return None if e is None else e["bytes"]


def flops_per_cell_stage(case):
    path = os.path.join(ROOT, "shock_b200", "roofline.json")
    with open(path) as f:
        counts = json.load(f)["counts"]
    key = f"{case.dim}d_w{case.order}_{'inviscid' if case.inviscid else 'viscous'}"
    return counts[key]


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
    name, nsteps = args
    # SHOCK's own code reports its set-up on stdout; keep the bench's stdout
    # to the one JSON line
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from refbind import RefSolver
    if isinstance(name, tuple):          # (builder name, kwargs) of shock_b200.cases
        from shock_b200 import cases
        case = getattr(cases, name[0])(**name[1])
    else:
        case = make_case(name)
    r = RefSolver(case)
    r.steps(1)                      # warm-up (first touch)
    t = r.time_steps(nsteps)
    return t, case.real_points * case.time_order * nsteps


def reference_throughput(name, steps, procs):
    ctx = mp.get_context("spawn")
    spec = CPU_SAMPLE.get(name, name)
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker, [(spec, steps)] * procs)
    tmax = max(t for t, _ in res)
    cells = sum(c for _, c in res)
    return cells / tmax, tmax, res


# SHOCK's CPU build keeps about 300 doubles per ghosted point, so a 512^3
# block (about 340 GB) does not fit in host memory: the reference arm of the
# 512^3 workloads times 128^3 blocks of the same flow and order instead and
# reports per-cell-stage rates.
CPU_SAMPLE = {
    "turb512_w9": ("decaying_turbulence", {"n": 128, "order": 9}),
    "tgv512_w5": ("taylor_green", {"n": 128, "order": 5}),
}


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


def batch_reference_sample(procs, steps=1, seed=4):
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
        res = pool.map(_ref_worker, [(sp, steps) for sp in specs[:procs]])
    tmax = max(t for t, _ in res)
    cells = sum(c for _, c in res)
    return cells / tmax, tmax


def run_reference(args, rank):
    if rank != 0:
        return
    if args.workload == "batch_vortex256":
        procs = ref_procs(256 ** 2, 5)
        v, t = batch_reference_sample(procs, steps=max(1, min(args.steps, args.ref_steps)))
        print(json.dumps({
            "metric": "cell-stage updates/s", "value": v, "unit": "cell-stage updates/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "description": WORKLOADS[args.workload]},
            "cpu_baseline": {"value": v, "unit": "cell-stage updates/s", "cores": procs, "kind": "reference",
                             "sample": f"first {procs} batch members, one SHOCK process each (oracle/_ref), "
                                       f"timed RK4 steps; {t:.1f} s"},
            "e2e": {"value": v, "unit": "cell-stage updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    if args.workload == "serve_poisson":
        print(json.dumps({"impl": "reference", "unavailable": "SHOCK has no request loop; its per-block CPU "
                                                                "throughput is the tgv64_w5 / batch_vortex256 reference arms"}))
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from refbind import ref_available
    order, dim = (9, 3) if "w9" in args.workload else (5, 3 if args.workload != "mms64_w5" else 2)
    if not ref_available(order, dim):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent)"}))
        return
    sample = CPU_SAMPLE.get(args.workload)
    case = make_case(args.workload) if sample is None else None
    pts = case.real_points if case is not None else sample[1]["n"] ** 3
    procs = ref_procs(pts, order)
    steps = max(1, min(args.steps, args.ref_steps))
    v, t, _ = reference_throughput(args.workload, steps, procs)
    what = f"the {args.workload} block" if sample is None else \
        f"a {sample[1]['n']}^3 block of the same flow and order (512^3 does not fit in host memory)"
    line = {
        "metric": "cell-stage updates/s", "value": v, "unit": "cell-stage updates/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": pts * 4 * 1e3 / v * procs, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "description": WORKLOADS[args.workload],
                   "points": pts, "stages_per_step": 4},
        "cpu_baseline": {"value": v, "unit": "cell-stage updates/s", "cores": procs, "kind": "reference",
                         "sample": f"{procs} single-block processes x {steps} timed RK4 steps (after 1 warm-up step) "
                                   f"of {what}, SHOCK's own C code (oracle/_ref); {t:.1f} s"},
        "e2e": {"value": v, "unit": "cell-stage updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="tgv64_w5", choices=sorted(WORKLOADS))
    ap.add_argument("--ref-steps", type=int, default=3, help="cap on timed RK steps in the reference arm")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--tune-budget", type=float, default=60.0, help="seconds the batch autotuner may spend")
    ap.add_argument("--requests", type=int, default=48, help="serve_poisson: requests in the stream")
    ap.add_argument("--hbm-gb", type=float, default=150.0, help="serve_poisson: HBM budget")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank)
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
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def timed_device(precision):
        s = shock_b200.Solver(case, precision=precision, device=local)
        for _ in range(args.warmup):
            s.steps(1)
        barrier()
        total_ms = 0.0
        for _ in range(args.steps):
            flush_l2(torch, flush)
            torch.cuda.synchronize()
            s.steps(1)
            total_ms += s.last_ms()
        barrier()
        return s, total_ms

    sampler = ClockSampler(local)
    sampler.start()
    solver, ms64 = timed_device(shock_b200.SHOCK_FP64)
    clocks = sampler.stop()
    ms64 = max_over_ranks(ms64)
    value = replica_value(stage_cells * args.steps, world, ms64 * 1e-3)

    mixed = None
    if not args.no_mixed:
        try:
            smix, msmix = timed_device(shock_b200.SHOCK_MIXED)
            msmix = max_over_ranks(msmix)
            mixed = {"value": stage_cells * args.steps * world / (msmix * 1e-3),
                     "ms_per_step": msmix / args.steps}
            del smix
        except shock_b200.ShockError as e:
            mixed = {"error": str(e)}

    # end to end through the C ABI with pinned host buffers
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

    # per-kernel profile of one stage and the roofline of the dominant kernel
    prof = solver_profile(solver)
    fl = flops_per_cell_stage(case)
    peaks = measure_peaks(local)
    dom = max(prof, key=lambda kv: kv[1]) if prof else ("n/a", 0.0)
    dom_flops = fl.get(dom[0], 0.0) * case.real_points
    achieved = dom_flops / (dom[1] * 1e-3) / 1e12 if dom[1] > 0 else None
    roofline = {"bound": "fp64", "kernel": dom[0], "achieved": achieved, "peak": peaks["fp64_tflops"],
                "unit": "TFLOP/s", "frac": (achieved / peaks["fp64_tflops"]) if achieved else None,
                "traffic": measured_traffic(args.workload, dom[0]),
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch, "
                                  "shock_b200/roofline.json (command recorded there)",
                "peak_source": "measured on this GPU by shock_measure_fma_peak (register-only FP64 FMA loop)",
                "flops_per_launch": dom_flops, "launch_ms": dom[1],
                "step_fp64_tflops": fl["total"] * stage_cells * args.steps / (ms64 * 1e-3) / 1e12,
                "step_frac": fl["total"] * stage_cells * args.steps / (ms64 * 1e-3) / 1e12 / peaks["fp64_tflops"],
                "kernels_ms": {k: v for k, v in prof}}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from refbind import ref_available
        if ref_available(case.order, case.dim):
            sample = CPU_SAMPLE.get(args.workload)
            pts = case.real_points if sample is None else sample[1]["n"] ** 3
            procs = ref_procs(pts, case.order)
            v, tmax, _ = reference_throughput(args.workload, 1, procs)
            what = f"the {args.workload} block" if sample is None else \
                f"a {sample[1]['n']}^3 block of the same flow and order (512^3 does not fit in host memory)"
            cpu = {"value": v, "unit": "cell-stage updates/s", "cores": procs, "kind": "reference",
                   "sample": f"{procs} single-block processes x 1 RK4 step of {what}, "
                             f"SHOCK's own C code (oracle/_ref); {tmax:.1f} s"}

    if rank == 0:
        line = {
            "metric": "cell-stage updates/s", "value": value, "unit": "cell-stage updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms64 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "description": WORKLOADS[args.workload],
                       "points": case.real_points, "stages_per_step": case.time_order,
                       "l2": "flushed (256 MiB write) between timed steps",
                       "parallelism": f"replicas x{world}"},
            "mixed": mixed, "e2e": e2e, "gpu_launches": solver.kernels_per_step() * args.steps,
            "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
            "fp32_peak_tflops": peaks["fp32_tflops"],
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def _l2_conserved(case, a, r):
    """Relative L2 of each conserved variable (real points) between two states."""
    import numpy as np
    g = case.ghosts
    sl = (slice(None), slice(g, g + case.ni), slice(g, g + case.nj),
          slice(g, g + case.nk) if case.dim == 3 else slice(None))
    a, r = a[sl], r[sl]
    ca = np.stack([a[0], a[0] * a[1], a[0] * a[2], a[0] * a[3], a[0] * a[4]])
    cr = np.stack([r[0], r[0] * r[1], r[0] * r[2], r[0] * r[3], r[0] * r[4]])
    out = np.zeros(5)
    for k in range(5):
        den = np.sqrt(np.mean(cr[k] ** 2))
        num = np.sqrt(np.mean((ca[k] - cr[k]) ** 2))
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
        worst = np.maximum(worst, _l2_conserved(c, sm, s64))
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
            v, t = batch_reference_sample(procs, steps=1)
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


def solver_profile(solver):
    import ctypes as C
    L = solver.lib
    names = C.create_string_buffer(48 * 32)
    ms = (C.c_float * 32)()
    cnt = C.c_int()
    best = {}
    for _ in range(5):
        rc = L.shock_profile_stage(solver.h, 32, names, ms, C.byref(cnt))
        if rc != 0:
            return []
        for i in range(cnt.value):
            nm = names.raw[48 * i:48 * i + 48].split(b"\0")[0].decode()
            best[nm] = min(best.get(nm, 1e30), ms[i])
    return list(best.items())


def measure_peaks(device):
    import ctypes as C
    import shock_b200
    a, b = C.c_double(), C.c_double()
    shock_b200.lib().shock_measure_fma_peak(device, C.byref(a), C.byref(b))
    return {"fp64_tflops": a.value, "fp32_tflops": b.value}


if __name__ == "__main__":
    main()
