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
    "turb256_w9": "3D decaying turbulence 256^3, WENO9, viscous, RK4, Mt=0.6",
    "turb512_w9": "3D decaying turbulence 512^3, WENO9, viscous, RK4, Mt=0.6",
    "tgv512_w5": "3D Taylor-Green vortex 512^3, WENO5, viscous, RK4",
    "mms64_w5": "2D manufactured solution 64^2, WENO5, viscous, RK4",
}


def make_case(name):
    from shock_b200 import cases
    if name == "tgv64_w5":
        return cases.taylor_green(64, order=5)
    if name == "tgv128_w5":
        return cases.taylor_green(128, order=5)
    if name == "tgv512_w5":
        return cases.taylor_green(512, order=5)
    if name == "turb256_w9":
        return cases.decaying_turbulence(256, order=9)
    if name == "turb512_w9":
        return cases.decaying_turbulence(512, order=9)
    if name == "mms64_w5":
        return cases.mms_square(64, 5, family="baseline")
    raise SystemExit(f"unknown workload {name}")


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


def flush_l2(torch, buf):
    buf.zero_()


# ---------------------------------------------------------------------------
# reference arm (CPU)
# ---------------------------------------------------------------------------
def _ref_worker(args):
    name, nsteps = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from refbind import RefSolver
    case = make_case(name)
    r = RefSolver(case)
    r.steps(1)                      # warm-up (first touch)
    t = r.time_steps(nsteps)
    return t, case.real_points * case.time_order * nsteps


def reference_throughput(name, steps, procs):
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker, [(name, steps)] * procs)
    tmax = max(t for t, _ in res)
    cells = sum(c for _, c in res)
    return cells / tmax, tmax, res


def ref_procs():
    # one single-block SHOCK process per host core, capped so the host RAM
    # (about 0.8 GB per 64^3 reference block) is not exhausted
    return max(1, min(os.cpu_count() or 1, 32))


def run_reference(args, rank):
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from refbind import ref_available
    case = make_case(args.workload)
    if not ref_available(case.order, case.dim):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent)"}))
        return
    procs = ref_procs()
    steps = max(1, min(args.steps, args.ref_steps))
    v, t, _ = reference_throughput(args.workload, steps, procs)
    stage_cells = case.real_points * case.time_order
    line = {
        "metric": "cell-stage updates/s", "value": v, "unit": "cell-stage updates/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": stage_cells * 1e3 / v * procs, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "description": WORKLOADS[args.workload],
                   "points": case.real_points, "stages_per_step": case.time_order},
        "cpu_baseline": {"value": v, "unit": "cell-stage updates/s", "cores": procs, "kind": "reference",
                         "sample": f"{procs} single-block processes x {steps} timed RK4 steps (after 1 warm-up step) "
                                   f"of the {args.workload} block, SHOCK's own C code (oracle/_ref); {t:.1f} s"},
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

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

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
    value = stage_cells * args.steps * world / (ms64 * 1e-3)

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
        host[:] = solver.state().ravel()
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
                "traffic": None,
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
            procs = ref_procs()
            v, tmax, _ = reference_throughput(args.workload, 1, procs)
            cpu = {"value": v, "unit": "cell-stage updates/s", "cores": procs, "kind": "reference",
                   "sample": f"{procs} single-block processes x 1 RK4 step of the {args.workload} block, "
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
