"""Autotuner for batched execution (shock_batch_tuning).

For a batch class (dimension, WENO order, precision, viscous or not) and a
representative set of members, every launch configuration in the search
space is timed on a scratch batch holding copies of those members (the
caller's own batch never advances), and the fastest one is kept:

  persistent      one cooperative launch per RK stage, or one launch per phase
  blocks_per_sm   resident 256-thread tiles per SM (1 .. occupancy limit)
  chunk           points per item of the point-wise phases
  small_tile_max  members whose longest axis is at most this many points sweep
                  with 7-cell tiles (one face per thread) instead of 15-cell
                  tiles: short lines waste less of a tile, long lines stage
                  less halo per cell.

Results are kept in a JSON table keyed by the class and the members' size
class, so a batch of similar composition reuses them without timing again
(shock_b200/tuning.json by default; SHOCK_B200_TUNING overrides the path).
"""
from __future__ import annotations

import itertools
import json
import math
import os
import time

from . import Batch, SHOCK_FP64, SHOCK_MIXED

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.environ.get("SHOCK_B200_TUNING", os.path.join(HERE, "tuning.json"))

CHUNKS = (1024, 4096)
SMALL_TILE = (0, 64, 128, 1 << 30)


def class_key(dim: int, order: int, precision: int, cases) -> str:
    """Table key: the batch class plus the members' size class (log2 of the
    mean real points per member, rounded) and whether any member is viscous."""
    visc = any(not c.inviscid for c in cases)
    mean = sum(c.real_points for c in cases) / max(1, len(cases))
    size = int(round(math.log2(max(mean, 1.0))))
    prec = "mixed" if precision == SHOCK_MIXED else "fp64"
    return f"{dim}d_w{order}_{prec}_{'visc' if visc else 'inv'}_s{size}"


def load_table(path: str = TABLE) -> dict:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save_table(table: dict, path: str = TABLE):
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _time(batch: Batch, steps: int, reps: int) -> float:
    batch.step(1)   # capture + warm
    best = float("inf")
    for _ in range(reps):
        batch.step(steps)
        best = min(best, batch.last_ms() / steps)
    return best


def tune(cases, dim: int, order: int, precision=SHOCK_FP64, time_order: int = 4, steps: int = 2,
         reps: int = 3, device: int = 0, path: str = TABLE, force: bool = False, budget_s: float = 120.0,
         arena_bytes: int | None = None) -> dict:
    """Best tuning for batches like `cases` (a list of shock_b200.cases.Case).
    Reuses the table entry unless force; otherwise times the search space
    (bounded by budget_s seconds) and stores the winner."""
    key = class_key(dim, order, precision, cases)
    table = load_table(path)
    if key in table and not force:
        return table[key]
    from . import member_bytes
    need = sum(member_bytes(c, precision) for c in cases)
    arena = arena_bytes or int(need * 1.05) + (64 << 20)
    b = Batch(dim, order, precision, time_order=time_order, arena_bytes=arena, device=device)
    for c in cases:
        b.add(c, 1 << 30)
    t0 = time.time()
    results = []
    try:
        for persistent in (1, 0):
            b.set_tuning(persistent=persistent, blocks_per_sm=1)
            occ = b.tuning().max_blocks_per_sm
            for bps, chunk, small in itertools.product(range(1, max(1, occ) + 1), CHUNKS, SMALL_TILE):
                if time.time() - t0 > budget_s:
                    break
                b.set_tuning(persistent=persistent, blocks_per_sm=bps, chunk=chunk, small_tile_max=small)
                ms = _time(b, steps, reps)
                results.append({"persistent": persistent, "blocks_per_sm": bps, "chunk": chunk,
                                "small_tile_max": small, "ms_per_step": ms})
    finally:
        b.close()
    results.sort(key=lambda r: r["ms_per_step"])
    best = dict(results[0])
    best["candidates"] = len(results)
    best["members"] = len(cases)
    best["points"] = sum(c.real_points for c in cases)
    table = load_table(path)
    table[key] = best
    save_table(table, path)
    return best


def apply(batch: Batch, entry: dict):
    """Set a table entry on a batch."""
    batch.set_tuning(persistent=entry["persistent"], blocks_per_sm=entry["blocks_per_sm"],
                     chunk=entry["chunk"], small_tile_max=entry["small_tile_max"])


def lookup(dim: int, order: int, precision, cases, path: str = TABLE):
    """Table entry for batches like `cases`, or None."""
    return load_table(path).get(class_key(dim, order, precision, cases))
