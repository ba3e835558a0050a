"""Algorithmic FLOPs per cell-stage of SHOCK's stage right-hand side.

Compiles the oracle as C++ with an operation-counting scalar
(oracle/flopcount.hpp, oracle/flopcount_main.cpp), runs one RK time step
on a periodic block and writes the per-phase counts per real point and
stage to shock_b200/roofline.json.  Every +, -, *, /, sqrt, fabs and pow
counts one.  The counts are those of SHOCK's own arithmetic (the oracle
reproduces it bit for bit), so they include the reference's redundant
work (for example the full 30-factor viscous sums on a diagonal metric).

Usage: python oracle/count_flops.py
"""
import json
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BIN = os.path.join(HERE, "_bin", "flopcount")

# (dim, order, inviscid, time_order, n) -- n is the block edge the count is taken on
COMBOS = [
    (3, 5, 0, 4, 64), (3, 9, 0, 4, 48), (3, 5, 1, 4, 64), (3, 9, 1, 4, 48),
    (2, 5, 0, 4, 256), (2, 9, 0, 4, 256), (2, 5, 1, 4, 256), (2, 9, 1, 4, 256),
]


def main():
    os.makedirs(os.path.dirname(BIN), exist_ok=True)
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fpermissive", "-w", "-o", BIN,
                    os.path.join(HERE, "flopcount_main.cpp")], check=True, cwd=HERE)
    out = {"_doc": "algorithmic FLOPs per real point per RK stage of SHOCK's arithmetic, "
                   "counted on the oracle (oracle/count_flops.py); key dim_order_viscous",
           "counts": {}}
    for dim, order, inv, to, n in COMBOS:
        r = subprocess.run([BIN, str(dim), str(order), str(inv), str(to), str(n)], check=True,
                           capture_output=True, text=True)
        key = f"{dim}d_w{order}_{'inviscid' if inv else 'viscous'}"
        d = json.loads(r.stdout)
        d["block_edge"] = n
        out["counts"][key] = d
        print(key, d["total"])
    with open(os.path.join(ROOT, "shock_b200", "roofline.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
