#!/usr/bin/env python
"""Algorithmic FP64 operation counts per atom for the per-step hot path.

Test/measurement infrastructure: runs the op-counting instantiation of the
CPU restatement (restate.cpp, scalar type `Counted`) on the step-0 state of a
workload and prints the per-atom counts of each term, raw and weighted.  The
weighted figures are the `flops_per_atom` constants that bench.py divides by
a kernel's measured time for its roofline entry.

Conventions (stated once, used everywhere):
  * add/sub, mul = 1 flop (an FMA is 2, matching the FP64 pipe peak, which
    counts an FMA as 2 flops);
  * div 4, sqrt 4, exp 12, cos 12, pow 24 - the FMA-class operation counts of
    a plain software evaluation (Newton-Raphson reciprocal/root from a seed;
    range reduction plus a polynomial for exp/cos; pow as exp(y*log x));
  * the restatement computes the energy only; energy + gradient is counted
    as 3x the energy's operations (one forward and a reverse sweep of about
    twice its cost - the cheap-gradient bound of reverse-mode differentiation).

    python oracle/opcount.py [--molecules 5461] [--seed 1]
"""
from __future__ import annotations

import argparse
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

WEIGHTS = {"add": 1, "mul": 1, "div": 4, "sqrt": 4, "exp": 12, "cos": 12, "pow": 24}
GRAD_FACTOR = 3


def weighted(c: dict) -> float:
    return float(sum(WEIGHTS[k] * v for k, v in c.items()))


def counts(s) -> dict:
    from oracle import ref
    n = len(s["z"])
    rebo = ref.rs_opcount(s, 1)
    rt = ref.rs_opcount(s, 5)
    rl = ref.rs_opcount(s, 3)
    bst = ref.rs_opcount(s, 3, bstar=True)
    sub = lambda a, b: {k: a[k] - b[k] for k in a}
    terms = {"rebo": rebo, "tors": sub(rt, rebo), "lj_total": sub(rl, rebo), "lj_bstar": bst}
    terms["lj_pairs"] = sub(terms["lj_total"], bst)
    out = {"atoms": n, "weights": WEIGHTS, "grad_factor": GRAD_FACTOR, "terms": {}}
    for k, c in terms.items():
        out["terms"][k] = {"raw_per_atom": {o: v / n for o, v in c.items()},
                           "energy_flops_per_atom": weighted(c) / n,
                           "flops_per_atom": GRAD_FACTOR * weighted(c) / n}
    return out


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--molecules", type=int, default=5461)
    ap.add_argument("--seed", type=int, default=1)
    a = ap.parse_args()
    from mdtk_b200 import builders as B
    s = B.ethane_liquid(a.molecules, density_g_cm3=0.55, temp_k=300.0, seed=a.seed)
    print(json.dumps(counts(s), indent=1))
    return 0


if __name__ == "__main__":
    sys.exit(main())
