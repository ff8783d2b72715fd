"""Regenerate the golden fixtures in this folder from the oracle (the
reference MDTK compiled from its own sources, oracle/_ref/libmdtkref.so).

    python tests/golden/make_golden.py

Each fixture holds one seeded system, the oracle's per-potential energies and
total gradient for one potential stack, the sorted Verlet pair sets of every
list, and the oracle's 1-ulp reproducibility floor for that system."""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from mdtk_b200 import builders as B  # noqa: E402
from oracle import ref  # noqa: E402
from parity import oracle_floor  # noqa: E402

CASES = {
    "c2h6_rebo": (lambda: B.c2h6_example(), ref.POT_REBO),
    "c2h6_brenner1": (lambda: B.c2h6_example(), ref.POT_BRENNER),
    "diamond3_disp_rebo_tors": (lambda: B.diamond(3, disp_sigma=0.15, seed=11), ref.POT_REBO | ref.POT_ETORS),
    "ach200_rebo_tors": (lambda: B.amorphous_carbon(200, h_fraction=0.3, seed=12), ref.POT_REBO | ref.POT_ETORS),
    "ethane30_airebo": (lambda: B.ethane_liquid(30, seed=13, min_dist=1.6, jitter=0.4), ref.POT_AIREBO),
    "diamond4_disp_airebo": (lambda: B.diamond(4, disp_sigma=0.1, seed=14), ref.POT_AIREBO),
    "ach300_airebo": (lambda: B.amorphous_carbon(300, h_fraction=0.25, seed=15), ref.POT_AIREBO),
}


def make(name):
    build, pot = CASES[name]
    s = build()
    r = ref.RefSystem(pot, 2 if "brenner2" in name else 1)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    e, et, g = r.compute()
    pairs = [r.nl_pairs(i) for i in range(r.npot)]
    fe, ff = oracle_floor(lambda: ref.RefSystem(pot, 2 if "brenner2" in name else 1), s)
    out = dict(s)
    out.update(potset=pot, e_total=e, e_terms=et, grad=g, floor=np.array([fe, ff]))
    for i, p in enumerate(pairs):
        out[f"pairs{i}"] = p
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(f"{name}: n={len(s['z'])} E={e:.12f} floor=({fe:.2e}, {ff:.2e})")


if __name__ == "__main__":
    for name in (sys.argv[1:] or CASES):
        make(name)
