"""Shared parity helpers for the tests.

The reference evaluates its correction splines as monomials in absolute
coordinates whose terms cancel heavily, so perturbing its inputs by one ulp
moves its energy and forces by far more than one ulp.  `oracle_floor`
measures that reproducibility floor for a configuration; parity bounds are
max(fixed tolerance, FLOOR_FACTOR * floor).

Every `assert_parity` call records the achieved errors beside the floor and
the bound it was held to (`RECORDS`); the session prints them as a table and,
when the environment names a file in MDG_PARITY_LOG, writes them there as
JSON lines."""
from __future__ import annotations

import numpy as np

TOL_E = 1e-12      # relative energy, FP64
TOL_F = 1e-10      # ||dF|| / ||F||, FP64
FLOOR_FACTOR = 4.0
RECORDS: list = []


def rel_e(e, eo):
    return abs(e - eo) / max(abs(eo), 1e-300)


def rel_f(g, go):
    return float(np.linalg.norm(g - go) / max(np.linalg.norm(go), 1e-300))


def oracle_floor(make_ref, s, samples: int = 3, seed: int = 0):
    """(energy, force) relative spread of the oracle under 1-ulp input perturbations."""
    r = make_ref()
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s.get("fixed"))
    e0, _, g0 = r.compute()
    rng = np.random.default_rng(seed)
    fe, ff = 0.0, 0.0
    for _ in range(samples):
        p = s["pos"] * (1 + rng.choice([-1.0, 1.0], size=s["pos"].shape) * 2.0 ** -52)
        r = make_ref()
        r.set_atoms(s["z"], p, s["vel"], s["box"], s["pbc"], s.get("fixed"))
        e1, _, g1 = r.compute()
        fe = max(fe, rel_e(e1, e0))
        ff = max(ff, rel_f(g1, g0))
    return fe, ff


def assert_parity(e, g, eo, go, floor=(0.0, 0.0), tol_e=TOL_E, tol_f=TOL_F, label=""):
    be = max(tol_e, FLOOR_FACTOR * floor[0])
    bf = max(tol_f, FLOOR_FACTOR * floor[1])
    re_, rf = rel_e(e, eo), rel_f(g, go)
    RECORDS.append({"label": label, "rel_e": re_, "rel_f": rf, "floor_e": float(floor[0]),
                    "floor_f": float(floor[1]), "bound_e": be, "bound_f": bf,
                    "fixed_bars_hold": bool(re_ <= tol_e and rf <= tol_f)})
    assert re_ <= be, f"{label}: energy rel err {re_:.3e} > {be:.3e} (E {e!r} vs oracle {eo!r})"
    assert rf <= bf, f"{label}: force rel err {rf:.3e} > {bf:.3e} (max abs {np.abs(g - go).max():.3e})"
