"""GPU parity of the FP32-mixed mode against the FP64 oracle.

The mixed mode computes the REBO / torsion bond orders and the plain LJ pairs
in FP32 (splines re-expanded in cell-local coordinates), and keeps in FP64
the pair exponentials, the LJ powers, switches and connectivity products,
the b* bond orders of close non-bonded pairs, all accumulation and the
integration.  Bars (forces, at thermal displacements): ||F - F_ref|| /
||F_ref|| <= 1e-5 and max |F - F_ref| / RMS(F_ref) <= 1e-5; energy within
1e-6 of the sum of the magnitudes of the oracle's terms."""
import numpy as np
import pytest

import mdtk_b200 as M
from mdtk_b200 import builders as B
from oracle import ref

pytestmark = pytest.mark.gpu

TOL_F_MIXED = 1e-5       # ||dF||/||F|| and max|dF|/rms(F)
TOL_E_MIXED = 1e-6       # |dE| / sum |E_term|


def _displaced(s, sigma, seed):
    rng = np.random.default_rng(seed)
    s = dict(s)
    s["pos"] = s["pos"] + rng.normal(0.0, sigma, s["pos"].shape)
    return s


SYSTEMS = {
    "ethane30_thermal": lambda: _displaced(B.ethane_liquid(30, seed=41, min_dist=1.6, jitter=0.4), 0.03, 1),
    "diamond4_disp": lambda: B.diamond(4, disp_sigma=0.1, seed=42),
    "diamond4_hot": lambda: B.diamond(4, disp_sigma=0.25, seed=43),
    "ach300": lambda: B.amorphous_carbon(300, h_fraction=0.25, seed=44),
    "ac300": lambda: B.amorphous_carbon(300, seed=45),
    "ach500_dense": lambda: B.amorphous_carbon(500, h_fraction=0.4, density_g_cm3=1.5, min_sep=1.0, seed=46),
}

POTS = {
    "airebo": (M.POT_AIREBO, ref.POT_AIREBO),
    "rebo": (M.POT_REBO, ref.POT_REBO),
    "rebo_tors": (M.POT_REBO | M.POT_ETORS, ref.POT_REBO | ref.POT_ETORS),
}


def _ctx(s, pot, precision=M.PREC_FP32_MIXED, task_mode=0):
    ctx = M.Context(potentials=pot, precision=precision, task_mode=task_mode)
    ctx.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    return ctx


def _oracle(s, pot):
    r = ref.RefSystem(pot)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    return r.compute()


def force_errors(g, go):
    d = g - go
    rel = float(np.linalg.norm(d) / np.linalg.norm(go))
    maxrms = float(np.abs(d).max() / np.sqrt((go ** 2).mean()))
    return rel, maxrms


@pytest.mark.parametrize("pot", sorted(POTS))
@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_mixed_force_error(name, pot):
    s = SYSTEMS[name]()
    pm, pr = POTS[pot]
    e, et, g = _ctx(s, pm).compute()
    eo, eto, go = _oracle(s, pr)
    rel, maxrms = force_errors(g, go)
    assert rel <= TOL_F_MIXED, f"{name}/{pot}: ||dF||/||F|| = {rel:.2e}"
    assert maxrms <= TOL_F_MIXED, f"{name}/{pot}: max|dF|/rms(F) = {maxrms:.2e}"
    scale = float(np.abs(eto[:3]).sum())
    assert abs(e - eo) <= TOL_E_MIXED * scale, (e, eo, scale)


def test_mixed_trajectory_tracks_fp64():
    # 100 steps of REBO NVE from the same state: the two precisions stay
    # within 1e-5 A (no chaotic separation yet) and their total energies
    # within 1e-6 eV per atom.
    s = B.diamond(3, temp_k=600.0, disp_sigma=0.05, seed=47)
    a = _ctx(s, M.POT_REBO, M.PREC_FP64)
    b = _ctx(s, M.POT_REBO)
    ea = a.run(100, 0.5)[1]
    eb = b.run(100, 0.5)[1]
    pa = a.get_state()[0]
    pb = b.get_state()[0]
    d = pa - pb
    d -= s["box"] * np.round(d / s["box"])
    assert np.abs(d).max() < 1e-5
    n = len(s["z"])
    assert np.abs(eb - ea).max() / n < 1e-6


def test_mixed_nve_drift_comparable():
    s = B.diamond(4, temp_k=300.0, seed=48)
    n = len(s["z"])
    e64 = _ctx(s, M.POT_REBO, M.PREC_FP64).run(800, 0.5)[1]
    e32 = _ctx(s, M.POT_REBO).run(800, 0.5)[1]
    t = np.arange(800)[80:]
    slope64 = np.polyfit(t, e64[80:] / n, 1)[0]
    slope32 = np.polyfit(t, e32[80:] / n, 1)[0]
    # FP32 arithmetic adds no drift: the fitted per-atom slopes differ by
    # less than 1e-8 eV per step
    assert abs(slope32 - slope64) < 1e-8, (slope32, slope64)
    assert np.ptp(e32[80:]) / n < 2e-4


def test_mixed_deterministic_and_graph():
    # one REBO split for both (the autotuner may time two splits as equal
    # and keep either; splits agree to rounding, not bit for bit)
    s = SYSTEMS["ach300"]()
    a = _ctx(s, M.POT_AIREBO, task_mode=2)
    b = _ctx(s, M.POT_AIREBO, task_mode=2)
    a.run(10, 0.25, energies=False)   # graph replay
    b.run(10, 0.25, energies=True)    # eager, energies each step
    pa, va, _ = a.get_state()
    pb, vb, _ = b.get_state()
    assert np.array_equal(pa, pb) and np.array_equal(va, vb)
