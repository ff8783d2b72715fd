"""NVE energy behaviour over long runs: the GPU FP64 path against the
reference's own SimLoop (AIREBO here; REBO over 10^4 steps of the 1,728-atom
diamond in test_gpu_configs.py), and the FP32-mixed path against FP64.  Trajectories decorrelate after a few hundred steps (chaos), so the
long-run comparison is statistical: the linear drift of E_total after the
first 1% of the steps and the RMS fluctuation about that line."""
import numpy as np
import pytest

import mdtk_b200 as M
from mdtk_b200 import builders as B
from oracle import ref

pytestmark = pytest.mark.gpu


def drift_stats(etot, n_atoms, dt_fs):
    """(slope in eV/atom/ps, RMS fluctuation in eV/atom) after the first 1%."""
    k0 = max(1, len(etot) // 100)
    e = np.asarray(etot[k0:]) / n_atoms
    t = (np.arange(k0, len(etot)) + 1) * dt_fs * 1e-3
    a, b = np.polyfit(t, e, 1)
    return float(a), float(np.sqrt(np.mean((e - (a * t + b)) ** 2)))


def test_airebo_drift_matches_reference():
    """Full AIREBO (its torsion force is not the energy's gradient, so the
    reference need not conserve energy): diamond 512 C at 300 K, 1,000
    steps; the same drift and fluctuation as the reference's."""
    s = B.diamond(4, temp_k=300.0, seed=102)
    n = len(s["z"])
    ctx = M.Context(potentials=M.POT_AIREBO)
    ctx.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    _, et = ctx.run(1000, 0.5)
    r = ref.RefSystem(ref.POT_AIREBO)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    out = r.run(1000, 0.5)
    assert np.max(np.abs(et[:50] - out["etot"][:50])) / n < 1e-9
    sg, fg = drift_stats(et, n, 0.5)
    sr, fr = drift_stats(out["etot"], n, 0.5)
    T = 1000 * 0.5e-3
    assert abs(sg - sr) <= 0.25 * abs(sr) + 10 * fr / T, (sg, sr, fg, fr)
    assert 0.5 < fg / fr < 2.0, (fg, fr)


def test_fp32_mixed_drift_matches_fp64():
    """The mixed path keeps FP64 accumulation and integration: over 10^4
    steps (AIREBO, diamond 512 C with 0.05 A displacements, 600 K) its
    drift and fluctuation equal the FP64 path's statistically."""
    s = B.diamond(4, temp_k=600.0, disp_sigma=0.05, seed=103)
    n = len(s["z"])
    res = {}
    for prec in (M.PREC_FP64, M.PREC_FP32_MIXED):
        ctx = M.Context(potentials=M.POT_AIREBO, precision=prec)
        ctx.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
        _, et = ctx.run(10000, 0.5)
        assert np.all(np.isfinite(et))
        res[prec] = drift_stats(et, n, 0.5)
    (s64, f64), (s32, f32) = res[M.PREC_FP64], res[M.PREC_FP32_MIXED]
    T = 10000 * 0.5e-3
    assert abs(s32 - s64) <= 0.25 * abs(s64) + 10 * f64 / T, (s32, s64, f64)
    assert 0.8 < f32 / f64 < 1.25, (f32, f64)
