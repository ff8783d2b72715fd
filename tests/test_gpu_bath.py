"""The SimLoop step's thermal bath and adaptive time step on the device,
against the reference's own SimLoop with the same settings (oracle harness:
ref_set_bath / ref_set_adaptive): per-step total energies and time steps of
the first steps (before trajectories decorrelate), geometry and per-atom
flags, per-system state of a batched context, and the argument checks that
mirror the geometries' REQUIREs."""
import numpy as np
import pytest

import mdtk_b200 as M
from mdtk_b200 import builders as B
from oracle import ref

pytestmark = pytest.mark.gpu


def _pair(s, pot, mpot, bath=None, adaptive=None, flags=None, dt=0.5, nsteps=60):
    """Runs the device and the reference with the same bath / dt settings;
    returns (device etot, reference etot, device dts, reference dts)."""
    c = M.Context(potentials=mpot, task_mode=1)
    c.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    r = ref.RefSystem(pot)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    if bath is not None:
        geom, T0, gamma_s, params = bath
        c.set_thermal_bath(geom, T0, gamma_s * 1e-15, params, flags)
        r.set_bath(geom, T0, gamma_s, params, flags)
    dts_dev = None
    if adaptive is not None:
        timeaccel, dt0 = adaptive
        c.set_adaptive_dt(True, timeaccel, dt0)
        r.set_adaptive(True, timeaccel, dt0)
        dts_dev = []
        et = []
        for _ in range(nsteps):
            dts_dev.append(c.get_time()[1][0])
            et.append(c.run(1, dt)[1][0])
        et = np.array(et)
    else:
        _, et = c.run(nsteps, dt)
    out = r.run(nsteps, dt)
    return et, out["etot"], None if dts_dev is None else np.array(dts_dev), r.last_run_dts(nsteps)


def test_universe_bath_heats_like_the_reference():
    s = B.diamond(3, temp_k=300.0, seed=121)
    n = len(s["z"])
    et, eo, _, _ = _pair(s, ref.POT_REBO, M.POT_REBO, bath=(M.TB_UNIVERSE, 1000.0, 1e13, None), nsteps=80)
    assert eo[-1] - eo[0] > 1e-4 * n  # the bath heats the lattice
    assert np.max(np.abs(et[:40] - eo[:40])) / n < 1e-9
    assert abs(et[-1] - eo[-1]) / n < 1e-6


def test_box_bath_with_adaptive_dt_on_an_impact():
    s = B.impact(3, n_target=900)
    zmin = s["pos"][:, 2].min()
    params = [1e6, 3.0, zmin + 1.0]  # no top zone; a 3 A lateral boundary zone above the bottom layer
    et, eo, dd, dr = _pair(s, ref.POT_AIREBO, M.POT_AIREBO, bath=(M.TB_BOX, 300.0, 1e13, params),
                           adaptive=(1.0, 0.2), nsteps=60)
    n = len(s["z"])
    assert dr[0] == pytest.approx(0.2) and np.any(np.abs(np.diff(dr)) > 0)  # the step adapts
    assert np.allclose(dd[:30], dr[:30], rtol=1e-10, atol=0)
    assert np.max(np.abs(et[:30] - eo[:30])) / n < 1e-9


def test_sphere_bath_and_flags():
    s = B.c2h6_example()
    s = dict(s)
    s["vel"] = B.thermal_velocities(s["z"], 600.0, np.random.default_rng(7))
    centre = s["pos"].mean(axis=0)
    flags = np.ones(len(s["z"]), np.uint8)
    flags[::2] = 0
    params = [centre[0], centre[1], centre[2], 1.2, -1e3]
    et, eo, _, _ = _pair(s, ref.POT_REBO, M.POT_REBO, bath=(M.TB_SPHERE, 50.0, 1e14, params), flags=flags,
                         dt=0.25, nsteps=60)
    assert np.max(np.abs(et - eo)) < 1e-9 * max(1.0, np.abs(eo).max())


def test_batched_adaptive_dt_per_system():
    systems = [B.impact(k, n_target=900) for k in (4, 5, 6)]
    bx = M.Context(potentials=M.POT_AIREBO, task_mode=1)
    bx.set_batch(systems)
    bx.set_adaptive_dt(True, 1.0, 0.2)
    singles = []
    for s in systems:
        c = M.Context(potentials=M.POT_AIREBO, task_mode=1)
        c.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
        c.set_adaptive_dt(True, 1.0, 0.2)
        singles.append(c)
    for step in range(20):
        bx.run(1, 0.5, energies=False)
        for c in singles:
            c.run(1, 0.5, energies=False)
        tb, db = bx.get_time()
        for k, c in enumerate(singles):
            t1, d1 = c.get_time()
            assert db[k] == pytest.approx(d1[0], rel=1e-12) and tb[k] == pytest.approx(t1[0], rel=1e-12)
    assert len(set(np.round(db, 12))) > 1  # systems keep their own steps


def test_bath_argument_checks():
    s = B.diamond(3, seed=122)
    c = M.Context(potentials=M.POT_REBO)
    c.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    with pytest.raises(M.MdgError):
        c.set_thermal_bath(M.TB_SPHERE, 300.0, 0.01, [0, 0, 0, 5, 0])  # periodic box
    with pytest.raises(M.MdgError):
        c.set_thermal_bath(7, 300.0, 0.01)
    with pytest.raises(M.MdgError):
        c.set_adaptive_dt(True, -1.0, 0.5)
    c.set_thermal_bath(M.TB_UNIVERSE, 300.0, 0.01)
    with pytest.raises(M.MdgError):  # the adjoint differentiates plain fixed-dt steps
        c.adjoint_forward(2, 0.5, 1)
