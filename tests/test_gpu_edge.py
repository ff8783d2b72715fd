"""Edge cases and full-size properties, through the C ABI.

* empty and ragged inputs are rejected;
* a single atom (no pair, no bond) has no energy and moves in free flight;
* an isolated C-C pair (an LJ pair that needs b*_ij, no bonds) matches the
  reference;
* coincident atoms are reported as an error status (the reference stops in
  the REQUIRE of CosTheta);
* at the configurations' full sizes (the 43,688-atom ethane liquid, the
  512,000-atom diamond) the size-independent properties hold: zero net force
  (every term is a sum of pair-antisymmetric pieces), translation invariance
  of the energy, and the FP32-mixed force error bound."""
import numpy as np
import pytest

import mdtk_b200 as M
from mdtk_b200 import builders as B
from oracle import ref

pytestmark = pytest.mark.gpu


def _ctx(s, pot=M.POT_AIREBO, **kw):
    c = M.Context(potentials=pot, **kw)
    c.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    return c


def _system(z, pos, vel=None, box=(20.0, 20.0, 20.0), pbc=(1, 1, 1)):
    z = np.asarray(z, np.int32)
    pos = np.asarray(pos, float).reshape(-1, 3)
    return {"z": z, "pos": pos, "vel": np.zeros_like(pos) if vel is None else np.asarray(vel, float),
            "box": np.asarray(box, float), "pbc": np.asarray(pbc, np.int32), "fixed": np.zeros(len(z), np.uint8)}


def test_empty_and_ragged_inputs_rejected():
    c = M.Context(potentials=M.POT_AIREBO)
    with pytest.raises(M.MdgError) as e:
        c.set_system(np.zeros(0, np.int32), np.zeros((0, 3)), np.zeros((0, 3)), (20, 20, 20), (1, 1, 1))
    assert e.value.code == -1
    with pytest.raises(M.MdgError):
        c.compute()  # nothing loaded
    with pytest.raises(Exception):
        c.set_system(np.full(4, 6, np.int32), np.zeros(10), None, (20, 20, 20), (1, 1, 1))


def test_single_atom_free_flight():
    s = _system([6], [[5.0, 5.0, 5.0]], [[0.01, -0.02, 0.005]])
    c = _ctx(s)
    e, et, g = c.compute()
    assert e == 0.0 and np.all(g == 0.0)
    ep, etot = c.run(10, 0.5)
    pos, vel, img = c.get_state()
    assert np.all(ep == 0.0)
    assert np.allclose(pos[0], s["pos"][0] + s["vel"][0] * 5.0, rtol=0, atol=1e-13)
    assert np.array_equal(vel, s["vel"])


def test_isolated_pair_matches_reference():
    # 3.5 A: inside the LJ cutoff, below 2^(1/6) sigma_CC (S(t_r) != 0, so b*_ij is evaluated)
    s = _system([6, 6], [[8.0, 10.0, 10.0], [11.5, 10.0, 10.0]])
    e, et, g = _ctx(s).compute()
    r = ref.RefSystem(ref.POT_AIREBO)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"])
    eo, eto, go = r.compute()
    assert et[0] == 0.0 and et[2] == 0.0 and et[1] != 0.0  # LJ only
    assert abs(e - eo) <= 1e-12 * abs(eo)
    assert np.linalg.norm(g - go) <= 1e-10 * np.linalg.norm(go)


def test_coincident_atoms_reported():
    # The reference stops in the REQUIRE of CosTheta (FGeneral.hpp:147) (the
    # oracle process does not survive it, so it is not called here); this
    # build reports an error status.
    s = B.diamond(3, seed=111)
    s["pos"][1] = s["pos"][0]
    with pytest.raises(M.MdgError) as e:
        _ctx(s, M.POT_REBO).compute()
    assert e.value.code in (-5, -7)  # cos(theta) out of range / non-finite


def _net_force_ok(g):
    return np.linalg.norm(g.sum(axis=0)) <= 1e-11 * np.sqrt(len(g)) * np.sqrt((g ** 2).sum(axis=1).mean())


def test_full_size_ethane_invariants():
    s = B.ethane_liquid(5461, density_g_cm3=0.55, temp_k=300.0, seed=1)
    c = _ctx(s)
    e, _, g = c.compute()
    assert _net_force_ok(g)
    shifted = dict(s)
    shifted["pos"] = np.mod(s["pos"] + np.array([1.2345, -2.5, 0.77]), s["box"])
    e2, _, g2 = _ctx(shifted).compute()
    assert abs(e2 - e) <= 1e-12 * abs(e)
    assert np.linalg.norm(g2 - g) <= 1e-10 * np.linalg.norm(g)
    _, _, g32 = _ctx(s, precision=M.PREC_FP32_MIXED).compute()
    assert np.linalg.norm(g32 - g) <= 1e-5 * np.linalg.norm(g)


def test_full_size_diamond_512000():
    s = B.diamond(40, temp_k=600.0, disp_sigma=0.05, seed=7)
    assert len(s["z"]) == 512000
    c = _ctx(s)
    e, et, g = c.compute()
    assert np.isfinite(e) and _net_force_ok(g)
    _, _, g32 = _ctx(s, precision=M.PREC_FP32_MIXED).compute()
    assert np.linalg.norm(g32 - g) <= 1e-5 * np.linalg.norm(g)


def test_step_host_multi_step_calls_equal_device_runs():
    """mdg_step_host with k steps per call from a host-held state gives the
    state and energies of k device-resident steps, bit for bit."""
    s = B.ethane_liquid(60, seed=91, min_dist=1.6, jitter=0.4)
    a = M.Context(potentials=M.POT_AIREBO, task_mode=2)
    a.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    b = M.Context(potentials=M.POT_AIREBO, task_mode=2)
    b.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    pos, vel, _ = b.get_state()
    ep_h, et_h = [], []
    for _ in range(3):
        ep, et = b.step_host(10, 0.25, pos, vel)
        ep_h.append(ep)
        et_h.append(et)
    ep_d, et_d = a.run(30, 0.25)
    pa, va, _ = a.get_state()
    assert np.array_equal(np.concatenate(ep_h), ep_d) and np.array_equal(np.concatenate(et_h), et_d)
    assert np.array_equal(pos, pa) and np.array_equal(vel, va)


def test_nl_update_reports_rebuilds():
    s = B.ethane_liquid(60, seed=92, min_dist=1.6, jitter=0.4)
    c = M.Context(potentials=M.POT_AIREBO)
    c.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    assert list(c.nl_update(force=True)[:2]) == [1, 1]
    assert list(c.nl_update()[:2]) == [0, 0]       # nothing moved since
    pos, vel, _ = c.get_state()
    c.set_state(pos + 1.3, vel)                   # every atom 2.25 A: past both triggers
    assert list(c.nl_update()[:2]) == [1, 1]


def test_launch_floor_diagnostic():
    g, c = M.launch_floor(0, 24)
    assert 0.0 < g < 1e4 and 0.0 < c < 1e4
