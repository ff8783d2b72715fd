"""GPU parity of the full AIREBO stack (REBO + LJ + torsion) against the
oracle, through the C ABI: LJ Verlet pair sets bit-exact, per-term energies
and total gradient within the FP64 bars (or the oracle's own 1-ulp floor)."""
import glob
import os

import numpy as np
import pytest

import mdtk_b200 as M
from mdtk_b200 import builders as B
from oracle import ref
from parity import assert_parity, oracle_floor, rel_e

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

SYSTEMS = {
    "ethane30": lambda: B.ethane_liquid(30, seed=31, min_dist=1.6, jitter=0.4),
    "diamond4_disp": lambda: B.diamond(4, disp_sigma=0.1, seed=32),
    "diamond4_hot": lambda: B.diamond(4, disp_sigma=0.25, seed=33),
    "ach300": lambda: B.amorphous_carbon(300, h_fraction=0.25, seed=34),
    "ac300": lambda: B.amorphous_carbon(300, seed=35),
    "ach500_dense": lambda: B.amorphous_carbon(500, h_fraction=0.4, density_g_cm3=1.5, min_sep=1.0, seed=36),
}


def _gpu(s, pot=M.POT_AIREBO, **kw):
    ctx = M.Context(potentials=pot, **kw)
    ctx.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    return ctx


def _oracle(s, pot=ref.POT_AIREBO, lj_cut_mode=0):
    r = ref.RefSystem(pot, 1, lj_cut_mode)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    return r


@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_lj_list_pairs_bit_exact(name):
    s = SYSTEMS[name]()
    ctx = _gpu(s)
    r = _oracle(s)
    assert np.array_equal(ctx.nl_pairs(0), r.nl_pairs(0))
    assert np.array_equal(ctx.nl_pairs(1), r.nl_pairs(1))


@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_airebo_parity(name):
    s = SYSTEMS[name]()
    e, et, g = _gpu(s).compute()
    eo, eto, go = _oracle(s).compute()
    floor = oracle_floor(lambda: ref.RefSystem(ref.POT_AIREBO), s)
    assert_parity(e, g, eo, go, floor, label=name)
    for t in range(3):
        assert abs(et[t] - eto[t]) <= max(1e-12 * abs(eo), 4 * floor[0] * abs(eo)), (t, et, eto)


def test_lj_only_with_rebo_parity():
    s = SYSTEMS["ach300"]()
    pot = M.POT_REBO | M.POT_AIREBO_LJ
    e, et, g = _gpu(s, pot).compute()
    eo, eto, go = _oracle(s, ref.POT_REBO | ref.POT_AIREBO_LJ).compute()
    floor = oracle_floor(lambda: ref.RefSystem(ref.POT_REBO | ref.POT_AIREBO_LJ), s)
    assert_parity(e, g, eo, go, floor, label="rebo+lj")


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*airebo*.npz"))))
def test_golden_fixture(path):
    f = np.load(path)
    s = {k: f[k] for k in ("z", "pos", "vel", "box", "pbc", "fixed")}
    ctx = _gpu(s, int(f["potset"]))
    e, et, g = ctx.compute()
    assert_parity(e, g, float(f["e_total"]), f["grad"], tuple(f["floor"]), label=os.path.basename(path))
    assert np.array_equal(ctx.nl_pairs(1), f["pairs1"])


def test_three_sigma_cutoff_mode():
    s = B.ethane_liquid(120, seed=37, min_dist=1.8)
    ctx = _gpu(s, lj_cut_mode=1, cap_lj_list=2048)
    e, et, g = ctx.compute()
    eo, eto, go = _oracle(s, lj_cut_mode=1).compute()
    assert_parity(e, g, eo, go, label="3 sigma")
    assert np.array_equal(ctx.nl_pairs(1), _oracle(s, lj_cut_mode=1).nl_pairs(1))


def test_md_run_tracks_oracle():
    s = B.ethane_liquid(30, seed=38, temp_k=300.0)
    ctx = _gpu(s)
    ep, et = ctx.run(10, 0.25)
    pos, vel, img = ctx.get_state()
    out = _oracle(s).run(10, 0.25)
    assert np.max(np.abs(ep - out["epot"])) < 1e-9 * len(s["z"])
    d = pos - out["pos"]
    d -= s["box"] * np.round(d / s["box"])
    assert np.abs(d).max() < 1e-9
    assert np.abs(vel - out["vel"]).max() < 1e-9


def test_lj_near_sublist_through_rebuilds():
    # A hot liquid moves its atoms several Angstrom in 300 steps, so the LJ
    # list's 0.5 A near sublist (which the in-range filter reads) is taken
    # again many times and the LJ list itself too; the forces at the end equal
    # the oracle's, whose lists are built afresh at those positions.
    s = B.ethane_liquid(30, seed=39, temp_k=2000.0)
    ctx = _gpu(s)
    ctx.run(300, 0.25, energies=False)
    pos, vel, _ = ctx.get_state()
    moved = pos - s["pos"]
    moved -= s["box"] * np.round(moved / s["box"])
    assert np.sqrt((moved ** 2).sum(1)).max() > 2.0
    e, et, g = ctx.compute()
    s2 = dict(s, pos=pos, vel=vel)
    eo, eto, go = _oracle(s2).compute()
    floor = oracle_floor(lambda: ref.RefSystem(ref.POT_AIREBO), s2)
    assert_parity(e, g, eo, go, floor, label="hot ethane30 after 300 steps")


def test_deterministic_repeat():
    s = SYSTEMS["diamond4_hot"]()
    ctx = _gpu(s)
    e1, _, g1 = ctx.compute()
    e2, _, g2 = _gpu(s).compute()
    assert e1 == e2
    assert np.array_equal(g1, g2)


def test_record_capacity_overflow_is_reported():
    s = SYSTEMS["diamond4_hot"]()
    ctx = _gpu(s, cap_special=1)
    with pytest.raises(M.MdgError) as e:
        ctx.compute()
    assert e.value.code == -8


def test_dependent_launch_matches_ordinary_launch():
    """Programmatic dependent launch changes when blocks are scheduled, never
    what they compute: the same trajectory bit for bit, list rebuilds and the
    three streams included, through the graph and through host steps."""
    s = B.ethane_liquid(400, seed=40, temp_k=1500.0)
    out = []
    for pdl in (True, False):
        c = _gpu(s, task_mode=2)  # the launch configuration is still tuned (overlap)
        c.set_dependent_launch(pdl)
        _, et = c.run(120, 0.5)
        c.run(60, 0.5, energies=False)
        c.sync()
        p, v, img = c.get_state()
        out.append((et, p, v, img, c.compute()))
        assert c.task_mode()[0] == 2
    (ea, pa, va, ia, (ga, ta, fa)), (eb, pb, vb, ib, (gb, tb, fb)) = out
    assert np.array_equal(ea, eb) and np.array_equal(pa, pb) and np.array_equal(va, vb)
    assert np.array_equal(ia, ib) and ga == gb and np.array_equal(ta, tb) and np.array_equal(fa, fb)


def test_graph_replay_matches_eager_steps():
    s = B.ethane_liquid(30, seed=39, temp_k=300.0)
    a = _gpu(s)
    a.run(25, 0.25, energies=False)
    a.sync()
    pa, va, _ = a.get_state()
    b = _gpu(s)
    b.run(25, 0.25, energies=True)
    pb, vb, _ = b.get_state()
    assert np.array_equal(pa, pb) and np.array_equal(va, vb)
