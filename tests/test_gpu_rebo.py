"""GPU parity of the REBO / torsion path against the oracle, through the C ABI.

Bars: Verlet pair sets bit-exact once sorted; energy <= 1e-12 relative and
||dF||/||F|| <= 1e-10, or FLOOR_FACTOR times the oracle's own 1-ulp
reproducibility floor when that is larger (see tests/parity.py)."""
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
    "c2h6": lambda: B.c2h6_example(),
    "diamond3_disp": lambda: B.diamond(3, disp_sigma=0.12, seed=21),
    "diamond4_hot": lambda: B.diamond(4, disp_sigma=0.2, seed=22),
    "ach250": lambda: B.amorphous_carbon(250, h_fraction=0.3, seed=23),
    "ac300": lambda: B.amorphous_carbon(300, seed=24),
    "ethane30": lambda: B.ethane_liquid(30, seed=25, min_dist=1.6, jitter=0.4),
}


def _gpu(s, pot, **kw):
    ctx = M.Context(potentials=pot, **kw)
    ctx.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    return ctx


def _oracle(s, pot):
    r = ref.RefSystem(pot)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    return r


@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_rebo_list_pairs_bit_exact(name):
    s = SYSTEMS[name]()
    ctx = _gpu(s, M.POT_REBO)
    r = _oracle(s, ref.POT_REBO)
    assert np.array_equal(ctx.nl_pairs(0), r.nl_pairs(0))


@pytest.mark.parametrize("pot", [M.POT_REBO, M.POT_REBO | M.POT_ETORS])
@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_energy_gradient_parity(name, pot):
    s = SYSTEMS[name]()
    e, et, g = _gpu(s, pot).compute()
    eo, eto, go = _oracle(s, pot).compute()
    floor = oracle_floor(lambda: ref.RefSystem(pot), s)
    assert_parity(e, g, eo, go, floor, label=f"{name}/{pot}")
    assert rel_e(et[0], eto[0]) <= max(1e-12, 4 * floor[0])
    if pot & M.POT_ETORS:
        assert abs(et[2] - eto[1]) <= max(1e-12 * abs(eo), 4 * floor[0] * abs(eo))


@pytest.mark.parametrize("path", [p for p in sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))
                                  if "airebo" not in p and "brenner" not in p])
def test_golden_fixture(path):
    f = np.load(path)
    s = {k: f[k] for k in ("z", "pos", "vel", "box", "pbc", "fixed")}
    ctx = _gpu(s, int(f["potset"]))
    e, et, g = ctx.compute()
    assert_parity(e, g, float(f["e_total"]), f["grad"], tuple(f["floor"]), label=os.path.basename(path))
    assert np.array_equal(ctx.nl_pairs(0), f["pairs0"])


def test_gradient_is_added_into_caller_buffer():
    s = SYSTEMS["ach250"]()
    ctx = _gpu(s, M.POT_REBO)
    e, _, g = ctx.compute()
    base = np.full((len(s["z"]), 3), 0.25)
    import ctypes
    et = np.zeros(4)
    ee = np.zeros(1)
    M._check(M.lib().mdg_compute(ctx.h, M._dp(ee), M._dp(et), M._dp(base)))
    assert np.allclose(base - 0.25, g, rtol=0, atol=1e-12)


def test_cgs_units_match_reference_units():
    s = SYSTEMS["diamond3_disp"]()
    e1, _, g1 = _gpu(s, M.POT_REBO).compute()
    ctx = M.Context(potentials=M.POT_REBO, units=M.UNITS_CGS)
    ctx.set_system(s["z"], s["pos"] * 1e-8, s["vel"] * 1e7, s["box"] * 1e-8, s["pbc"])
    e2, _, g2 = ctx.compute()
    # the two unit systems see inputs that differ in the last bits, so they
    # agree to the oracle's 1-ulp floor, not bitwise
    floor = oracle_floor(lambda: ref.RefSystem(ref.POT_REBO), s)
    assert rel_e(e2 / 1.6021e-12, e1) <= max(1e-12, 4 * floor[0])
    g2a = g2 * 1e-8 / 1.6021e-12
    assert np.linalg.norm(g2a - g1) / np.linalg.norm(g1) <= max(1e-10, 4 * floor[1])


def test_md_run_tracks_oracle():
    s = B.diamond(3, temp_k=600.0, disp_sigma=0.05, seed=26)
    ctx = _gpu(s, M.POT_REBO)
    ep, et = ctx.run(20, 0.5)
    pos, vel, img = ctx.get_state()
    r = _oracle(s, ref.POT_REBO)
    out = r.run(20, 0.5)
    assert np.max(np.abs(ep - out["epot"])) < 1e-8 * len(s["z"])
    d = pos - out["pos"]
    d -= s["box"] * np.round(d / s["box"])
    assert np.abs(d).max() < 1e-9
    assert np.abs(vel - out["vel"]).max() < 1e-9
    assert np.array_equal(img, out["image"])


def test_energy_conservation_short_nve():
    # REBO alone is conservative: total energy stays flat after the start-up
    s = B.diamond(4, temp_k=300.0, seed=27)
    ctx = _gpu(s, M.POT_REBO)
    ep, et = ctx.run(400, 0.5)
    n = len(s["z"])
    assert np.all(np.isfinite(et))
    assert np.ptp(et[40:]) / n < 2e-4


def test_torsion_drift_matches_reference():
    # The reference's torsion force omits the factor 5 of d/dcos of the fifth
    # power (AIREBO_ETors.cxx:110), so REBO + ETors does not conserve energy;
    # the drift must be the reference's own.
    s = B.diamond(3, temp_k=300.0, seed=28)
    pot = M.POT_REBO | M.POT_ETORS
    ep, et = _gpu(s, pot).run(200, 0.5)
    out = _oracle(s, ref.POT_REBO | ref.POT_ETORS).run(200, 0.5)
    n = len(s["z"])
    assert np.ptp(out["etot"]) / n > 2e-4  # the reference itself drifts
    assert np.max(np.abs(et - out["etot"])) / n < 1e-8


def test_bond_capacity_overflow_is_reported():
    s = SYSTEMS["ac300"]()
    ctx = _gpu(s, M.POT_REBO, cap_bonds=1)
    with pytest.raises(M.MdgError) as e:
        ctx.compute()
    assert e.value.code == -4


def test_list_capacity_overflow_is_reported():
    s = SYSTEMS["ac300"]()
    ctx = _gpu(s, M.POT_REBO, cap_rebo_list=2)
    with pytest.raises(M.MdgError) as e:
        ctx.compute()
    assert e.value.code == -3


def test_unknown_element_rejected():
    s = SYSTEMS["c2h6"]()
    z = s["z"].copy()
    z[0] = 29
    ctx = M.Context(potentials=M.POT_REBO)
    with pytest.raises(M.MdgError) as e:
        ctx.set_system(z, s["pos"], s["vel"], s["box"], s["pbc"])
    assert e.value.code == -1


def test_nonfinite_position_reported():
    s = SYSTEMS["diamond3_disp"]()
    pos = s["pos"].copy()
    ctx = _gpu(s, M.POT_REBO)
    ctx.compute()
    pos[5, 0] = 1e-300 + pos[7, 0]
    pos[5, 1:] = pos[7, 1:]  # two atoms on top of each other: r = 0
    ctx.set_state(pos)
    with pytest.raises(M.MdgError):
        ctx.compute()


def test_deterministic_repeat():
    s = SYSTEMS["ach250"]()
    ctx = _gpu(s, M.POT_REBO | M.POT_ETORS)
    e1, _, g1 = ctx.compute()
    e2, _, g2 = ctx.compute()
    ctx2 = _gpu(s, M.POT_REBO | M.POT_ETORS)
    e3, _, g3 = ctx2.compute()
    assert e1 == e2 == e3
    assert np.array_equal(g1, g2) and np.array_equal(g1, g3)


def test_graph_replay_matches_eager_steps():
    # energies=False replays a captured CUDA graph per step; with energies the
    # kernels are launched one by one.  Both must give the same trajectory.
    s = B.diamond(3, temp_k=500.0, disp_sigma=0.05, seed=29)
    a = _gpu(s, M.POT_REBO | M.POT_ETORS)
    a.run(30, 0.5, energies=False)
    a.sync()
    pa, va, ia = a.get_state()
    b = _gpu(s, M.POT_REBO | M.POT_ETORS)
    b.run(30, 0.5, energies=True)
    pb, vb, ib = b.get_state()
    assert np.array_equal(pa, pb) and np.array_equal(va, vb) and np.array_equal(ia, ib)
