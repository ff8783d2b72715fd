"""Oracle parity at the benchmark configurations' own sizes.

C1: REBO and Brenner (sets 1 and 2) carbon, diamond-cubic 6x6x6 unit cells
(1,728 atoms, a = 3.567 A), periodic, seeded Maxwell-Boltzmann velocities at
300 K with zero net momentum, dt 0.5 fs.  C2: the AIREBO ethane liquid of the
throughput benchmark, 5,461 C2H6 (43,688 atoms) at 0.55 g/cm^3 and 300 K.

Bars: Verlet pair sets bit-exact; energy <= 1e-12 relative and ||dF||/||F||
<= 1e-10, or FLOOR_FACTOR times the oracle's own 1-ulp reproducibility floor
where that is larger (tests/parity.py; the achieved errors are recorded).
Trajectories: the diamond at 300 K is not chaotic over 1,000 steps (two
oracle runs whose inputs differ by one ulp stay within 1e-13 A), so the GPU
run must track the oracle's step by step; over 10^4 steps the comparison is
statistical (drift slope and fluctuation)."""
import numpy as np
import pytest

import mdtk_b200 as M
from mdtk_b200 import builders as B
from oracle import ref
from parity import assert_parity, oracle_floor, rel_e
from test_gpu_nve import drift_stats

pytestmark = pytest.mark.gpu

C1_SEED = 1
C2_SEED = 1  # the throughput benchmark's single-GPU system


def c1():
    return B.diamond(6, temp_k=300.0, seed=C1_SEED)


# (product potential flags, oracle potential flags, Brenner parameter set)
C1_POTS = {
    "rebo": (M.POT_REBO, ref.POT_REBO, 1),
    "brenner1": (M.POT_BRENNER, ref.POT_BRENNER, 1),
    "brenner2": (M.POT_BRENNER, ref.POT_BRENNER, 2),
}


def _gpu(s, pot, bset=1, **kw):
    ctx = M.Context(potentials=pot, brenner_set=bset, **kw)
    ctx.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    return ctx


def _oracle(s, pot, bset=1):
    r = ref.RefSystem(pot, bset)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    return r


def test_c1_system_is_the_configuration():
    s = c1()
    n = len(s["z"])
    assert n == 1728 and np.allclose(s["box"], 6 * 3.567)
    assert B.temperature(s["z"], s["vel"]) == pytest.approx(300.0, rel=1e-12)
    p = (B.masses(s["z"])[:, None] * s["vel"]).sum(0)
    assert np.abs(p).max() < 1e-10


@pytest.mark.parametrize("name", sorted(C1_POTS))
def test_c1_list_pairs_bit_exact(name):
    pot, rpot, bset = C1_POTS[name]
    s = c1()
    assert np.array_equal(_gpu(s, pot, bset).nl_pairs(0), _oracle(s, rpot, bset).nl_pairs(0))


@pytest.mark.parametrize("name", sorted(C1_POTS))
def test_c1_energy_force_parity(name):
    """C1 starts on the perfect lattice, where every force vanishes by
    symmetry (the oracle's are ~1e-13 eV/A of rounding), so a relative force
    error means nothing there: step 0 is held to the energy bar and an
    absolute force bar, and the forces are compared relatively at the state
    the oracle's own SimLoop reaches after 200 steps (thermal displacements,
    forces of order 1 eV/A)."""
    pot, rpot, bset = C1_POTS[name]
    s = c1()
    e, et, g = _gpu(s, pot, bset).compute()
    eo, eto, go = _oracle(s, rpot, bset).compute()
    floor = oracle_floor(lambda: ref.RefSystem(rpot, bset), s)
    assert rel_e(e, eo) <= max(1e-12, 4 * floor[0]), (e, eo)
    assert np.abs(g - go).max() < 1e-10, np.abs(g - go).max()
    out = _oracle(s, rpot, bset).run(200, 0.5)
    s2 = dict(s, pos=out["pos"], vel=out["vel"])
    e, et, g = _gpu(s2, pot, bset).compute()
    eo, eto, go = _oracle(s2, rpot, bset).compute()
    assert np.sqrt((go ** 2).mean()) > 0.1
    floor = oracle_floor(lambda: ref.RefSystem(rpot, bset), s2)
    assert_parity(e, g, eo, go, floor, label=f"C1 diamond 1728 after 200 steps / {name}")


@pytest.mark.parametrize("name", ["rebo", "brenner1"])
def test_c1_1000_steps_track_oracle(name):
    """1,000 velocity-Verlet steps of C1 (dt 0.5 fs): per-step energies,
    final positions, velocities and image counters against the reference's
    own SimLoop."""
    pot, rpot, bset = C1_POTS[name]
    s = c1()
    n = len(s["z"])
    ctx = _gpu(s, pot, bset)
    ep, et = ctx.run(1000, 0.5)
    pos, vel, img = ctx.get_state()
    out = _oracle(s, rpot, bset).run(1000, 0.5)
    de = np.abs(et - out["etot"]).max() / n
    d = pos - out["pos"]
    d -= s["box"] * np.round(d / s["box"])
    dv = np.abs(vel - out["vel"]).max()
    print(f"C1/{name} 1000 steps: max |dE_total|/atom {de:.2e} eV, max |dx| {np.abs(d).max():.2e} A, "
          f"max |dv| {dv:.2e} A/fs")
    assert de < 1e-11
    assert np.abs(ep - out["epot"]).max() / n < 1e-11
    assert np.abs(d).max() < 1e-10
    assert dv < 1e-11
    assert np.array_equal(img, out["image"])


def test_c1_nve_drift_over_1e4_steps():
    """10^4 REBO steps of C1 on both: the first 1,000 steps' total energies
    agree step by step, and the drift slope and fluctuation over the whole
    run agree statistically."""
    s = c1()
    n = len(s["z"])
    _, et = _gpu(s, M.POT_REBO).run(10000, 0.5)
    out = _oracle(s, ref.POT_REBO).run(10000, 0.5)
    assert np.abs(et[:1000] - out["etot"][:1000]).max() / n < 1e-11
    sg, fg = drift_stats(et, n, 0.5)
    sr, fr = drift_stats(out["etot"], n, 0.5)
    T = 10000 * 0.5e-3  # ps
    print(f"C1 drift: GPU {sg:.3e} oracle {sr:.3e} eV/atom/ps; fluctuation GPU {fg:.4e} oracle {fr:.4e} eV/atom")
    assert abs(sr) < 10 * fr / T and abs(sg) < 10 * fr / T, (sg, sr, fr)
    assert abs(sg - sr) < 10 * fr / T, (sg, sr, fr)
    assert 0.8 < fg / fr < 1.25, (fg, fr)


@pytest.fixture(scope="module")
def c2_pair():
    from bench import build_system
    s = build_system(C2_SEED)
    assert len(s["z"]) == 43688
    ctx = _gpu(s, M.POT_AIREBO)
    r = _oracle(s, ref.POT_AIREBO)
    return s, ctx, r


def test_c2_list_pairs_bit_exact(c2_pair):
    s, ctx, r = c2_pair
    for lst in (0, 1):
        assert np.array_equal(ctx.nl_pairs(lst), r.nl_pairs(lst)), lst


def test_c2_energy_terms_and_forces(c2_pair):
    s, ctx, r = c2_pair
    e, et, g = ctx.compute()
    eo, eto, go = r.compute()
    floor = oracle_floor(lambda: ref.RefSystem(ref.POT_AIREBO), s, samples=2)
    assert_parity(e, g, eo, go, floor, label="C2 ethane 43688 / AIREBO")
    for t, name in enumerate(("REBO", "LJ", "torsion")):
        assert abs(et[t] - eto[t]) <= max(1e-12 * abs(eo), 4 * floor[0] * abs(eo)), (name, et, eto)
    assert rel_e(et[0], eto[0]) <= max(1e-12, 4 * floor[0])
