"""The oracle (reference MDTK compiled from its own sources) against the
known answers available for this path: the diamond cohesive energies
measured when the path was surveyed, the reference's own spline knot tables
(AIREBO/cubici.cxx), and the committed golden fixtures."""
import glob
import os

import numpy as np
import pytest

from mdtk_b200 import builders as B
from oracle import ref

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle not built (make -C oracle)")

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("pot,anchor", [
    (ref.POT_REBO, -7.3699259815),
    (ref.POT_BRENNER, -7.3461346746),
    (ref.POT_AIREBO, -7.4213317044),
])
def test_diamond_cohesive_energy(pot, anchor):
    s = B.diamond(4)
    r = ref.RefSystem(pot)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"])
    e, _, g = r.compute()
    assert abs(e / len(s["z"]) - anchor) < 5e-11
    assert np.abs(g).max() < 1e-9  # perfect lattice: zero net force on every atom


def test_spline_knots_reproduce_tables():
    # FuncG knots (AIREBO/cubici.cxx:52-56, 73-77, 94-97)
    g_c1 = [(-1.0, -0.010000), (-2.0 / 3.0, 0.028207), (-0.5, 0.052804), (-1.0 / 3.0, 0.097321), (1.0, 1.0)]
    g_h = [(-1.0, 11.235700), (-5.0 / 6.0, 12.595300), (-0.5, 16.811100), (1.0, 19.991800)]
    for fn, knots in ((0, g_c1), (2, g_h)):
        x = np.array([[k[0], 0, 0] for k in knots])
        assert np.allclose(ref.spline_eval(fn, x), [k[1] for k in knots], atol=1e-10, rtol=0)
    # P_CC / P_CH knot values (AIREBO/cubici.cxx:130-135, 217-225); non-integer
    # neighbours of a knot approach the knot value continuously
    for fn, knots in ((10, {(2, 0): -0.0005, (3, 0): 0.016125, (1, 1): -0.01096, (0, 2): -0.027603}),
                      (13, {(1, 0): 0.209337, (2, 1): -0.298905, (0, 3): -0.307585})):
        for (h, c), v in knots.items():
            near = np.array([[h + 1e-9, c + 1e-9, 0]])
            assert abs(ref.spline_eval(fn, np.array([[h, c, 0]]))[0] - v) < 1e-10
            assert abs(ref.spline_eval(fn, near)[0] - v) < 1e-7
    # pi_rc_CC and Tij (AIREBO/cubici.cxx:420-458, 529-531), including the
    # FCCfillUp continuation in Nconj and the empty k = 15 cells
    cases = [(20, (1, 1, 1), 0.0525), (20, (2, 2, 8), 0.003309), (20, (0, 0, 9), 0.004959),
             (20, (1, 0, 12), 0.004959), (32, (2, 2, 1), -0.03514), (32, (2, 2, 7), -0.004048),
             (20, (2, 2, 15), 0.0), (20, (4, 1, 2), 0.0)]
    for fn, (i, j, k), v in cases:
        assert abs(ref.spline_eval(fn, np.array([[i, j, k]], float))[0] - v) < 1e-10


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))))
def test_oracle_matches_golden(path):
    f = np.load(path)
    pot = int(f["potset"])
    r = ref.RefSystem(pot, 2 if "brenner2" in path else 1)
    r.set_atoms(f["z"], f["pos"], f["vel"], f["box"], f["pbc"], f["fixed"])
    e, et, g = r.compute()
    assert e == pytest.approx(float(f["e_total"]), rel=1e-14, abs=1e-12)
    assert np.allclose(g, f["grad"], rtol=1e-12, atol=1e-12)
    for i in range(r.npot):
        assert np.array_equal(r.nl_pairs(i), f[f"pairs{i}"])


def test_oracle_run_conserves_energy():
    s = B.diamond(3, temp_k=300.0, seed=3)
    r = ref.RefSystem(ref.POT_REBO)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"])
    out = r.run(40, 0.5)
    et = out["etot"]
    assert np.all(np.isfinite(et))
    assert np.ptp(et) / len(s["z"]) < 2e-4  # eV/atom


# ---------------------------------------------------------------- restatement
RS_CASES = {
    "c2h6": lambda: B.c2h6_example(),
    "diamond3_disp": lambda: B.diamond(3, disp_sigma=0.15, seed=61),
    "ach250": lambda: B.amorphous_carbon(250, h_fraction=0.3, seed=62),
    "ethane30": lambda: B.ethane_liquid(30, seed=63, min_dist=1.6, jitter=0.4),
}
RS_POTS = {"rebo": (ref.POT_REBO, 0), "tors": (ref.POT_REBO | ref.POT_ETORS, None),
           "brenner": (ref.POT_BRENNER, 3), "airebo": (ref.POT_AIREBO, None)}


def _oracle_eg(s, pot):
    r = ref.RefSystem(pot)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    return r.compute()


@pytest.mark.skipif(not ref.restatement_available(), reason="restatement not built")
@pytest.mark.parametrize("pot", sorted(RS_POTS))
@pytest.mark.parametrize("name", sorted(RS_CASES))
def test_restatement_energy_matches_reference(name, pot):
    s = RS_CASES[name]()
    if pot == "airebo" and s["pbc"][0] and s["box"][0] < 11.1:
        pytest.skip("box below twice the LJ cutoff")
    bits = RS_POTS[pot][0]
    e = ref.rs_energy(s, bits).sum()
    eo, _, _ = _oracle_eg(s, bits)
    # the reference's spline coefficients carry ~1e-11 of LU noise; the
    # restatement evaluates the exact Hermite interpolants
    assert abs(e - eo) <= 5e-11 * max(abs(eo), 1.0) + 1e-10


@pytest.mark.skipif(not ref.restatement_available(), reason="restatement not built")
@pytest.mark.parametrize("pot", ["rebo", "brenner"])
@pytest.mark.parametrize("name", sorted(RS_CASES))
def test_reference_adjoint_is_exact_gradient(name, pot):
    # forward-mode derivatives of the restated energy equal the reference's
    # hand-written gradient for REBO and Brenner
    s = RS_CASES[name]()
    bits = RS_POTS[pot][0]
    _, _, go = _oracle_eg(s, bits)
    rng = np.random.default_rng(7)
    for _ in range(2):
        d = rng.normal(size=s["pos"].shape)
        dd = ref.rs_energy_dir(s, bits, d).sum()
        assert abs(dd - np.sum(go * d)) <= 1e-9 * np.linalg.norm(go) * np.linalg.norm(d) + 1e-12


@pytest.mark.skipif(not ref.restatement_available(), reason="restatement not built")
def test_reference_torsion_force_is_not_the_energy_gradient():
    # AIREBO_ETors.cxx:110 differentiates ((1+cos w)/2)^5 without the factor 5;
    # the restatement's exact derivative exposes the difference
    s = RS_CASES["diamond3_disp"]()
    bits = ref.POT_REBO | ref.POT_ETORS
    _, _, go = _oracle_eg(s, bits)
    d = np.random.default_rng(8).normal(size=s["pos"].shape)
    dd = ref.rs_energy_dir(s, bits, d).sum()
    assert abs(dd - np.sum(go * d)) > 1e-6 * np.linalg.norm(go) * np.linalg.norm(d)


def test_parameter_override_acts_on_the_reference():
    """ref_set_param changes the reference's own members: REBO's V_R is
    linear in A_CC and the LJ energy of pure carbon is linear in eps_CC, so
    equal steps of the parameter give equal energy steps; sigma_CC moves the
    LJ energy; restoring a parameter restores the energy bitwise."""
    s = B.amorphous_carbon(300, seed=91)
    r = ref.RefSystem(ref.POT_AIREBO)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"])
    e0, et0, _ = r.compute()
    for pid, base, term in ((2, 10953.544, 0), (0, 0.00284, 1)):
        es = []
        for k in range(3):
            r.set_param(pid, base * (1 + 0.01 * k))
            es.append(r.compute()[1][term])
        d1, d2 = es[1] - es[0], es[2] - es[1]
        assert d1 != 0.0 and abs(d1 - d2) <= 1e-9 * abs(d1), (pid, d1, d2)
        r.set_param(pid, base)
    e1, et1, _ = r.compute()
    assert e1 == e0
    r.set_param(1, 3.41)
    assert r.compute()[1][1] != et0[1]


@pytest.mark.parametrize("zip_mode,ext", [(0, ""), (1, ".gz"), (2, ".xz")])
def test_reference_state_files_round_trip(tmp_path, zip_mode, ext):
    """The harness drives the reference's own SimLoopSaver: a state written
    after 10 steps (box bath, fixed atoms, tags) loads back unchanged, in
    each of yaatk's compressions, and the loaded run continues where the
    first would have gone."""
    s = B.impact(3, n_target=900)
    zmin = s["pos"][:, 2].min()
    r = ref.RefSystem(ref.POT_REBO)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    tags = np.zeros(len(s["z"]), np.uint8)
    tags[-13:] = 1 << 2  # ATOMTAG_PROJECTILE
    r.set_tags(tags)
    r.set_bath(2, 300.0, 1e13, [zmin - 1.0, 3.0, zmin + 1.0])
    r.run(10, 0.5)
    ref.set_zip(zip_mode)
    try:
        r.write_state(str(tmp_path / "md0000000010"))
    finally:
        ref.set_zip(0)
    assert os.path.exists(str(tmp_path / "md0000000010.r") + ext)
    assert os.path.exists(str(tmp_path / "md0000000010.thermal_bath.box") + ext)
    r2 = ref.RefSystem(ref.POT_REBO)
    assert r2.load_state(str(tmp_path / "md0000000010"), 10) == 127
    a, b = r.atoms(), r2.atoms()
    for k in ("pos", "vel", "acc", "image", "fixed", "tb_apply", "tags", "z"):
        assert np.array_equal(a[k], b[k]), k
    la, lb = r.loop(), r2.loop()
    for k in ("time", "dt", "dt_prev", "iteration", "tb_geom", "tb_T0", "tb_gamma", "e0", "e_cur", "e_bath", "T"):
        assert la[k] == lb[k], k
    assert np.array_equal(la["tb_params"], lb["tb_params"]) and np.array_equal(la["box"], lb["box"])


def test_reference_xva_layout(tmp_path):
    """SimLoop::saveToStreamXVA's text layout as the device writer restates
    it: velocity scale (%g), distance scale, atom count, three lines per atom
    (V/scale and coords/Ao with two decimals, image counters), the Check
    record, simTime, dt, iteration, run time (%.10e)."""
    s = B.diamond(3, temp_k=300.0, seed=9)
    r = ref.RefSystem(ref.POT_REBO)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    r.run(4, 0.5)
    r.write_xva(str(tmp_path / "f.xva"))
    lines = open(tmp_path / "f.xva").read().splitlines()
    n = len(s["z"])
    v = r.atoms()["vel"] * 1e-8 / 1e-15  # cm/s
    scale = 10.0 ** (np.ceil(np.log10(np.abs(v).sum() / (3.0 * n))) - 2)
    assert lines[0] == "%g" % scale and lines[1] == "1e-08" and lines[2] == str(n)
    assert len(lines) == 3 + 3 * n + 11
    a = r.atoms()
    for i in (0, n // 2, n - 1):
        assert lines[3 + 3 * i] == "%.2f %.2f %.2f" % tuple(a["vel"][i] * 1e7 / scale)
        assert lines[4 + 3 * i] == "%.2f %.2f %.2f" % tuple(a["pos"][i] * 1e-8 / 1e-8)
        assert lines[5 + 3 * i] == "%d %d %d" % tuple(a["image"][i])
    tail = lines[3 + 3 * n:]
    assert tail[0] == "1" and tail[2] == "1" and tail[1].endswith(" ") and tail[9] == "4"
    assert all(len(t.split("e")) == 2 for t in tail[3:9] + [tail[10]])


@pytest.mark.skipif(not os.path.exists(ref.SHIM_PATH), reason="shim library not built")
def test_gpu_classes_load_and_fail_loudly_without_a_device():
    """The drop-in GPU classes compiled against the reference headers load
    beside the oracle; without a CUDA device their construction reports the
    C ABI's error through the reference's own exception type instead of
    falling back to anything."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    ref.install_gpu_shim()
    with pytest.raises(RuntimeError, match="no CUDA device"):
        ref.RefSystem(ref.POT_AIREBO | ref.POT_GPU)
