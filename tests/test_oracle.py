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
