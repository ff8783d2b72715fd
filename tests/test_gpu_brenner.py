"""GPU parity of the first-generation Brenner potential (both parameter sets)
against the oracle, through the C ABI; includes the reference's own C2H6
example (examples/C2H6/main.cpp:31-57, Brenner set 1)."""
import glob
import os

import numpy as np
import pytest

import mdtk_b200 as M
from mdtk_b200 import builders as B
from oracle import ref
from parity import assert_parity, oracle_floor

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

SYSTEMS = {
    "c2h6": lambda: B.c2h6_example(),
    "diamond3_disp": lambda: B.diamond(3, disp_sigma=0.15, seed=51),
    "ach250": lambda: B.amorphous_carbon(250, h_fraction=0.3, seed=52),
    "ac300": lambda: B.amorphous_carbon(300, seed=53),
    "ethane30_hot": lambda: B.ethane_liquid(30, seed=54, min_dist=1.5, jitter=0.5),
}


def _gpu(s, bset, pot=M.POT_BRENNER):
    ctx = M.Context(potentials=pot, brenner_set=bset)
    ctx.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    return ctx


def _oracle(s, bset, pot=ref.POT_BRENNER):
    r = ref.RefSystem(pot, bset)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    return r


@pytest.mark.parametrize("bset", [1, 2])
@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_brenner_parity(name, bset):
    s = SYSTEMS[name]()
    e, et, g = _gpu(s, bset).compute()
    eo, eto, go = _oracle(s, bset).compute()
    floor = oracle_floor(lambda: ref.RefSystem(ref.POT_BRENNER, bset), s)
    assert_parity(e, g, eo, go, floor, label=f"{name}/set{bset}")
    assert et[0] == pytest.approx(e, rel=0, abs=0)


def test_brenner_with_torsion_parity():
    s = SYSTEMS["diamond3_disp"]()
    pot = M.POT_BRENNER | M.POT_ETORS
    e, et, g = _gpu(s, 1, pot).compute()
    eo, eto, go = _oracle(s, 1, ref.POT_ETORS | ref.POT_BRENNER).compute()
    floor = oracle_floor(lambda: ref.RefSystem(ref.POT_ETORS | ref.POT_BRENNER, 1), s)
    assert_parity(e, g, eo, go, floor, label="brenner+tors")


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*brenner*.npz"))))
def test_golden_fixture(path):
    f = np.load(path)
    s = {k: f[k] for k in ("z", "pos", "vel", "box", "pbc", "fixed")}
    e, et, g = _gpu(s, 2 if "brenner2" in path else 1).compute()
    assert_parity(e, g, float(f["e_total"]), f["grad"], tuple(f["floor"]), label=os.path.basename(path))


def test_c2h6_example_trajectory():
    # the reference's installation test: 8-atom ethane, Brenner set 1 (here
    # with a fixed 0.2 fs step instead of the adaptive one)
    s = B.c2h6_example()
    ep, et = _gpu(s, 1).run(200, 0.2)
    out = _oracle(s, 1).run(200, 0.2)
    assert np.max(np.abs(ep - out["epot"])) < 1e-8
    assert np.max(np.abs(et - out["etot"])) < 1e-8


def test_brenner_excludes_rebo():
    with pytest.raises(M.MdgError):
        M.Context(potentials=M.POT_BRENNER | M.POT_REBO)
