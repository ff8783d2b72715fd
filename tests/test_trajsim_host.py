"""Host logic of the impact-sequence driver (no GPU): its reader of the
SimLoopSaver files against states the reference writes itself (oracle
harness), in each of yaatk's compressions, and SimLoopSaver::removeIterations'
choice of which iteration files to keep."""
import os

import numpy as np
import pytest

import mdtk_b200 as M
from mdtk_b200 import builders as B
from mdtk_b200 import trajsim as T
from oracle import ref


@pytest.mark.parametrize("zip_mode", [0, 1, 2])
def test_read_state_of_reference_files(tmp_path, zip_mode):
    s = B.impact(3, n_target=900)
    zmin = s["pos"][:, 2].min()
    r = ref.RefSystem(ref.POT_AIREBO)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    tags = np.zeros(len(s["z"]), np.uint8)
    tags[-13:] = M.TAG_PROJECTILE | M.TAG_CLUSTER
    r.set_tags(tags)
    flags = np.ones(len(s["z"]), np.uint8)
    flags[:10] = 0
    r.set_bath(M.TB_BOX, 300.0, 1e13, [zmin - 1.0, 3.0, zmin + 1.0], flags)
    r.set_time(0.0, 25.0, 0.2)
    r.run(5, 0.5)
    ref.set_zip(zip_mode)
    try:
        r.write_state(str(tmp_path / "st"))
    finally:
        ref.set_zip(0)
    st = T.read_state(str(tmp_path / "st"))
    a, lp = r.atoms(), r.loop()
    assert np.array_equal(st["z"], a["z"]) and np.array_equal(st["image"], a["image"])
    assert np.allclose(st["pos"], a["pos"], rtol=1e-15, atol=0)
    assert np.allclose(st["vel"], a["vel"], rtol=1e-15, atol=1e-300)
    assert np.array_equal(st["fixed"], a["fixed"]) and np.array_equal(st["tags"], tags)
    assert np.array_equal(st["tb_apply"], flags)
    assert list(st["pbc"]) == [1, 1, 0] and np.allclose(st["box"][:2], s["box"][:2], rtol=1e-15)
    assert st["bath"]["geom"] == M.TB_BOX and st["bath"]["T0"] == 300.0 and st["bath"]["gamma"] == 1e13
    assert np.allclose(st["bath"]["params"][:3], lp["tb_params"][:3], rtol=1e-15)
    assert st["time"] == pytest.approx(lp["time"], rel=1e-14) and st["dt"] == pytest.approx(lp["dt"], rel=1e-14)


def test_remove_iterations(tmp_path):
    for it in (0, 1000, 2000, 2417):
        for attr in (".r", ".z", ".time.xz"):
            open(tmp_path / ("md%010d%s" % (it, attr)), "w").close()
    open(tmp_path / "mde0000000000.xva", "w").close()
    open(tmp_path / "snapshots.conf", "w").close()
    T.remove_iterations(str(tmp_path), keep_first=True, keep_last=True)
    names = sorted(os.listdir(tmp_path))
    assert {n[:12] for n in names if n.startswith("md0")} == {"md0000000000", "md0000002417"}
    assert "mde0000000000.xva" in names and "snapshots.conf" in names
    T.remove_iterations(str(tmp_path), keep_first=False, keep_last=True)
    assert {n[:12] for n in os.listdir(tmp_path) if n.startswith("md0")} == {"md0000002417"}
