"""The metal and ion potentials (FBZL, FLJ, Ackland; MDG_POT_METAL) against
the reference's own classes run by the oracle harness in the same potential
order as applications/common.h:36-77:

* Cu, Ag, Au crystals and a Cu-Au alloy (Ackland: pair knots, density, the
  geometric-mean density between unlike metals, embedding);
* hydrocarbons on a metal surface with pairs in every FLJ regime (ZBL below
  1.2 A, the joining cubic, Lennard-Jones, the 5.0-5.5 A switch) beside full
  AIREBO;
* Ar and Xe ions among hydrocarbon and metal atoms (FBZL);
* energies per potential, total energy and gradient; MD steps; a batched
  context; the flag checks."""
import numpy as np
import pytest

import mdtk_b200 as M
from mdtk_b200 import builders as B
from oracle import ref

pytestmark = pytest.mark.gpu

POT = M.POT_AIREBO | M.POT_METAL
RPOT = ref.POT_AIREBO | ref.POT_METAL


def both(s, pot=POT, rpot=RPOT, **kw):
    c = M.Context(potentials=pot, **kw)
    c.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    r = ref.RefSystem(rpot)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    return c, r


def check(s, pot=POT, rpot=RPOT, rtol_e=1e-12, rtol_g=1e-10):
    c, r = both(s, pot, rpot)
    e, et, g = c.compute()
    eo, eto, go = r.compute()
    assert abs(e - eo) <= rtol_e * max(abs(eo), 1.0), (e, eo)
    assert np.linalg.norm(g - go) <= rtol_g * np.linalg.norm(go)
    # per potential: the reference's order FBZL, FLJ, REBO, AIREBO LJ, ETors, Ackland
    if rpot == RPOT:
        assert et[3] == pytest.approx(eto[0] + eto[1] + eto[5], rel=1e-12, abs=1e-12)
        assert et[0] == pytest.approx(eto[2], rel=1e-12, abs=1e-12)
        assert et[1] == pytest.approx(eto[3], rel=1e-12, abs=1e-12)
    return c, r, e


@pytest.mark.parametrize("z", [29, 47, 79])
def test_metal_crystal(z):
    s = B.fcc(z, 4, temp_k=300.0, disp_sigma=0.08, seed=z)  # periods above 2 x 5.5 A (checkMIC)
    c, r, e = check(s)
    assert e < 0


def test_cu_au_alloy_and_close_pairs():
    s = B.fcc(29, 3, disp_sigma=0.05, seed=5, a=3.8)
    rng = np.random.default_rng(6)
    s["z"][rng.random(len(s["z"])) < 0.4] = 79
    s["z"][rng.random(len(s["z"])) < 0.1] = 47
    # a pair in the ZBL range and one on the joining cubic (1.0-1.4 A)
    s["pos"][1] = s["pos"][0] + [0.9, 0.0, 0.0]
    s["pos"][5] = s["pos"][4] + [0.0, 1.2, 0.0]
    s["pos"] = np.mod(s["pos"], s["box"])
    check(s)


def hydrocarbon_on_metal(zm=29, seed=11):
    slab = B.fcc(zm, 4, 4, 3, pbc=(1, 1, 0), disp_sigma=0.03, seed=seed)
    top = slab["pos"][:, 2].max()
    rng = np.random.default_rng(seed)
    mol = B.c2h6_example()
    atoms_z, atoms_p = [], []
    for k, h in enumerate((2.6, 3.4, 4.8, 5.3)):  # LJ, LJ, inside the switch, beyond it
        off = np.array([2.0 + 3.5 * k, 2.0 + 1.7 * k, top + h]) - mol["pos"].mean(axis=0)
        atoms_z.append(mol["z"])
        atoms_p.append(mol["pos"] + off + rng.normal(scale=0.02, size=mol["pos"].shape))
    # close pairs: an H at 1.5 A (joining cubic) and a C at 1.0 A (ZBL) above metal atoms
    hi = np.argsort(slab["pos"][:, 2])[-2:]
    atoms_z.append(np.array([1, 6], np.int32))
    atoms_p.append(slab["pos"][hi] + np.array([[0, 0, 1.5], [0, 0, 1.0]]))
    return B.add_atoms(slab, np.concatenate(atoms_z), np.concatenate(atoms_p))


@pytest.mark.parametrize("zm", [29, 79, 47])
def test_hydrocarbon_on_metal(zm):
    """Cu and Au interact with H and C through FLJ; Ag has no hydrocarbon
    pair potential in the reference (no interaction)."""
    s = hydrocarbon_on_metal(zm)
    check(s)


def test_ions():
    s = hydrocarbon_on_metal(29, seed=12)
    top = s["pos"][:, 2].max()
    ions = np.array([[3.0, 3.0, top + 1.5], [7.0, 5.0, top + 2.2], [9.0, 9.0, top + 6.5], [9.0, 9.0, top + 11.7]])
    s = B.add_atoms(s, [18, 54, 18, 18], ions)  # the last two 5.2 A apart: inside the switch
    check(s)


def test_md_with_metal_and_ion_matches_reference():
    s = hydrocarbon_on_metal(29, seed=13)
    top = s["pos"][:, 2].max()
    s = B.add_atoms(s, [18], [[5.0, 5.0, top + 4.0]], vel=[[0.0, 0.0, -0.05]])
    s["vel"][:-1] = B.thermal_velocities(s["z"][:-1], 300.0, np.random.default_rng(3))
    c, r = both(s, task_mode=1)
    _, et = c.run(40, 0.25)
    out = r.run(40, 0.25)
    assert np.max(np.abs(et - out["etot"])) / len(s["z"]) < 1e-9


def test_batched_metal_systems_match_single():
    systems = [B.fcc(29, 4, disp_sigma=0.05, seed=21), hydrocarbon_on_metal(79, seed=22)]
    bx = M.Context(potentials=POT, task_mode=1)
    bx.set_batch(systems)
    eb = bx.batch_energies()
    _, eta = bx.batch_run(10, 0.25)
    for k, s in enumerate(systems):
        c = M.Context(potentials=POT, task_mode=1)
        c.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
        e, et, _ = c.compute()
        assert eb[k, :3].sum() == pytest.approx(e, rel=1e-12)
        _, et1 = c.run(10, 0.25)
        assert np.allclose(eta[:, k], et1, rtol=1e-10, atol=1e-10)


def test_flag_checks():
    s = B.fcc(29, 4, seed=1)
    c = M.Context(potentials=M.POT_AIREBO)
    with pytest.raises(M.MdgError):
        c.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    c = M.Context(potentials=POT)
    c.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    with pytest.raises(M.MdgError):
        c.adjoint_forward(2, 0.5, 1)


def test_metal_state_files_both_ways(tmp_path):
    """Metal and ion atoms in SimLoopSaver's files: ElementID of Cu, Au, Ar in
    ".z"; the reference loads our state and we load the reference's."""
    s = hydrocarbon_on_metal(79, seed=31)
    top = s["pos"][:, 2].max()
    s = B.add_atoms(s, [18], [[4.0, 4.0, top + 4.0]])
    c, r = both(s, task_mode=1)
    c.run(5, 0.25)
    r.run(5, 0.25)
    c.write_state(str(tmp_path / "dev"), zip=M.ZIP_GZIP)
    r2 = ref.RefSystem(RPOT)
    assert r2.load_state(str(tmp_path / "dev"), 5) == 127
    a = r2.atoms()
    pos, vel, img = c.get_state()
    assert np.array_equal(a["z"], s["z"]) and np.allclose(a["pos"], pos, rtol=1e-14, atol=0)
    ref.set_zip(0)
    r.write_state(str(tmp_path / "ref"))
    d = M.Context(potentials=POT, task_mode=1)
    assert d.load_state(str(tmp_path / "ref"), 5) == 127
    e1, _, g1 = d.compute()
    e0, _, g0 = r.compute()
    assert abs(e1 - e0) <= 1e-12 * abs(e0) and np.linalg.norm(g1 - g0) <= 1e-10 * np.linalg.norm(g0)


def test_fp32_mixed_with_metal():
    """The mixed mode keeps the metal and ion kernels in FP64; its error stays
    that of the hydrocarbon terms."""
    s = hydrocarbon_on_metal(29, seed=32)
    c64 = M.Context(potentials=POT)
    c64.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    c32 = M.Context(potentials=POT, precision=M.PREC_FP32_MIXED)
    c32.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    e64, t64, g64 = c64.compute()
    e32, t32, g32 = c32.compute()
    assert t32[3] == t64[3]  # metal and ion energies identical
    assert np.linalg.norm(g32 - g64) <= 1e-5 * np.linalg.norm(g64)
