"""Checkpoint and trajectory files through the C ABI, against the reference's
own SimLoopSaver and SimLoop::saveToStreamXVA run by the oracle harness on
the same state:

* the state files after the same steps: integer, flag and layout files
  byte-identical, floating-point records within the trajectories' agreement;
* the XVA text frame line by line;
* interchange both ways: the reference loads our files (plain, .gz, .xz) and
  we load the reference's, then continue the run (thermal bath, fixed atoms,
  tags) in step with the reference continuing from the same files;
* SimLoop::executeMain's output schedule: the same state and XVA files at
  the same iterations as the reference writing its own;
* per-system output of a batched context, argument and I/O errors."""
import bz2
import gzip
import lzma
import os

import numpy as np
import pytest

import mdtk_b200 as M
from mdtk_b200 import builders as B
from oracle import ref

pytestmark = pytest.mark.gpu

EXACT = [".z", ".pbc_rect", ".pbc_rect.count", ".pbc_rect.enabled", ".indices", ".tag.thermal_bath_applicable",
         ".tag.fixed", ".tag.target", ".tag.projectile", ".tag.substrate", ".tag.monomer", ".tag.cluster",
         ".tag.fullerene"]


def read(path):
    """A file as yaatk::Stream finds it: plain, .xz, .bz2, .gz."""
    for ext, op in (("", open), (".xz", lzma.open), (".bz2", bz2.open), (".gz", gzip.open)):
        if os.path.exists(path + ext):
            with op(path + ext, "rb") as f:
                return f.read()
    raise FileNotFoundError(path)


def close(a, b, rtol):
    a, b = np.asarray(a, float), np.asarray(b, float)
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() <= rtol * scale


def compare_state(ours, theirs, rtol=1e-7, adaptive=False):
    """rtol: the agreement of the two trajectories' coordinates, velocities
    and accelerations (relative to each array's largest value); the
    colliding cluster atoms of an impact amplify rounding differences to
    ~1e-9 within 20 steps."""
    for attr in EXACT:
        assert read(ours + attr) == read(theirs + attr), attr
    for attr in (".r", ".v", ".a"):
        a = np.frombuffer(read(ours + attr), np.float64)
        b = np.frombuffer(read(theirs + attr), np.float64)
        assert a.shape == b.shape and close(a, b, rtol), attr
    ta = np.frombuffer(read(ours + ".time"), np.float64)
    tb = np.frombuffer(read(theirs + ".time"), np.float64)
    # simTime and dt_prev; dt only with adaptive steps: the reference adapts
    # dt after every step (SimLoop.cxx:405-416) and the harness's fixed-dt
    # runs set it back before the next one, so after a fixed-dt run its dt is
    # the adapted value while ours is the fixed step
    assert ta[0] == pytest.approx(tb[0], rel=1e-14) and ta[3] == tb[3]
    if adaptive:
        assert ta[2] == pytest.approx(tb[2], rel=1e-9)
    ca, cb = read(ours + ".check"), read(theirs + ".check")
    assert len(ca) == len(cb) == 58 and ca[0] == cb[0] and ca[25] == cb[25]
    fa = np.frombuffer(ca[1:25], np.float64)
    fb = np.frombuffer(cb[1:25], np.float64)
    ea = np.frombuffer(ca[26:58], np.float64)
    eb = np.frombuffer(cb[26:58], np.float64)
    fscale = np.abs(np.frombuffer(read(theirs + ".a"), np.float64)).max() * 12 * 1.6605655e-24
    assert np.abs(fa - fb).max() <= 1e-9 * fscale * len(read(theirs + ".z"))  # net force: sums to ~0
    assert np.allclose(ea[[0, 1]], eb[[0, 1]], rtol=1e-10, atol=0)  # E0, E
    assert ea[3] == pytest.approx(eb[3], rel=1e-8)  # T
    assert abs(ea[2] - eb[2]) <= 1e-9 * max(abs(eb[1]), 1e-300)  # energy from the bath


def _unsign_zero(line):
    # atoms at rest carry velocities of rounding size whose sign the two
    # implementations need not share: "-0.00" and "0.00" are the same value
    return " ".join("0.00" if w == "-0.00" else w for w in line.split(" "))


def _atom_lines(lines, n, box):
    """(velocity/scale, unwrapped coordinate/Ao) per atom from an XVA body:
    an atom on a periodic boundary may sit at 0 in one frame and at L with
    one image less in the other."""
    v = np.array([lines[3 + 3 * i].split() for i in range(n)], float)
    x = np.array([lines[4 + 3 * i].split() for i in range(n)], float)
    im = np.array([lines[5 + 3 * i].split() for i in range(n)], float)
    return v, x + im * np.asarray(box, float)


def compare_xva(ours, theirs, box=(0.0, 0.0, 0.0), adaptive=False):
    a = [_unsign_zero(x) for x in read(ours).decode().splitlines()]
    b = [_unsign_zero(x) for x in read(theirs).decode().splitlines()]
    assert len(a) == len(b)
    n = int(b[2])
    assert a[:3] == b[:3]
    body_a, body_b = a[3:3 + 3 * n], b[3:3 + 3 * n]
    same = sum(x == y for x, y in zip(body_a, body_b))
    assert same >= 0.99 * len(body_b)  # a last-digit flip needs a value within rounding of an edge
    va, xa = _atom_lines(a, n, box)
    vb, xb = _atom_lines(b, n, box)
    assert np.abs(va - vb).max() <= 0.0100001 and np.abs(xa - xb).max() <= 0.0100001 + 1e-9
    tail_a, tail_b = a[3 + 3 * n:], b[3 + 3 * n:]
    assert tail_a[0] == tail_b[0] == "1" and tail_a[2] == tail_b[2] == "1"
    fa, fb = np.array(tail_a[1].split(), float), np.array(tail_b[1].split(), float)
    assert np.abs(fa - fb).max() <= 1e-6 * max(np.abs(fb).max(), 1e-3)
    for k, tol in ((3, 1e-10), (4, 1e-10), (6, 1e-8)):  # E0, E, T
        assert float(tail_a[k]) == pytest.approx(float(tail_b[k]), rel=tol)
    # simTime and iteration; dt only with adaptive steps (see compare_state)
    assert float(tail_a[7]) == pytest.approx(float(tail_b[7]), rel=1e-9 if adaptive else 1e-14)
    assert tail_a[9] == tail_b[9]
    if adaptive:
        assert float(tail_a[8]) == pytest.approx(float(tail_b[8]), rel=1e-9)


def pair(s, pot=M.POT_AIREBO, rpot=ref.POT_AIREBO, tags=None):
    c = M.Context(potentials=pot, task_mode=1)
    c.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    r = ref.RefSystem(rpot)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    if tags is not None:
        c.set_atom_tags(tags)
        r.set_tags(tags)
    return c, r


def tagged_impact():
    s = B.impact(3, n_target=900)
    s = dict(s)
    n = len(s["z"])
    zmin = s["pos"][:, 2].min()
    s["fixed"] = (s["pos"][:, 2] < zmin + 0.5).astype(np.uint8)
    s["vel"] = np.where(s["fixed"][:, None] == 1, 0.0, s["vel"])
    tags = np.full(n, M.TAG_TARGET, np.uint8)
    tags[-5:] = M.TAG_PROJECTILE | M.TAG_CLUSTER
    return s, tags


def test_state_and_xva_after_steps_match_reference(tmp_path):
    s, tags = tagged_impact()
    c, r = pair(s, tags=tags)
    nsteps = 20
    c.set_time_final(0.5 * (nsteps - 0.5))
    c.run(nsteps, 0.5)
    r.run(nsteps, 0.5)
    ref.set_zip(0)
    r.write_state(str(tmp_path / "ref"))
    c.write_state(str(tmp_path / "dev"))
    compare_state(str(tmp_path / "dev"), str(tmp_path / "ref"))
    r.write_xva(str(tmp_path / "ref.xva"))
    c.write_xva(str(tmp_path / "dev.xva"))
    compare_xva(str(tmp_path / "dev.xva"), str(tmp_path / "ref.xva"), box=s["box"] * np.asarray(s["pbc"]))


def test_fresh_state_is_byte_identical(tmp_path):
    """Before any step both hold the loaded values and the Check record's
    constructor defaults: every file is byte-identical."""
    s = B.diamond(3, temp_k=300.0, seed=131)
    c, r = pair(s, M.POT_REBO, ref.POT_REBO)
    ref.set_zip(0)
    r.write_state(str(tmp_path / "ref"))
    c.write_state(str(tmp_path / "dev"))
    # (.indices: the reference numbers its atoms when a run prepares them,
    # AtomsContainer.cxx:107-123; before that every index is 0)
    for attr in [a for a in EXACT if a != ".indices"] + [".r", ".v", ".a", ".check"]:
        assert read(str(tmp_path / "dev") + attr) == read(str(tmp_path / "ref") + attr), attr
    r.write_xva(str(tmp_path / "ref.xva"))
    c.write_xva(str(tmp_path / "dev.xva"))
    a = read(str(tmp_path / "dev.xva")).decode().splitlines()
    b = read(str(tmp_path / "ref.xva")).decode().splitlines()
    assert a[:-4] == b[:-4] and a[-2] == b[-2]  # all but simTime/dt (dt set by a run) and the run time


@pytest.mark.parametrize("zip_mode", [M.ZIP_NONE, M.ZIP_GZIP, M.ZIP_XZ])
def test_reference_loads_our_state(tmp_path, zip_mode):
    s, tags = tagged_impact()
    c = M.Context(potentials=M.POT_AIREBO, task_mode=1)
    c.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    c.set_atom_tags(tags)
    zmin = s["pos"][:, 2].min()
    c.set_thermal_bath(M.TB_BOX, 300.0, 1e13 * 1e-15, [zmin - 1.0, 3.0, zmin + 1.0])
    c.run(15, 0.5)
    c.write_state(str(tmp_path / "md0000000015"), zip=zip_mode)
    ext = {M.ZIP_NONE: "", M.ZIP_GZIP: ".gz", M.ZIP_XZ: ".xz"}[zip_mode]
    assert os.path.exists(str(tmp_path / "md0000000015.r") + ext)
    r = ref.RefSystem(ref.POT_AIREBO)
    got = r.load_state(str(tmp_path / "md0000000015"), 15)
    assert got == 127
    a = r.atoms()
    pos, vel, img = c.get_state()
    assert np.allclose(a["pos"], pos, rtol=1e-14, atol=0)
    assert np.allclose(a["vel"], vel, rtol=1e-14, atol=1e-300)
    assert np.array_equal(a["image"], img)
    assert np.array_equal(a["fixed"], s["fixed"]) and np.array_equal(a["tags"], tags)
    assert np.array_equal(a["z"], s["z"])
    lp = r.loop()
    assert lp["iteration"] == 15 and lp["time"] == pytest.approx(7.5, rel=1e-14) and lp["dt"] == 0.5
    assert lp["tb_geom"] == M.TB_BOX and lp["tb_T0"] == 300.0 and lp["tb_gamma"] == pytest.approx(1e13, rel=1e-14)
    assert np.allclose(lp["tb_params"][:3], [zmin - 1.0, 3.0, zmin + 1.0], rtol=1e-14)


def test_load_reference_state_and_continue(tmp_path):
    """The reference writes its state after 30 steps with a box bath; we load
    it and both continue from the same files for 30 more steps."""
    s, tags = tagged_impact()
    zmin = s["pos"][:, 2].min()
    params = [zmin - 1.0, 3.0, zmin + 1.0]
    r = ref.RefSystem(ref.POT_AIREBO)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    r.set_tags(tags)
    r.set_bath(M.TB_BOX, 300.0, 1e13, params)
    r.run(30, 0.5)
    ref.set_zip(1)
    r.write_state(str(tmp_path / "md0000000030"))
    ref.set_zip(0)
    c = M.Context(potentials=M.POT_AIREBO, task_mode=1)
    got = c.load_state(str(tmp_path / "md0000000030"), 30)
    assert got == 127 and c.n == len(s["z"]) and c.iteration() == 30
    a = r.atoms()
    pos, vel, img = c.get_state()
    assert np.allclose(pos, a["pos"], rtol=1e-14, atol=0) and np.allclose(vel, a["vel"], rtol=1e-14, atol=1e-300)
    assert np.array_equal(img, a["image"]) and np.array_equal(c.get_atom_tags(), tags)
    r2 = ref.RefSystem(ref.POT_AIREBO)
    r2.load_state(str(tmp_path / "md0000000030"), 30)
    _, et = c.run(30, 0.5)
    out = r2.run(30, 0.5)
    n = len(s["z"])
    assert np.max(np.abs(et - out["etot"])) / n < 1e-9
    assert c.iteration() == 60 and r2.loop()["iteration"] == 60
    c.write_state(str(tmp_path / "dev60"))
    r2.write_state(str(tmp_path / "ref60"))
    compare_state(str(tmp_path / "dev60"), str(tmp_path / "ref60"))


def test_output_schedule_matches_simloop(tmp_path):
    s, tags = tagged_impact()
    c, r = pair(s, tags=tags)
    ddir, rdir = tmp_path / "dev", tmp_path / "ref"
    os.makedirs(rdir)
    ref.set_zip(0)
    r.set_output(str(rdir), 5, 2.0)
    r.run(12, 0.5)
    c.set_time_final(0.5 * 11.5)
    c.set_output(str(ddir), 5, 2.0)
    c.run(12, 0.5)
    c.flush_output()
    c.write_state(str(ddir / "md0000000012"))  # executeMain's closing writestate (SimLoop.cxx:460-464)
    dev_files = sorted(os.listdir(ddir))
    ref_files = sorted(os.listdir(rdir))
    assert dev_files == ref_files
    ids = sorted({f.split(".")[0] for f in ref_files})
    assert ids == ["md0000000005", "md0000000010", "md0000000012", "mde0000000000", "mde0000000004",
                   "mde0000000008"]
    for i in ids:
        if i.startswith("mde"):
            compare_xva(str(ddir / (i + ".xva")), str(rdir / (i + ".xva")), box=s["box"] * np.asarray(s["pbc"]))
        else:
            compare_state(str(ddir / i), str(rdir / i))


def test_adaptive_dt_output_schedule(tmp_path):
    s = B.impact(4, n_target=900)
    c, r = pair(s)
    c.set_adaptive_dt(True, 1.0, 0.2)
    r.set_adaptive(True, 1.0, 0.2)
    ddir, rdir = tmp_path / "dev", tmp_path / "ref"
    os.makedirs(rdir)
    ref.set_zip(0)
    r.set_output(str(rdir), 1000000, 1.7)
    r.run(40, 0.5)
    c.set_output(str(ddir), 0, 1.7)
    c.run(40, 0.5)
    c.flush_output()
    dev_x = sorted(f for f in os.listdir(ddir) if f.endswith(".xva"))
    ref_x = sorted(f for f in os.listdir(rdir) if f.endswith(".xva"))
    assert dev_x == ref_x and len(ref_x) > 3
    for f in ref_x:
        compare_xva(str(ddir / f), str(rdir / f), box=s["box"] * np.asarray(s["pbc"]), adaptive=True)


def test_batched_output_per_system(tmp_path):
    systems = [B.impact(k, n_target=900) for k in (5, 6)]
    bx = M.Context(potentials=M.POT_AIREBO, task_mode=1)
    bx.set_batch(systems)
    bx.set_output(str(tmp_path / "b"), 4, 1.0)
    bx.run(9, 0.5)
    bx.flush_output()
    for k, s in enumerate(systems):
        c = M.Context(potentials=M.POT_AIREBO, task_mode=1)
        c.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
        d = tmp_path / f"s{k}"
        c.set_output(str(d), 4, 1.0)
        c.run(9, 0.5)
        c.flush_output()
        sd = tmp_path / "b" / f"sys{k:05d}"
        assert sorted(os.listdir(sd)) == sorted(os.listdir(d))
        for f in os.listdir(d):
            if f.endswith(".xva"):
                compare_xva(str(sd / f), str(d / f), box=s["box"] * np.asarray(s["pbc"]))
        compare_state(str(sd / "md0000000008"), str(d / "md0000000008"), rtol=1e-8)


def test_round_trip_and_errors(tmp_path):
    s = B.diamond(3, temp_k=300.0, seed=132)
    c = M.Context(potentials=M.POT_REBO)
    c.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    c.run(5, 0.5)
    for zmode in (M.ZIP_GZIP, M.ZIP_XZ):
        c.write_state(str(tmp_path / "x"), zip=zmode)
        d = M.Context(potentials=M.POT_REBO)
        assert d.load_state(str(tmp_path / "x"), 5) == 127
        p0, v0, i0 = c.get_state()
        p1, v1, i1 = d.get_state()
        assert np.allclose(p1, p0, rtol=1e-15, atol=0) and np.allclose(v1, v0, rtol=1e-15, atol=1e-300)
        assert np.array_equal(i1, i0)
        # a restart continues like the original run
        _, e0 = c.run(10, 0.5)
        _, e1 = d.run(10, 0.5)
        assert np.max(np.abs(e0 - e1)) / len(s["z"]) < 1e-10
    with pytest.raises(M.MdgError) as e:
        M.Context(potentials=M.POT_REBO).load_state(str(tmp_path / "missing"))
    assert e.value.code == -1
    with pytest.raises(M.MdgError) as e:
        c.write_state(str(tmp_path / "no_such_dir" / "x"))
    assert e.value.code == -12
    with pytest.raises(M.MdgError):
        c.write_state(str(tmp_path / "y"), zip=7)
    with pytest.raises(M.MdgError):
        c.write_state(str(tmp_path / "y"), sys=1)
