"""mdtrajsim's impact-sequence mode: the batched driver (mdtk_b200.trajsim)
against the reference's own impact loop and runTraj with CustomSimLoop's
snapshots (oracle harness, applications/mdtrajsim/main.cpp:113-345), from the
same base state and ionpos.bin: the same files in each impact directory, the
same final iteration, state files, XVA frames and snapshot lists within the
trajectories' agreement; and SnapshotList's capture itself."""
import os

import numpy as np
import pytest

import mdtk_b200 as M
from mdtk_b200 import builders as B
from mdtk_b200 import trajsim as T
from oracle import ref

from test_gpu_io import compare_state, compare_xva, read

pytestmark = pytest.mark.gpu


def base_system(layers=2, nx=5, ny=3):
    s = B.graphite_slab(layers, nx, ny, temp_k=0.0, seed=1)
    n = len(s["z"])
    top = s["pos"][:, 2].max()
    z = np.concatenate([s["z"], [6]]).astype(np.int32)
    pos = np.concatenate([s["pos"], [[s["box"][0] / 2, s["box"][1] / 2, top + 3.0]]])
    vel = np.concatenate([s["vel"], [[0.0, 0.0, -0.04]]])  # ~100 eV C projectile
    fixed = np.concatenate([s["fixed"], [0]]).astype(np.uint8)
    tags = np.zeros(n + 1, np.uint8)
    tags[:n] = M.TAG_TARGET
    tags[-1] = M.TAG_PROJECTILE
    return z, pos, vel, s["box"], fixed, tags


def read_snapshots(path):
    b = read(path)
    o = 0

    def take(dt, k):
        nonlocal o
        a = np.frombuffer(b, dt, k, o)
        o += a.nbytes
        return a

    nsel = int(take(np.uint32, 1)[0])
    idx = take(np.uint32, nsel)
    nshots = int(take(np.uint32, 1)[0])
    times, recs = [], []
    for _ in range(nshots):
        times.append(float(take(np.float64, 1)[0]))
        size = int(take(np.uint32, 1)[0])
        assert size == nsel
        raw = take(np.uint8, 36 * size)
        recs.append((np.frombuffer(raw.tobytes(), np.int32).reshape(size, 9)[:, :3],
                     np.frombuffer(raw.tobytes(), np.float32).reshape(size, 9)[:, 3:]))
    assert o == len(b)
    return idx, np.array(times), recs


def test_impact_sequence_matches_mdtrajsim(tmp_path):
    z, pos, vel, box, fixed, tags = base_system()
    r = ref.RefSystem(ref.POT_AIREBO)
    r.set_atoms(z, pos, vel, box, (1, 1, 0), fixed)
    r.set_tags(tags)
    r.set_time(0.0, 40.0, 0.2)
    ref.set_zip(0)
    r.write_state(str(tmp_path / "base"))
    xy = np.array([[2.0e-8, 3.0e-8], [5.0e-8, 1.0e-8], [9.5e-8, 11.0e-8]])
    xy.tofile(str(tmp_path / "ionpos.bin"))
    os.makedirs(tmp_path / "ref")
    ref.impact_sequence(ref.POT_AIREBO, str(tmp_path / "base"), str(tmp_path / "ionpos.bin"), str(tmp_path / "ref"))
    ran = T.impact_sequence(str(tmp_path / "base"), str(tmp_path / "ionpos.bin"), str(tmp_path / "dev"),
                            task_mode=1)
    assert ran == [0, 1, 2]
    for k in range(3):
        dd, rd = tmp_path / "dev" / ("%08d" % k), tmp_path / "ref" / ("%08d" % k)
        files = sorted(os.listdir(rd))
        assert sorted(os.listdir(dd)) == files
        assert "completed.ok" in files and "snapshots.conf" in files
        assert read(str(dd / "ionpos_used.bin")) == read(str(rd / "ionpos_used.bin"))
        assert read(str(dd / "ionpos_used.txt")) == read(str(rd / "ionpos_used.txt"))
        final = [f[:-2] for f in files if f.endswith(".r")]
        assert len(final) == 1
        compare_state(str(dd / final[0]), str(rd / final[0]), adaptive=True)
        for f in files:
            if f.endswith(".xva"):
                compare_xva(str(dd / f), str(rd / f), box=np.asarray(box) * [1, 1, 0], adaptive=True)
        ia, ta, ra = read_snapshots(str(dd / "snapshots.conf"))
        ib, tb, rb = read_snapshots(str(rd / "snapshots.conf"))
        assert np.array_equal(ia, ib) and list(ia) == [len(z) - 1]
        assert len(ta) == len(tb) >= 4
        assert np.allclose(ta, tb, rtol=1e-9, atol=0)
        for (pa, fa), (pb, fb) in zip(ra, rb):
            assert np.array_equal(pa, pb)
            assert np.allclose(fa[:, :3], fb[:, :3], rtol=1e-6, atol=0)  # coordinates (cm)
            assert np.allclose(fa[:, 3:], fb[:, 3:], rtol=1e-5, atol=1e-3)  # velocities (cm/s)
    # a second call finds every impact completed (isAlreadyFinished)
    assert T.impact_sequence(str(tmp_path / "base"), str(tmp_path / "ionpos.bin"), str(tmp_path / "dev")) == []


def test_impact_sequence_matches_the_mdtrajsim_application(tmp_path):
    """The unmodified mdtrajsim application (applications/mdtrajsim/main.cpp
    built from its own sources, `mdtrajsim base -i 0`) and the batched driver
    with the application's potential set and compression."""
    import subprocess
    app = os.path.join(os.path.dirname(ref.LIB_PATH), "mdtrajsim")
    z, pos, vel, box, fixed, tags = base_system()
    r = ref.RefSystem(ref.POT_AIREBO | ref.POT_METAL)
    r.set_atoms(z, pos, vel, box, (1, 1, 0), fixed)
    r.set_tags(tags)
    r.set_time(0.0, 30.0, 0.2)
    ref.set_zip(0)
    os.makedirs(tmp_path / "ref")
    r.write_state(str(tmp_path / "ref" / "base"))
    xy = np.array([[2.0e-8, 3.0e-8], [9.5e-8, 11.0e-8]])
    xy.tofile(str(tmp_path / "ref" / "ionpos.bin"))
    p = subprocess.run([app, "base", "-i", "0"], cwd=str(tmp_path / "ref"), capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    T.impact_sequence(str(tmp_path / "ref" / "base"), str(tmp_path / "ref" / "ionpos.bin"), str(tmp_path / "dev"),
                      zip=M.ZIP_XZ, task_mode=1)
    for k in range(2):
        dd, rd = tmp_path / "dev" / ("%08d" % k), tmp_path / "ref" / ("%08d" % k)
        files = sorted(f for f in os.listdir(rd) if f not in ("stdout.txt", "stderr.txt"))
        assert sorted(os.listdir(dd)) == files and all(f.endswith(".xz") for f in files)
        assert read(str(dd / "ionpos_used.txt")) == read(str(rd / "ionpos_used.txt"))
        final = [f[:-5] for f in files if f.endswith(".r.xz")]
        compare_state(str(dd / final[0]), str(rd / final[0]), adaptive=True)
        compare_xva(str(dd / "mde0000000000.xva"), str(rd / "mde0000000000.xva"), box=np.asarray(box) * [1, 1, 0],
                    adaptive=True)
        ia, ta, ra = read_snapshots(str(dd / "snapshots.conf"))
        ib, tb, rb = read_snapshots(str(rd / "snapshots.conf"))
        assert np.array_equal(ia, ib) and len(ta) == len(tb) and np.allclose(ta, tb, rtol=1e-9, atol=0)


def test_snapshot_capture_and_reload(tmp_path):
    """The device SnapshotList: snapshots at CustomSimLoop's times, the same
    list through the API and the file, text form, reload, capacity."""
    z, pos, vel, box, fixed, tags = base_system()
    c = M.Context(potentials=M.POT_AIREBO, task_mode=1)
    c.set_system(z, pos, vel, box, (1, 1, 0), fixed)
    c.set_atom_tags(tags)
    with pytest.raises(M.MdgError):
        c.snapshots_enable(True)  # snapshots follow simTime: adaptive dt first
    c.set_adaptive_dt(True, 1.0, 0.2)
    c.snapshots_enable(True, 64)
    c.set_time_final(35.0)
    c.set_stop_at_time_final(True)
    steps, done = c.run_until_final()
    assert done and steps > 0
    t, _ = c.get_time()
    assert t[0] >= 35.0
    sn = c.snapshots()
    assert list(sn["indices"]) == [len(z) - 1]
    # one snapshot at t = 0 and one per crossed multiple of 10 fs
    assert sn["time"][0] == 0.0 and len(sn["time"]) == 1 + int(sn["time"][-1] // 10.0)
    assert np.all(np.diff(np.floor(sn["time"] / 10.0 + 1e-9)) == 1)
    c.snapshots_write(str(tmp_path / "snapshots.conf"))
    idx, times, recs = read_snapshots(str(tmp_path / "snapshots.conf"))
    assert np.allclose(times * 1e15, sn["time"], rtol=1e-12)
    assert np.array_equal(recs[-1][1][:, :3], sn["pos"][-1])
    c.snapshots_write(str(tmp_path / "snap.txt"), text=True)
    lines = open(tmp_path / "snap.txt").read().splitlines()
    assert lines[0].split() == [str(len(z) - 1)] and len(lines) == 1 + 4 * len(times)
    # a resumed list appends: reload into a fresh capture
    c.snapshots_enable(True, 64)
    c.snapshots_load(str(tmp_path / "snapshots.conf"))
    assert np.array_equal(c.snapshots()["time"], sn["time"])
    # capacity
    d = M.Context(potentials=M.POT_AIREBO, task_mode=1)
    d.set_system(z, pos, vel, box, (1, 1, 0), fixed)
    d.set_atom_tags(tags)
    d.set_adaptive_dt(True, 1.0, 0.2)
    d.snapshots_enable(True, 2)
    with pytest.raises(M.MdgError) as e:
        d.run(200, 0.5)
        d.snapshots()
    assert e.value.code == -8
