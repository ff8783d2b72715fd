"""mdtrajsim's impact-sequence mode on one GPU (applications/mdtrajsim/main.cpp:113-345).

The reference loads a base state, then for each (x, y) of ``ionpos.bin``
places the projectile (the last atom) there and runs one trajectory after
another, each in its own directory ``%08d``.  Here the impacts of a chunk run
at the same time as one batched context: every impact is a system of its own
(adaptive dt, bath, fixed atoms and tags of the base), the step kernels cover
all of them, each system stops when its simTime reaches the base's
simTimeFinal, and each directory receives what runTraj leaves behind:

* ``ionpos_used.bin`` / ``ionpos_used.txt`` (main.cpp:304-317);
* the state files of SimLoopSaver, only the last iteration kept
  (main.cpp:163-169, 341);
* the XVA frames of SimLoop's schedule with CustomSimLoop's intervals
  (1 ps below 2 ps, then 5 ps, main.cpp:59-60);
* ``snapshots.conf``, CustomSimLoop's SnapshotList of the projectile and
  cluster atoms (main.cpp:62-85, 160);
* ``completed.ok`` once simTimeFinal is reached (main.cpp:162-166).

Impacts whose directory holds ``completed.ok`` or ``completed.error`` are
skipped, as isAlreadyFinished does (main.cpp:92-111).
"""
from __future__ import annotations

import bz2
import gzip
import lzma
import os
import re
from typing import Dict, List, Optional

import numpy as np

from . import (Context, POT_AIREBO, POT_METAL, TB_NONE, TB_UNIVERSE, TB_BOX, TB_SPHERE, ZIP_NONE, ZIP_GZIP, ZIP_XZ)

AO = 1e-8    # Angstrom in cm (consts.cxx:30)
FS = 1e-15   # fs in s (consts.cxx:36)
EL_Z = {1: 1, 12: 6, 64: 29, 108: 47, 197: 79, 40: 18, 131: 54}  # ElementID (consts.hpp:46-55) -> atomic number
_EXT = {ZIP_NONE: "", ZIP_GZIP: ".gz", ZIP_XZ: ".xz"}


def read_file(path: str) -> Optional[bytes]:
    """A file as yaatk::Stream finds it (plain, .xz, .bz2, .gz), or None."""
    for ext, op in (("", open), (".xz", lzma.open), (".bz2", bz2.open), (".gz", gzip.open)):
        if os.path.exists(path + ext):
            with op(path + ext, "rb") as f:
                return f.read()
    return None


def write_file(path: str, data: bytes, zip: int = ZIP_NONE):
    """A file as yaatk::Stream writes it with the given compression."""
    for ext in ("", ".gz", ".xz", ".bz2"):
        if os.path.exists(path + ext):
            os.remove(path + ext)
    op = {ZIP_NONE: open, ZIP_GZIP: gzip.open, ZIP_XZ: lzma.open}[zip]
    with op(path + _EXT[zip], "wb") as f:
        f.write(data)


def exists(path: str) -> bool:
    return any(os.path.exists(path + e) for e in ("", ".xz", ".bz2", ".gz"))


def read_state(id: str) -> Dict[str, np.ndarray]:
    """The SimLoopSaver files of ``id`` in Angstrom / fs / eV-free units:
    z, pos, vel, image, box, pbc, fixed, tb_apply, tags, bath, time, dt,
    time_final (SimLoopSaver.cxx:275-625)."""
    z = read_file(id + ".z")
    r = read_file(id + ".r")
    if z is None or r is None:
        raise FileNotFoundError(f"no state {id} (.z and .r are needed)")
    n = len(z)
    zz = np.array([EL_Z[b] for b in z], np.int32)
    pos = np.frombuffer(r, np.float64).reshape(n, 3) / AO
    v = read_file(id + ".v")
    vel = np.zeros((n, 3)) if v is None else np.frombuffer(v, np.float64).reshape(n, 3) / (AO / FS)
    pr = read_file(id + ".pbc_rect")
    prv = np.full(3, 10000.0 * AO) if pr is None else np.frombuffer(pr, np.float64)
    en = read_file(id + ".pbc_rect.enabled")
    pbc = (prv != 10000.0 * AO).astype(np.int32) if en is None else \
        np.frombuffer(en, np.uint8).reshape(n, 3)[0].astype(np.int32)
    cnt = read_file(id + ".pbc_rect.count")
    image = np.zeros((n, 3), np.int32) if cnt is None else np.frombuffer(cnt, np.int32).reshape(n, 3).copy()

    def flags(name, default):
        b = read_file(id + name)
        return np.full(n, default, np.uint8) if b is None else (np.frombuffer(b, np.uint8) != 0).astype(np.uint8)

    tags = np.zeros(n, np.uint8)
    for k, name in enumerate((".tag.target", ".tag.projectile", ".tag.substrate", ".tag.monomer", ".tag.cluster",
                              ".tag.fullerene")):
        tags |= (flags(name, 0) << (k + 1)).astype(np.uint8)
    bath = {"geom": TB_NONE, "T0": 0.0, "gamma": 1e13, "params": np.zeros(5)}
    cm = read_file(id + ".thermal_bath.common")
    if cm is not None:
        bath["T0"], bath["gamma"] = np.frombuffer(cm, np.float64)
    for name, geom in ((".thermal_bath.univserse", TB_UNIVERSE), (".thermal_bath.box", TB_BOX),
                       (".thermal_bath.sphere", TB_SPHERE)):
        b = read_file(id + name)
        if b is not None:
            bath["geom"] = geom
            p = np.frombuffer(b, np.float64) / AO
            bath["params"][:len(p)] = p
    tm = read_file(id + ".time")
    t = np.frombuffer(tm, np.float64) if tm is not None else np.array([0.0, 4e-12, 1e-20, 1e-20])
    return {"z": zz, "pos": pos, "vel": vel, "image": image, "box": prv / AO, "pbc": pbc,
            "fixed": flags(".tag.fixed", 0), "tb_apply": flags(".tag.thermal_bath_applicable", 1), "tags": tags,
            "bath": bath, "time": t[0] / FS, "time_final": t[1] / FS, "dt": t[2] / FS}


def remove_iterations(dirname: str, keep_first: bool, keep_last: bool):
    """SimLoopSaver::removeIterations (SimLoopSaver.cxx:765-800): state files
    of the iterations "md<digits>" in dirname but the first / last."""
    names = os.listdir(dirname)
    its = sorted({int(m.group(1)) for m in (re.match(r"md(\d+)", f) for f in names) if m})
    if its and keep_last:
        its = its[:-1]
    if its and keep_first:
        its = its[1:]
    drop = {"md%010d" % i for i in its}
    for f in names:
        if f.split(".")[0] in drop:
            os.remove(os.path.join(dirname, f))


def impact_sequence(base_id: str, ionpos_path: str, workdir: str, start: int = 0, batch: int = 256,
                    potentials: int = POT_AIREBO | POT_METAL, zip: int = ZIP_NONE, snapshot_capacity: int = 8192,
                    max_steps: int = 10 ** 9, timeaccel: float = 1.0, task_mode: int = 0) -> List[int]:
    """Runs the impacts of ``ionpos_path`` (pairs of doubles, cm) from impact
    ``start`` on, ``batch`` at a time; returns the impacts run.  The default
    potentials are the application's (setupPotentials with REBO); the
    application compresses with yaatk's first working method (``.xz`` where
    the xz program exists): pass ``zip=ZIP_XZ`` for the same files."""
    base = read_state(base_id)
    raw = read_file(ionpos_path)
    if raw is None or len(raw) % 16:
        raise ValueError(f"{ionpos_path}: not a list of (x, y) doubles")
    xy = np.frombuffer(raw, np.float64).reshape(-1, 2)
    todo = []
    for k in range(start, len(xy)):
        d = os.path.join(workdir, "%08d" % k)
        os.makedirs(d, exist_ok=True)
        if exists(os.path.join(d, "completed.ok")) or exists(os.path.join(d, "completed.error")):
            continue
        todo.append(k)
    for c0 in range(0, len(todo), batch):
        _run_chunk(base, xy, todo[c0:c0 + batch], workdir, potentials, zip, snapshot_capacity, max_steps,
                   timeaccel, task_mode)
    return todo


def _run_chunk(base, xy, impacts, workdir, potentials, zip, capacity, max_steps, timeaccel, task_mode):
    systems, dirs = [], []
    for k in impacts:
        s = {key: base[key].copy() for key in ("z", "pos", "vel", "box", "pbc", "fixed")}
        # the projectile is the last atom (main.cpp:301-303)
        s["pos"][-1, 0] = xy[k, 0] / AO
        s["pos"][-1, 1] = xy[k, 1] / AO
        systems.append(s)
        d = os.path.join(workdir, "%08d" % k)
        dirs.append(d)
        write_file(os.path.join(d, "ionpos_used.bin"), xy[k].tobytes(), zip)
        write_file(os.path.join(d, "ionpos_used.txt"), ("%g %g\n" % (xy[k, 0], xy[k, 1])).encode(), zip)
    m = len(systems)
    ctx = Context(potentials=potentials, task_mode=task_mode)
    if m == 1:
        s = systems[0]
        ctx.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    else:
        ctx.set_batch(systems)
    ctx.set_images(np.tile(base["image"], (m, 1)))
    ctx.set_atom_tags(np.tile(base["tags"], m))
    b = base["bath"]
    if b["geom"] != TB_NONE:
        ctx.set_thermal_bath(b["geom"], b["T0"], b["gamma"] * FS, b["params"], np.tile(base["tb_apply"], m))
    ctx.set_adaptive_dt(True, timeaccel, base["dt"])
    ctx.set_time(base["time"], base["dt"])
    ctx.set_time_final(base["time_final"])
    ctx.set_stop_at_time_final(True)
    ctx.set_output_dirs(dirs)
    ctx.set_output(workdir, 1000, 1e6 * 1000.0, zip)
    ctx.set_traj_schedule([2000.0, np.inf], [1000.0, 5000.0])
    for s, d in enumerate(dirs):
        ctx.write_state(os.path.join(d, "md%010d" % 0), zip=zip, sys=s)  # mds.write() (main.cpp:325)
    ctx.snapshots_enable(True, capacity)
    ctx.run_until_final(max_steps)
    ctx.flush_output()
    for s, d in enumerate(dirs):
        ctx.snapshots_write(os.path.join(d, "snapshots.conf"), zip=zip, sys=s)
    t, _ = ctx.get_time()
    for s, d in enumerate(dirs):
        if t[s] >= base["time_final"]:
            write_file(os.path.join(d, "completed.ok"), b"", zip)
        remove_iterations(d, keep_first=False, keep_last=True)
