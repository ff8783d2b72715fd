"""ctypes binding of the oracle harness (oracle/_ref/libmdtkref.so).

Test infrastructure only: imported by tests/, by __graft_entry__.smoke() as
the checker, and by bench.py's CPU-baseline leg.  The library is the reference
MDTK code compiled from its own sources (see oracle/Makefile); nothing in the
product imports this module.

Units at this interface: Angstrom, eV, fs.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libmdtkref.so")
RS_PATH = os.path.join(HERE, "_ref", "librestate.so")

POT_REBO = 1
POT_AIREBO_LJ = 2
POT_ETORS = 4
POT_BRENNER = 8
POT_AIREBO = POT_REBO | POT_AIREBO_LJ | POT_ETORS
POT_METAL = 16
# the drop-in GPU classes (mdtk_b200/mdtk/GpuPotentials.hpp) in the FProxy in
# place of the reference's own; needs install_gpu_shim() first
POT_GPU = 64
SHIM_PATH = os.path.join(HERE, "_ref", "libmdtkshim.so")

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run `make -C oracle`)")
        L = ctypes.CDLL(LIB_PATH)
        vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_create.restype = vp
        L.ref_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.ref_destroy.argtypes = [vp]
        L.ref_num_potentials.argtypes = [vp]
        L.ref_set_atoms.argtypes = [vp, ctypes.c_int, ip, dp, dp, dp, ip, ctypes.POINTER(ctypes.c_ubyte)]
        L.ref_compute.argtypes = [vp, dp, dp, dp, dp]
        L.ref_energy_proxy.argtypes = [vp, dp, dp]
        L.ref_nl_pairs.restype = ctypes.c_long
        L.ref_nl_pairs.argtypes = [vp, ctypes.c_int, ip, ctypes.c_long]
        L.ref_set_param.argtypes = [vp, ctypes.c_int, ctypes.c_double]
        L.ref_set_bath.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, dp,
                                   ctypes.POINTER(ctypes.c_ubyte)]
        L.ref_set_adaptive.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.ref_last_run_dts.argtypes = [vp, dp, ctypes.c_int]
        L.ref_rcutoff.restype = ctypes.c_double
        L.ref_rcutoff.argtypes = [vp, ctypes.c_int]
        L.ref_run.argtypes = [vp, ctypes.c_int, ctypes.c_double, dp, dp, ip, dp, dp, dp]
        L.ref_last_run_times.argtypes = [vp, dp, ctypes.c_int]
        ub = ctypes.POINTER(ctypes.c_ubyte)
        L.ref_set_zip.argtypes = [ctypes.c_int]
        L.ref_write_state.argtypes = [vp, ctypes.c_char_p]
        L.ref_write_xva.argtypes = [vp, ctypes.c_char_p]
        L.ref_load_state.argtypes = [vp, ctypes.c_char_p, ctypes.c_ulong]
        L.ref_atom_count.argtypes = [vp]
        L.ref_get_atoms.argtypes = [vp, dp, dp, dp, ip, ub, ub, ub, ip]
        L.ref_set_tags.argtypes = [vp, ub]
        L.ref_get_loop.argtypes = [vp, dp]
        L.ref_set_output.argtypes = [vp, ctypes.c_char_p, ctypes.c_long, ctypes.c_double]
        L.ref_set_time.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.ref_impact_sequence.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
        L.ref_tables.restype = ctypes.c_long
        L.ref_tables.argtypes = [ctypes.c_int, ctypes.c_int, dp, ctypes.c_long]
        L.ref_spline_eval.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp]
        _lib = L
    return _lib


_shim = None


def install_gpu_shim():
    """Load oracle/_ref/libmdtkshim.so (the GPU classes compiled against the
    reference headers) and install its factory, so RefSystem(potset | POT_GPU)
    holds GpuREBO / GpuAIREBO / GpuETors / GpuBrenner."""
    global _shim
    if _shim is None:
        lib()
        if not os.path.exists(SHIM_PATH):
            raise RuntimeError(f"shim library missing: {SHIM_PATH} (run `make -C oracle`)")
        S = ctypes.CDLL(SHIM_PATH)
        S.shim_last_error.restype = ctypes.c_char_p
        if S.shim_install() != 0:
            raise RuntimeError("shim_install failed")
        _shim = S
    return _shim


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _check(rc):
    if rc is None or (isinstance(rc, int) and rc < 0):
        raise RuntimeError("oracle: " + lib().ref_last_error().decode())
    return rc


class RefSystem:
    """One reference SimLoop with a potential stack and an atom set."""

    def __init__(self, potset: int, brenner_set: int = 1, lj_cut_mode: int = 0):
        h = lib().ref_create(potset, brenner_set, lj_cut_mode)
        if not h:
            msg = lib().ref_last_error().decode()
            if potset & POT_GPU and _shim is not None:
                msg += ": " + _shim.shim_last_error().decode()
            raise RuntimeError("oracle: " + msg)
        self.h = ctypes.c_void_p(h)
        self.n = 0
        self.npot = lib().ref_num_potentials(self.h)

    def close(self):
        if self.h:
            lib().ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_atoms(self, z, pos, vel=None, box=(0.0, 0.0, 0.0), pbc=(1, 1, 1), fixed=None):
        z = np.ascontiguousarray(z, dtype=np.int32)
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        n = len(z)
        velp = None
        if vel is not None:
            self._vel = np.ascontiguousarray(vel, dtype=np.float64).reshape(-1, 3)
            velp = _dp(self._vel)
        boxa = np.ascontiguousarray(box, dtype=np.float64)
        pbca = np.ascontiguousarray(pbc, dtype=np.int32)
        fx = None
        if fixed is not None:
            self._fixed = np.ascontiguousarray(fixed, dtype=np.uint8)
            fx = self._fixed.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte))
        _check(lib().ref_set_atoms(self.h, n, _ip(z), _dp(pos), velp, _dp(boxa), _ip(pbca), fx))
        self.n = n

    def compute(self, per_term: bool = False):
        """Returns (E_total, E_terms[npot], grad[n,3]) (+ grad_terms[npot,n,3])."""
        e = np.zeros(1)
        et = np.zeros(self.npot)
        g = np.zeros((self.n, 3))
        gt = np.zeros((self.npot, self.n, 3)) if per_term else None
        _check(lib().ref_compute(self.h, _dp(e), _dp(et), _dp(g), _dp(gt) if per_term else None))
        if per_term:
            return float(e[0]), et, g, gt
        return float(e[0]), et, g

    def nl_pairs(self, index: int) -> np.ndarray:
        cnt = lib().ref_nl_pairs(self.h, index, None, 0)
        _check(cnt)
        out = np.zeros((max(cnt, 1), 2), dtype=np.int32)
        _check(lib().ref_nl_pairs(self.h, index, _ip(out), cnt))
        return out[:cnt]

    def set_bath(self, geom: int, T0: float, gamma_per_s: float, params=None, flags=None):
        """SimLoop's thermal bath (geom 0 none, 1 universe, 2 box, 3 sphere)."""
        self._bp = np.zeros(5) if params is None else np.ascontiguousarray(np.resize(params, 5), dtype=np.float64)
        fl = None
        if flags is not None:
            self._bf = np.ascontiguousarray(flags, dtype=np.uint8)
            fl = self._bf.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte))
        _check(lib().ref_set_bath(self.h, geom, T0, gamma_per_s, _dp(self._bp), fl))

    def set_adaptive(self, on: bool, timeaccel: float = 1.0, dt0: float = 0.5):
        _check(lib().ref_set_adaptive(self.h, 1 if on else 0, timeaccel, dt0))

    def last_run_dts(self, n: int) -> np.ndarray:
        out = np.zeros(n)
        lib().ref_last_run_dts(self.h, _dp(out), n)
        return out

    def set_param(self, pid: int, value: float):
        """Override a C-C pair parameter (ids as include/mdg.h MDG_PARAM_*)."""
        _check(lib().ref_set_param(self.h, pid, ctypes.c_double(value)))

    def rcutoff(self, index: int) -> float:
        return float(lib().ref_rcutoff(self.h, index))

    def run(self, nsteps: int, dt_fs: float):
        """Unmodified SimLoop::execute; returns dict of final state + per-step energies."""
        pos = np.zeros((self.n, 3))
        vel = np.zeros((self.n, 3))
        img = np.zeros((self.n, 3), dtype=np.int32)
        ep = np.zeros(nsteps)
        et = np.zeros(nsteps)
        e0 = np.zeros(1)
        _check(lib().ref_run(self.h, nsteps, dt_fs, _dp(pos), _dp(vel), _ip(img), _dp(ep), _dp(et), _dp(e0)))
        ts = np.zeros(nsteps + 2)
        lib().ref_last_run_times(self.h, _dp(ts), nsteps + 2)
        return {"pos": pos, "vel": vel, "image": img, "epot": ep, "etot": et, "e0": float(e0[0]), "times": ts}


def impact_sequence(potset: int, base_id: str, ionpos_path: str, workdir: str, start: int = 0):
    """mdtrajsim's impact-sequence mode (main.cpp:113-345) on the reference,
    with this harness's potential set."""
    _check(lib().ref_impact_sequence(potset, os.fsencode(base_id), os.fsencode(ionpos_path), os.fsencode(workdir),
                                     start))


def set_zip(mode: int):
    """Compression of the reference's files: 0 plain, 1 .gz, 2 .xz."""
    _check(lib().ref_set_zip(mode))


def _ub(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte))


def _write_state(self, id: str):
    """SimLoopSaver::write(id)."""
    _check(lib().ref_write_state(self.h, os.fsencode(id)))


def _write_xva(self, path: str):
    """SimLoop::saveToStreamXVA into path."""
    _check(lib().ref_write_xva(self.h, os.fsencode(path)))


def _load_state(self, id: str, iteration: int = 0) -> int:
    """SimLoopSaver::load(id) with SimLoop::iteration = iteration; later
    runs continue the loaded time and iteration."""
    got = lib().ref_load_state(self.h, os.fsencode(id), int(iteration))
    _check(-1 if got < 0 else 0)
    self.n = lib().ref_atom_count(self.h)
    return got


def _atoms(self) -> dict:
    """Per-atom state (A, A/fs, A/fs^2) and flags of the reference's atoms."""
    n = lib().ref_atom_count(self.h)
    out = {"pos": np.zeros((n, 3)), "vel": np.zeros((n, 3)), "acc": np.zeros((n, 3)),
           "image": np.zeros((n, 3), np.int32), "fixed": np.zeros(n, np.uint8), "tb_apply": np.zeros(n, np.uint8),
           "tags": np.zeros(n, np.uint8), "z": np.zeros(n, np.int32)}
    _check(lib().ref_get_atoms(self.h, _dp(out["pos"]), _dp(out["vel"]), _dp(out["acc"]), _ip(out["image"]),
                               _ub(out["fixed"]), _ub(out["tb_apply"]), _ub(out["tags"]), _ip(out["z"])))
    return out


def _set_tags(self, tags):
    t = np.ascontiguousarray(tags, dtype=np.uint8)
    _check(lib().ref_set_tags(self.h, _ub(t)))


def _loop(self) -> dict:
    """SimLoop scalars: time (fs), dt, dt_prev, iteration, bath, box, Check (eV, K)."""
    o = np.zeros(22)
    _check(lib().ref_get_loop(self.h, _dp(o)))
    return {"time": o[0], "dt": o[1], "dt_prev": o[2], "iteration": int(o[3]), "tb_geom": int(o[4]),
            "tb_T0": o[5], "tb_gamma": o[6], "tb_params": o[7:12].copy(), "box": o[12:15].copy(),
            "net_force": o[15:18].copy(), "e0": o[18], "e_cur": o[19], "e_bath": o[20], "T": o[21]}


def _set_output(self, dir, flush_interval: int = 0, traj_interval_fs: float = 0.0):
    """SimLoop's own file output (writestate, writetrajXVA) in later runs."""
    _check(lib().ref_set_output(self.h, None if dir is None else os.fsencode(dir), int(flush_interval),
                                float(traj_interval_fs)))


def _set_time(self, time_fs: float, time_final_fs: float, dt_fs: float):
    """SimLoop::simTime, simTimeFinal, dt."""
    _check(lib().ref_set_time(self.h, time_fs, time_final_fs, dt_fs))


RefSystem.set_time = _set_time
RefSystem.set_output = _set_output
RefSystem.write_state = _write_state
RefSystem.write_xva = _write_xva
RefSystem.load_state = _load_state
RefSystem.atoms = _atoms
RefSystem.set_tags = _set_tags
RefSystem.loop = _loop


def tables(which: int, brenner_set: int = 1) -> np.ndarray:
    n = lib().ref_tables(which, brenner_set, None, 0)
    _check(n)
    out = np.zeros(n)
    _check(lib().ref_tables(which, brenner_set, _dp(out), n))
    return out


def spline_eval(fn: int, x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
    out = np.zeros(len(x))
    _check(lib().ref_spline_eval(fn, len(x), _dp(x), _dp(out)))
    return out


# ---------------------------------------------------------------- restatement
_rs = None


def restatement_available() -> bool:
    return os.path.exists(RS_PATH)


def rs_lib():
    global _rs
    if _rs is None:
        if not restatement_available():
            raise RuntimeError(f"restatement library missing: {RS_PATH} (run `make -C oracle restate`)")
        L = ctypes.CDLL(RS_PATH)
        ip, dp = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        L.rs_energy.argtypes = [ctypes.c_int] * 4 + [ip, dp, dp, ip, dp]
        L.rs_energy_dir.argtypes = [ctypes.c_int] * 4 + [ip, dp, dp, dp, ip, dp]
        L.rs_opcount.argtypes = [ctypes.c_int] * 3 + [ip, dp, dp, ip, ctypes.POINTER(ctypes.c_long)]
        _rs = L
    return _rs


def _sys_args(s):
    z = np.ascontiguousarray(s["z"], dtype=np.int32)
    pos = np.ascontiguousarray(s["pos"], dtype=np.float64)
    box = np.ascontiguousarray(s["box"], dtype=np.float64)
    pbc = np.ascontiguousarray(s["pbc"], dtype=np.int32)
    return z, pos, box, pbc


def rs_energy(s, potset, brenner_set=1, lj_cut_mode=0) -> np.ndarray:
    """Restated energies (eV): [REBO, AIREBO LJ, torsion, Brenner]."""
    z, pos, box, pbc = _sys_args(s)
    out = np.zeros(4)
    rs_lib().rs_energy(potset, brenner_set, lj_cut_mode, len(z), _ip(z), _dp(pos), _dp(box), _ip(pbc), _dp(out))
    return out


def rs_energy_dir(s, potset, direction, brenner_set=1, lj_cut_mode=0) -> np.ndarray:
    """Exact directional derivatives dE/d(direction) of each term (forward-mode duals)."""
    z, pos, box, pbc = _sys_args(s)
    d = np.ascontiguousarray(direction, dtype=np.float64)
    out = np.zeros(4)
    rs_lib().rs_energy_dir(potset, brenner_set, lj_cut_mode, len(z), _ip(z), _dp(pos), _dp(d), _dp(box), _ip(pbc),
                           _dp(out))
    return out


OP_NAMES = ("add", "mul", "div", "sqrt", "exp", "cos", "pow")


def rs_opcount(s, potset, brenner_set=1, bstar=False) -> dict:
    """Floating-point operations of one restated energy evaluation (with
    bstar=True: only those spent in the LJ term's b*_ij evaluations)."""
    z, pos, box, pbc = _sys_args(s)
    out = np.zeros(16, dtype=np.int64)
    rs_lib().rs_opcount(potset, brenner_set, len(z), _ip(z), _dp(pos), _dp(box), _ip(pbc),
                        out.ctypes.data_as(ctypes.POINTER(ctypes.c_long)))
    o = out[8:15] if bstar else out[:7]
    return {k: int(v) for k, v in zip(OP_NAMES, o)}
