"""mdtk_b200: the MDTK per-step hot path on one B200, behind the C ABI of
include/mdg.h (library: mdtk_b200/libmdg.so, built by mdtk_b200.build).

This module is a thin ctypes view of that ABI for tests and benchmarks.  It
never computes anything itself: without the CUDA library (or without a GPU)
every call fails loudly.

    ctx = Context(potentials=POT_AIREBO)
    ctx.set_system(z, pos, vel, box, pbc, fixed)
    e, e_terms, grad = ctx.compute()          # FProxy::operator()
    epot, etot = ctx.run(100, dt=0.25)        # SimLoop step loop, fixed dt
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmdg.so")

POT_REBO = 1
POT_AIREBO_LJ = 2
POT_ETORS = 4
POT_BRENNER = 8
POT_METAL = 16  # FBZL, FLJ, Ackland (applications/common.h:36-77): Cu, Ag, Au, Ar, Xe
POT_AIREBO = POT_REBO | POT_AIREBO_LJ | POT_ETORS

# parameters the adjoint differentiates (include/mdg.h MDG_PARAM_*)
PARAM_LJ_EPS_CC = 0
PARAM_LJ_SIGMA_CC = 1
PARAM_REBO_A_CC = 2
PARAM_REBO_B1_CC = 3
PARAM_REBO_ALPHA_CC = 4
PARAM_REBO_BETA1_CC = 5
NPARAM = 6
PARAM_NAMES = ("eps_CC", "sigma_CC", "A_CC", "B1_CC", "alpha_CC", "beta1_CC")

TB_NONE, TB_UNIVERSE, TB_BOX, TB_SPHERE = 0, 1, 2, 3

# checkpoint and trajectory files (include/mdg.h MDG_ZIP_*, MDG_LOADED_*)
ZIP_NONE, ZIP_GZIP, ZIP_XZ = 0, 1, 2
LOADED_Z, LOADED_R, LOADED_V = 1, 2, 4
LOADED_PBC_RECT, LOADED_PBC_COUNT, LOADED_PBC_ENABLED, LOADED_A = 8, 16, 32, 64
# Atom tag bits (Atom.hpp:84-90)
TAG_TARGET, TAG_PROJECTILE, TAG_SUBSTRATE, TAG_MONOMER, TAG_CLUSTER, TAG_FULLERENE = (1 << k for k in range(1, 7))

UNITS_AEVFS = 0
UNITS_CGS = 1
PREC_FP64 = 0
PREC_FP32_MIXED = 1


class MdgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"mdg error {code}: {msg}")
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [
        ("potentials", ctypes.c_int),
        ("brenner_set", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("units", ctypes.c_int),
        ("lj_cut_mode", ctypes.c_int),
        ("nl_skin_mode", ctypes.c_int),
        ("nl_skin", ctypes.c_double),
        ("cap_rebo_list", ctypes.c_int),
        ("cap_lj_list", ctypes.c_int),
        ("cap_bonds", ctypes.c_int),
        ("cap_cij", ctypes.c_int),
        ("cap_special", ctypes.c_int),
        ("special_avg", ctypes.c_int),
        ("device", ctypes.c_int),
        ("bond_rec_avg", ctypes.c_int),
        ("task_mode", ctypes.c_int),
    ]


_lib = None


def lib():
    """Load libmdg.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -c 'import __graft_entry__ as g; g.build()'`")
        L = ctypes.CDLL(LIB_PATH)
        vp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
        i32p = ctypes.POINTER(ctypes.c_int32)
        L.mdg_default_params.argtypes = [ctypes.POINTER(Params)]
        L.mdg_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(vp)]
        L.mdg_destroy.argtypes = [vp]
        L.mdg_last_error.restype = ctypes.c_char_p
        L.mdg_set_stream.argtypes = [vp, vp]
        L.mdg_set_system.argtypes = [vp, ctypes.c_int, i32p, dp, dp, dp, i32p, ctypes.POINTER(ctypes.c_uint8)]
        L.mdg_set_positions.argtypes = [vp, dp]
        L.mdg_set_state.argtypes = [vp, dp, dp]
        L.mdg_compute.argtypes = [vp, dp, dp, dp]
        L.mdg_nl_pairs.argtypes = [vp, ctypes.c_int, i32p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
        L.mdg_nl_update.argtypes = [vp, ctypes.c_int, i32p]
        L.mdg_run.argtypes = [vp, ctypes.c_int, ctypes.c_double, dp, dp]
        L.mdg_set_batch.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int64), i32p, dp, dp, dp, i32p,
                                    ctypes.POINTER(ctypes.c_uint8)]
        L.mdg_batch_energies.argtypes = [vp, dp]
        L.mdg_task_mode.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float),
                                    ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
        L.mdg_batch_run.argtypes = [vp, ctypes.c_int, ctypes.c_double, dp, dp]
        L.mdg_tuned_launch.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.mdg_set_dependent_launch.argtypes = [vp, ctypes.c_int]
        L.mdg_set_thermal_bath.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, dp,
                                           ctypes.POINTER(ctypes.c_uint8)]
        L.mdg_set_adaptive_dt.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.mdg_get_time.argtypes = [vp, dp, dp]
        L.mdg_sync.argtypes = [vp]
        L.mdg_get_state.argtypes = [vp, dp, dp, i32p]
        L.mdg_launch_count.argtypes = [vp]
        L.mdg_launch_count.restype = ctypes.c_int64
        L.mdg_step_host.argtypes = [vp, ctypes.c_int, ctypes.c_double, dp, dp, dp, dp]
        L.mdg_set_profiling.argtypes = [vp, ctypes.c_int]
        L.mdg_profile_read.argtypes = [vp, ctypes.c_int, ctypes.c_char_p, dp, ctypes.POINTER(ctypes.c_int64),
                                       ctypes.POINTER(ctypes.c_int)]
        L.mdg_pipe_peak.argtypes = [ctypes.c_int, ctypes.c_int, dp]
        L.mdg_launch_floor.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp]
        L.mdg_debug_brenner_tables.argtypes = [ctypes.c_int, dp, ctypes.c_int64]
        L.mdg_debug_brenner_tables.restype = ctypes.c_int64
        L.mdg_debug_spline.argtypes = [ctypes.c_int] * 4 + [dp, dp]
        L.mdg_set_param.argtypes = [vp, ctypes.c_int, ctypes.c_double]
        L.mdg_get_param.argtypes = [vp, ctypes.c_int, dp]
        L.mdg_force_product.argtypes = [vp, dp, ctypes.c_int, dp, dp, dp, dp]
        L.mdg_adjoint_forward.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, dp, dp, dp]
        L.mdg_adjoint_backward.argtypes = [vp, dp, dp, ctypes.c_double, dp, dp, dp]
        L.mdg_debug_rebo_tables.argtypes = [dp, ctypes.c_int64]
        L.mdg_debug_rebo_tables.restype = ctypes.c_int64
        u8p = ctypes.POINTER(ctypes.c_uint8)
        L.mdg_set_atom_tags.argtypes = [vp, u8p]
        L.mdg_get_atom_tags.argtypes = [vp, u8p]
        L.mdg_write_state.argtypes = [vp, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        L.mdg_write_xva.argtypes = [vp, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        L.mdg_load_state.argtypes = [vp, ctypes.c_char_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int)]
        L.mdg_set_output.argtypes = [vp, ctypes.c_char_p, ctypes.c_int64, ctypes.c_double, ctypes.c_int]
        L.mdg_flush_output.argtypes = [vp]
        L.mdg_get_iteration.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64)]
        L.mdg_set_time_final.argtypes = [vp, ctypes.c_double]
        L.mdg_atom_count.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
        L.mdg_set_time.argtypes = [vp, dp, dp]
        L.mdg_set_stop_at_time_final.argtypes = [vp, ctypes.c_int]
        L.mdg_run_until_final.argtypes = [vp, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64),
                                          ctypes.POINTER(ctypes.c_int)]
        L.mdg_set_output_dirs.argtypes = [vp, ctypes.POINTER(ctypes.c_char_p)]
        L.mdg_set_traj_schedule.argtypes = [vp, ctypes.c_int, dp, dp]
        L.mdg_snapshots_enable.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.mdg_snapshots_set_schedule.argtypes = [vp, ctypes.c_int, dp, dp]
        L.mdg_snapshots_count.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.mdg_snapshots_get.argtypes = [vp, ctypes.c_int, dp, ctypes.POINTER(ctypes.c_uint32), i32p,
                                        ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
        L.mdg_snapshots_write.argtypes = [vp, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
        L.mdg_snapshots_load.argtypes = [vp, ctypes.c_int, ctypes.c_char_p]
        L.mdg_set_images.argtypes = [vp, i32p]
        _lib = L
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def _check(rc: int):
    if rc != 0:
        raise MdgError(rc, lib().mdg_last_error().decode())


def pipe_peak(device: int = 0, fp32: bool = False) -> float:
    """Measured FMA throughput (TFLOP/s) of the FP64 or FP32 CUDA-core pipe."""
    out = np.zeros(1)
    _check(lib().mdg_pipe_peak(device, 1 if fp32 else 0, _dp(out)))
    return float(out[0])


def launch_floor(device: int = 0, phases: int = 22):
    """(graph_us, coop_us): per-step floor of `phases` empty dependent phases
    as a graph of dependent launches and as one cooperative kernel."""
    g = np.zeros(1)
    c = np.zeros(1)
    _check(lib().mdg_launch_floor(device, phases, _dp(g), _dp(c)))
    return float(g[0]), float(c[0])


def debug_brenner_tables(set_: int) -> np.ndarray:
    n = lib().mdg_debug_brenner_tables(set_, None, 0)
    out = np.zeros(n)
    lib().mdg_debug_brenner_tables(set_, _dp(out), n)
    return out


def debug_spline(precision: int, kind: int, fam: int, args) -> np.ndarray:
    """Host evaluation of a REBO spline family (kind 0 = G, 1 = P, 2 = pi_rc/T)."""
    nin, nout = {0: (1, 2), 1: (2, 3), 2: (3, 4)}[kind]
    a = np.ascontiguousarray(np.asarray(args, dtype=np.float64).reshape(-1, nin))
    out = np.zeros((a.shape[0], nout))
    _check(lib().mdg_debug_spline(precision, kind, fam, a.shape[0], _dp(a), _dp(out)))
    return out


def debug_rebo_tables() -> np.ndarray:
    n = lib().mdg_debug_rebo_tables(None, 0)
    out = np.zeros(n)
    lib().mdg_debug_rebo_tables(_dp(out), n)
    return out


class Context:
    """One mdg context: a potential stack plus a loaded atom set."""

    def __init__(self, potentials: int = POT_REBO, precision: int = PREC_FP64, units: int = UNITS_AEVFS,
                 lj_cut_mode: int = 0, nl_skin_mode: int = 0, nl_skin: float = 0.3, brenner_set: int = 1,
                 device: int = 0, **caps):
        p = Params()
        lib().mdg_default_params(ctypes.byref(p))
        p.potentials = potentials
        p.precision = precision
        p.units = units
        p.lj_cut_mode = lj_cut_mode
        p.nl_skin_mode = nl_skin_mode
        p.nl_skin = nl_skin
        p.brenner_set = brenner_set
        p.device = device
        for k, v in caps.items():
            setattr(p, k, v)
        h = ctypes.c_void_p()
        _check(lib().mdg_create(ctypes.byref(p), ctypes.byref(h)))
        self.h = h
        self.n = 0

    def close(self):
        if self.h:
            lib().mdg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int):
        _check(lib().mdg_set_stream(self.h, ctypes.c_void_p(stream_ptr)))

    def set_system(self, z, pos, vel=None, box=(0, 0, 0), pbc=(1, 1, 1), fixed=None):
        z = np.ascontiguousarray(z, dtype=np.int32)
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        vel = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64).reshape(-1, 3)
        box = np.ascontiguousarray(box, dtype=np.float64)
        pbc = np.ascontiguousarray(pbc, dtype=np.int32)
        fx = None
        if fixed is not None:
            fixed = np.ascontiguousarray(fixed, dtype=np.uint8)
            fx = fixed.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
        _check(lib().mdg_set_system(self.h, len(z), _ip(z), _dp(pos), _dp(vel), _dp(box), _ip(pbc), fx))
        self.n = len(z)

    def set_batch(self, systems):
        """Load independent systems (dicts as the builders return) into one
        batched context; atoms are concatenated in list order."""
        self.first = np.zeros(len(systems) + 1, dtype=np.int64)
        self.first[1:] = np.cumsum([len(s["z"]) for s in systems])
        z = np.ascontiguousarray(np.concatenate([s["z"] for s in systems]), dtype=np.int32)
        pos = np.ascontiguousarray(np.concatenate([s["pos"] for s in systems]), dtype=np.float64)
        vel = np.ascontiguousarray(np.concatenate([s["vel"] for s in systems]), dtype=np.float64)
        box = np.ascontiguousarray(np.concatenate([np.asarray(s["box"], float) for s in systems]))
        pbc = np.ascontiguousarray(np.concatenate([np.asarray(s["pbc"]) for s in systems]), dtype=np.int32)
        fixed = np.ascontiguousarray(np.concatenate([s["fixed"] for s in systems]), dtype=np.uint8)
        _check(lib().mdg_set_batch(self.h, len(systems), self.first.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                   _ip(z), _dp(pos), _dp(vel), _dp(box), _ip(pbc),
                                   fixed.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))
        self.n = len(z)
        self.nsys = len(systems)

    def task_mode(self):
        """(mode, ms_directed, ms_per_bond, ms_split): REBO task mode in use
        (1 directed, 2 per bond, 3 per bond on lane pairs) and the autotuner's
        timings (0 when it did not run)."""
        m = ctypes.c_int()
        a = ctypes.c_float()
        b = ctypes.c_float()
        d = ctypes.c_float()
        _check(lib().mdg_task_mode(self.h, ctypes.byref(m), ctypes.byref(a), ctypes.byref(b), ctypes.byref(d)))
        return m.value, a.value, b.value, d.value

    def set_thermal_bath(self, geom: int, T0: float = 0.0, gamma: float = 0.01, params=None, apply=None):
        """SimLoop's thermal bath: geom TB_* , T0 (K), gamma (1/time unit),
        params (box: zMin, dBoundary, zMinOfFreeZone; sphere: cx, cy, cz,
        radius, zMinOfFreeZone), apply: per-atom flags or None."""
        prm = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
        ap = None
        if apply is not None:
            self._tb_apply = np.ascontiguousarray(apply, dtype=np.uint8)
            ap = self._tb_apply.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
        _check(lib().mdg_set_thermal_bath(self.h, geom, float(T0), float(gamma), _dp(prm), ap))

    def set_adaptive_dt(self, on: bool, timeaccel: float = 1.0, dt0: float = 0.5):
        _check(lib().mdg_set_adaptive_dt(self.h, 1 if on else 0, float(timeaccel), float(dt0)))

    def get_time(self):
        """(simulated time, current dt) per system."""
        ns = getattr(self, "nsys", 1)
        t = np.zeros(ns)
        d = np.zeros(ns)
        _check(lib().mdg_get_time(self.h, _dp(t), _dp(d)))
        return t, d

    # ---- checkpoint and trajectory files (SimLoopSaver, SimLoop::saveToStreamXVA)

    def set_atom_tags(self, tags=None):
        """Per-atom TAG_* bits carried into the '.tag.*' state files."""
        t = None if tags is None else np.ascontiguousarray(tags, dtype=np.uint8)
        _check(lib().mdg_set_atom_tags(self.h, None if t is None else t.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))

    def get_atom_tags(self) -> np.ndarray:
        t = np.zeros(self.n, np.uint8)
        _check(lib().mdg_get_atom_tags(self.h, t.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))
        return t

    def write_state(self, id: str, zip: int = ZIP_NONE, sys: int = 0):
        """SimLoopSaver::write(id): the state files '<id>.<attribute>'."""
        _check(lib().mdg_write_state(self.h, sys, os.fsencode(id), zip))

    def write_xva(self, path: str, zip: int = ZIP_NONE, sys: int = 0):
        """SimLoop::saveToStreamXVA into path."""
        _check(lib().mdg_write_xva(self.h, sys, os.fsencode(path), zip))

    def load_state(self, id: str, iteration: int = 0) -> int:
        """SimLoopSaver::loadIteration: loads '<id>.*' as this context's
        system at the given iteration; returns the LOADED_* bits."""
        got = ctypes.c_int()
        _check(lib().mdg_load_state(self.h, os.fsencode(id), int(iteration), ctypes.byref(got)))
        n = ctypes.c_int()
        _check(lib().mdg_atom_count(self.h, ctypes.byref(n)))
        self.n = n.value
        self.nsys = 1
        return got.value

    def set_output(self, dir, flush_interval: int = 0, traj_interval: float = 0.0, zip: int = ZIP_NONE):
        """SimLoop::executeMain's file output inside run(): state files every
        flush_interval iterations, XVA frames every traj_interval of time;
        dir None stops it."""
        _check(lib().mdg_set_output(self.h, None if dir is None else os.fsencode(dir), int(flush_interval),
                                    float(traj_interval), zip))

    def flush_output(self):
        _check(lib().mdg_flush_output(self.h))

    def iteration(self) -> int:
        it = ctypes.c_uint64()
        _check(lib().mdg_get_iteration(self.h, ctypes.byref(it)))
        return it.value

    def set_time_final(self, t: float):
        _check(lib().mdg_set_time_final(self.h, float(t)))

    def set_time(self, sim_time, dt):
        """Per-system simulated time and dt (time units)."""
        ns = getattr(self, "nsys", 1)
        t = np.ascontiguousarray(np.broadcast_to(np.asarray(sim_time, float), (ns,)))
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, float), (ns,)))
        _check(lib().mdg_set_time(self.h, _dp(t), _dp(d)))

    def set_images(self, image):
        """PBC_count of every atom ([n, 3])."""
        im = np.ascontiguousarray(image, dtype=np.int32)
        _check(lib().mdg_set_images(self.h, _ip(im)))

    def set_stop_at_time_final(self, on: bool = True):
        _check(lib().mdg_set_stop_at_time_final(self.h, 1 if on else 0))

    def run_until_final(self, max_steps: int = 10 ** 9):
        """Steps until every system reached simTimeFinal; (steps, finished)."""
        st = ctypes.c_int64()
        fin = ctypes.c_int()
        _check(lib().mdg_run_until_final(self.h, int(max_steps), ctypes.byref(st), ctypes.byref(fin)))
        return st.value, bool(fin.value)

    def set_output_dirs(self, dirs):
        arr = None
        if dirs is not None:
            self._dirs = [os.fsencode(d) for d in dirs]
            arr = (ctypes.c_char_p * len(self._dirs))(*self._dirs)
        _check(lib().mdg_set_output_dirs(self.h, arr))

    def set_traj_schedule(self, until, interval):
        u = np.ascontiguousarray(until, dtype=np.float64)
        v = np.ascontiguousarray(interval, dtype=np.float64)
        _check(lib().mdg_set_traj_schedule(self.h, len(u), _dp(u), _dp(v)))

    # ---- SnapshotList

    def snapshots_enable(self, on: bool = True, capacity: int = 4096):
        _check(lib().mdg_snapshots_enable(self.h, 1 if on else 0, int(capacity)))

    def snapshots_set_schedule(self, until, interval):
        u = np.ascontiguousarray(until, dtype=np.float64)
        v = np.ascontiguousarray(interval, dtype=np.float64)
        _check(lib().mdg_snapshots_set_schedule(self.h, len(u), _dp(u), _dp(v)))

    def snapshots(self, sys: int = 0) -> dict:
        """times (time units), indices, and per snapshot and atom the PBC
        counters, float coordinates (cm) and velocities (cm/s)."""
        ns, na = ctypes.c_int(), ctypes.c_int()
        _check(lib().mdg_snapshots_count(self.h, sys, ctypes.byref(ns), ctypes.byref(na)))
        t = np.zeros(ns.value)
        idx = np.zeros(na.value, np.uint32)
        pc = np.zeros((ns.value, na.value, 3), np.int32)
        p = np.zeros((ns.value, na.value, 3), np.float32)
        v = np.zeros((ns.value, na.value, 3), np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        _check(lib().mdg_snapshots_get(self.h, sys, _dp(t), idx.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                       _ip(pc), p.ctypes.data_as(fp), v.ctypes.data_as(fp)))
        return {"time": t, "indices": idx, "pbc_count": pc, "pos": p, "vel": v}

    def snapshots_write(self, path: str, zip: int = ZIP_NONE, text: bool = False, sys: int = 0):
        _check(lib().mdg_snapshots_write(self.h, sys, os.fsencode(path), zip, 1 if text else 0))

    def snapshots_load(self, path: str, sys: int = 0):
        _check(lib().mdg_snapshots_load(self.h, sys, os.fsencode(path)))

    def tuned_launch(self):
        """(overlap, rebo_blocks): the autotuner's launch choice."""
        o = ctypes.c_int()
        b = ctypes.c_int()
        _check(lib().mdg_tuned_launch(self.h, ctypes.byref(o), ctypes.byref(b)))
        return o.value, b.value

    def set_dependent_launch(self, on: bool):
        """Programmatic dependent launch of the step's kernels (default on)."""
        _check(lib().mdg_set_dependent_launch(self.h, 1 if on else 0))

    def batch_energies(self) -> np.ndarray:
        """[nsys, 4]: REBO, LJ, torsion, kinetic energy of each system."""
        out = np.zeros((self.nsys, 4))
        _check(lib().mdg_batch_energies(self.h, _dp(out)))
        return out

    def batch_run(self, nsteps: int, dt: float):
        """Steps every system; returns (epot, etot) as [nsteps, nsys]."""
        ep = np.zeros((nsteps, self.nsys))
        et = np.zeros((nsteps, self.nsys))
        _check(lib().mdg_batch_run(self.h, nsteps, dt, _dp(ep), _dp(et)))
        return ep, et

    def set_state(self, pos, vel=None):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        vel = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64)
        _check(lib().mdg_set_state(self.h, _dp(pos), _dp(vel)))

    def compute(self) -> Tuple[float, np.ndarray, np.ndarray]:
        e = np.zeros(1)
        et = np.zeros(4)
        g = np.zeros((self.n, 3))
        _check(lib().mdg_compute(self.h, _dp(e), _dp(et), _dp(g)))
        return float(e[0]), et, g

    def nl_update(self, force: bool = False) -> np.ndarray:
        """Rebuild the Verlet lists if the displacement criterion fires (or
        always, with force); returns which of the three lists were rebuilt."""
        out = np.zeros(3, np.int32)
        _check(lib().mdg_nl_update(self.h, 1 if force else 0, _ip(out)))
        return out

    def nl_pairs(self, list_id: int) -> np.ndarray:
        cnt = ctypes.c_int64()
        _check(lib().mdg_nl_pairs(self.h, list_id, None, 0, ctypes.byref(cnt)))
        out = np.zeros((max(cnt.value, 1), 2), dtype=np.int32)
        _check(lib().mdg_nl_pairs(self.h, list_id, _ip(out), cnt.value, ctypes.byref(cnt)))
        return out[: cnt.value]

    def run(self, nsteps: int, dt: float, energies: bool = True):
        if energies:
            ep = np.zeros(nsteps)
            et = np.zeros(nsteps)
            _check(lib().mdg_run(self.h, nsteps, dt, _dp(ep), _dp(et)))
            return ep, et
        _check(lib().mdg_run(self.h, nsteps, dt, None, None))
        return None

    def sync(self):
        _check(lib().mdg_sync(self.h))

    def get_state(self):
        pos = np.zeros((self.n, 3))
        vel = np.zeros((self.n, 3))
        img = np.zeros((self.n, 3), dtype=np.int32)
        _check(lib().mdg_get_state(self.h, _dp(pos), _dp(vel), _ip(img)))
        return pos, vel, img

    def launch_count(self) -> int:
        return int(lib().mdg_launch_count(self.h))

    def step_host(self, nsteps: int, dt: float, pos: np.ndarray, vel: np.ndarray):
        """Step from a host-held state (updated in place); returns (epot, etot) per step."""
        ep = np.zeros(nsteps)
        et = np.zeros(nsteps)
        _check(lib().mdg_step_host(self.h, nsteps, dt, _dp(pos), _dp(vel), _dp(ep), _dp(et)))
        return ep, et

    # ---- parameters and the adjoint ----
    def set_param(self, pid: int, value: float):
        _check(lib().mdg_set_param(self.h, pid, float(value)))

    def get_param(self, pid: int) -> float:
        out = np.zeros(1)
        _check(lib().mdg_get_param(self.h, pid, _dp(out)))
        return float(out[0])

    def force_product(self, u, transpose: bool = True) -> dict:
        """At the current positions, for a direction u [n, 3]: J^T u (or J u
        with transpose=False; J the Jacobian of the gradient) as "ju", the
        exact energy gradient, dE/dtheta and d(u . grad)/dtheta."""
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(-1, 3)
        ju = np.zeros((self.n, 3))
        g = np.zeros((self.n, 3))
        de = np.zeros(NPARAM)
        dp = np.zeros(NPARAM)
        _check(lib().mdg_force_product(self.h, _dp(u), 1 if transpose else 0, _dp(ju), _dp(g), _dp(de), _dp(dp)))
        return {"ju": ju, "grad": g, "de_dparam": de, "dprod_dparam": dp}

    def adjoint_forward(self, nsteps: int, dt: float, checkpoint_every: int = 20):
        """Forward run with checkpoints; returns (unwrapped final positions,
        final velocities, E_pot at the final positions)."""
        pos = np.zeros((self.n, 3))
        vel = np.zeros((self.n, 3))
        ep = np.zeros(1)
        _check(lib().mdg_adjoint_forward(self.h, nsteps, dt, checkpoint_every, _dp(pos), _dp(vel), _dp(ep)))
        return pos, vel, float(ep[0])

    def adjoint_backward(self, seed_pos=None, seed_vel=None, seed_epot: float = 0.0):
        """Gradients of a loss of the last forward run's final state:
        returns (dL/dtheta [NPARAM], dL/dx0 [n, 3], dL/dv0 [n, 3])."""
        sp = None if seed_pos is None else np.ascontiguousarray(seed_pos, dtype=np.float64).reshape(-1, 3)
        sv = None if seed_vel is None else np.ascontiguousarray(seed_vel, dtype=np.float64).reshape(-1, 3)
        gp = np.zeros(NPARAM)
        gx = np.zeros((self.n, 3))
        gv = np.zeros((self.n, 3))
        _check(lib().mdg_adjoint_backward(self.h, _dp(sp), _dp(sv), float(seed_epot), _dp(gp), _dp(gx), _dp(gv)))
        return gp, gx, gv

    def set_profiling(self, on: bool):
        _check(lib().mdg_set_profiling(self.h, 1 if on else 0))

    def profile_read(self, max_kernels: int = 64):
        """{kernel name: (total ms, launches)} since profiling was switched on / last read."""
        names = ctypes.create_string_buffer(32 * max_kernels)
        ms = np.zeros(max_kernels)
        cnt = np.zeros(max_kernels, dtype=np.int64)
        nout = ctypes.c_int()
        _check(lib().mdg_profile_read(self.h, max_kernels, names, _dp(ms),
                                      cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), ctypes.byref(nout)))
        out = {}
        for k in range(min(nout.value, max_kernels)):
            nm = names.raw[32 * k: 32 * k + 32].split(b"\0", 1)[0].decode()
            out[nm] = (float(ms[k]), int(cnt[k]))
        return out
