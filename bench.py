#!/usr/bin/env python
"""Throughput of the MDTK per-step hot path on B200 (atom-steps/s).

Workload: FP64 AIREBO (REBO + LJ + torsion) ethane liquid, 5,461 C2H6
(43,688 atoms) at 0.55 g/cm^3 and 300 K, dt = 0.25 fs, seeded synthetic
configuration (mdtk_b200.builders.ethane_liquid).  A step is one velocity-
Verlet step of the whole system (positions, list check/rebuild, bond list,
REBO + torsion, connectivity table, LJ pairs, force gather, velocities).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mdg|reference]

N > 1 runs N independent replicas (the path does not shard: one trajectory
per GPU), launched one rank per GPU by torchrun; the device time is the max
over ranks.  `--impl reference` times the reference's own CPU code (the
oracle build of MDTK) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom-steps/s on 1 B200: FP64 plain vs FP32-mixed/batched at ≤1e-5 force err"
N_MOL = 5461
DT_FS = 0.25
BATCH_SYSTEMS = 256
BATCH_DT_FS = 0.2
TASK_MODE_NAMES = {1: "directed", 2: "per bond", 3: "lane pairs"}
WORKLOAD = (f"FP64 AIREBO ethane liquid: {N_MOL} C2H6 ({8 * N_MOL} atoms), 0.55 g/cm^3, 300 K, "
            f"dt {DT_FS} fs, reference cutoffs and 0.44 Rcut skin")


def build_system(seed: int):
    from mdtk_b200 import builders as B
    return B.ethane_liquid(N_MOL, density_g_cm3=0.55, temp_k=300.0, seed=seed)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", f"mdg_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ CPU baseline
def _oracle_sample(args):
    """One process: the reference code on the workload; returns (atoms, steps, window s, build s)."""
    seed, nsteps = args
    sys.path.insert(0, ROOT)
    from oracle import ref
    s = build_system(seed)
    r = ref.RefSystem(ref.POT_AIREBO)
    r.set_atoms(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    out = r.run(nsteps, DT_FS)
    t = out["times"]
    # t[0] execute entry, t[1 + k] start of iteration k, t[-1] return: the
    # window starts at iteration 1 (after the O(N^2) list build and the initial
    # energy evaluation of iteration 0)
    return len(s["z"]), nsteps - 1, float(t[-1] - t[2]), float(t[1] - t[0])


def cpu_baseline(procs: int, nsteps: int):
    import multiprocessing as mp
    if procs <= 1:
        res = [_oracle_sample((1, nsteps))]
    else:
        ctx = mp.get_context("spawn")
        with ctx.Pool(procs) as pool:
            res = pool.map(_oracle_sample, [(1 + k, nsteps) for k in range(procs)])
    atoms = sum(r[0] * r[1] for r in res)
    window = max(r[2] for r in res)
    return atoms / window, res


def usable_cores() -> int:
    """Host cores this process may run on: its CPU affinity, lowered to the
    cgroup's CPU quota when one is set (a container may see every core of the
    machine but be granted fewer)."""
    n = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    try:
        quota, period = open("/sys/fs/cgroup/cpu.max").read().split()[:2]
        if quota != "max":
            n = min(n, max(1, int(float(quota) / float(period))))
    except (OSError, ValueError):
        pass
    return max(1, n)


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


# ------------------------------------------------------------------ main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="mdg", choices=["mdg", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=100)
    ap.add_argument("--e2e-steps-per-call", type=int, default=10,
                    help="steps per mdg_step_host call in the end-to-end measurement")
    ap.add_argument("--cpu-steps", type=int, default=4)
    ap.add_argument("--cpu-procs", type=int, default=0,
                    help="processes of the reference arm (default: every usable host core)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--task-mode", type=int, default=0, choices=[0, 1, 2, 3],
                    help="REBO work split of the headline context: 0 autotuned, 1 directed, 2 per bond, "
                         "3 per bond on lane pairs")
    ap.add_argument("--precision-study", action="store_true",
                    help="instead of the throughput line: the FP32-mixed vs FP64 study on the 512,000-atom diamond")
    ap.add_argument("--study-steps", type=int, default=5000)
    ap.add_argument("--rows", default=None,
                    help="instead of the throughput line: only the measurements of the rows around the step "
                         "(comma-separated subset of bath,files,impacts,metal; 'all')")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        procs = args.cpu_procs if args.cpu_procs > 0 else usable_cores()
        value, res = cpu_baseline(procs, args.cpu_steps)
        line = {
            "impl": "reference", "metric": METRIC, "value": value, "unit": "atom-steps/s",
            "n_gpus": args.gpus, "steps": args.cpu_steps - 1, "warmup": 1,
            "ms_per_step": 1000.0 * max(r[2] for r in res) / (args.cpu_steps - 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": WORKLOAD, "atoms": res[0][0], "parallelism": f"{procs} processes"},
            "cpu_baseline": {"value": value, "unit": "atom-steps/s", "cores": procs, "kind": "reference",
                             "sample": (f"{procs} independent processes of the reference MDTK SimLoop (oracle build, "
                                        f"g++ -O2) on {cpu_model()}; each times iterations 1..{args.cpu_steps - 1} "
                                        f"after its O(N^2) list build ({res[0][3]:.1f} s, excluded)")},
            "e2e": {"value": value, "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return 0

    import torch
    import mdtk_b200 as M

    from mdtk_b200.replicas import Replicas, aggregate_rate
    torch.cuda.set_device(local)
    reps = Replicas("nccl")
    barrier = reps.barrier

    if args.precision_study:
        return precision_study(args, local, rank)
    if args.rows:
        s = build_system(seed=1 + rank)
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
        flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
        want = None if args.rows == "all" else set(args.rows.split(","))
        out = next_rows(M, s, local, stream, flush, None, want)
        if rank == 0:
            print(json.dumps({"rows": out}))
        reps.close()
        return 0

    s = build_system(seed=1 + rank)
    n = len(s["z"])
    ctx = M.Context(potentials=M.POT_AIREBO, device=local, task_mode=args.task_mode)
    ctx.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    # one explicit stream for the library's kernels, the L2 flush and the events
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)

    # warm-up (also builds the lists and the initial accelerations)
    ctx.run(max(args.warmup, 3), DT_FS, energies=False)
    ctx.sync()
    mode, ms_dir, ms_pair, ms_split = ctx.task_mode()
    ovl, rblocks = ctx.tuned_launch()
    tuned = {"rebo_task_mode": TASK_MODE_NAMES[mode], "eval_ms_directed": ms_dir, "eval_ms_per_bond": ms_pair,
             "eval_ms_lane_pairs": ms_split, "overlap": bool(ovl), "rebo_blocks": rblocks}

    # L2 flush buffer (the per-step working set is below the 126 MB L2)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    l0 = ctx.launch_count()
    barrier()
    torch.cuda.synchronize()
    for k in range(args.steps):
        flush.zero_()
        ev[k][0].record(stream)
        ctx.run(1, DT_FS, energies=False)
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    barrier()
    launches = ctx.launch_count() - l0
    clk = clocks.stop()
    ctx.sync()
    total_ms = sum(a.elapsed_time(b) for a, b in ev)
    total_ms = reps.max(total_ms)
    value = aggregate_rate(n * args.steps, world, total_ms * 1e-3)

    # the same steps with ordinary launches (programmatic dependent launch off), for comparison
    ctx.set_dependent_launch(False)
    ctx.run(3, DT_FS, energies=False)
    nab = min(args.steps, 100)
    torch.cuda.synchronize()
    for k in range(nab):
        flush.zero_()
        ev[k][0].record(stream)
        ctx.run(1, DT_FS, energies=False)
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    tuned["dependent_launch"] = True
    tuned["ms_per_step_ordinary_launch"] = sum(a.elapsed_time(b) for a, b in ev[:nab]) / nab
    ctx.set_dependent_launch(True)
    ctx.run(1, DT_FS, energies=False)

    # per-kernel device times over a short profiled window (same stream)
    ctx.set_profiling(True)
    prof_steps = 20
    for k in range(prof_steps):
        flush.zero_()
        ctx.run(1, DT_FS, energies=False)
    prof = ctx.profile_read()
    ctx.set_profiling(False)
    kern = {k: {"ms_per_launch": v[0] / max(v[1], 1), "launches": v[1], "share": 0.0} for k, v in prof.items()}
    ktot = sum(v[0] for v in prof.values())
    for k, v in prof.items():
        kern[k]["share"] = v[0] / ktot if ktot else 0.0
    top = max(kern, key=lambda k: kern[k]["ms_per_launch"] * kern[k]["launches"])

    # roofline of the dominant kernel: FP64-pipe bound (bond-order / LJ arithmetic)
    fp64_peak = M.pipe_peak(local, fp32=False)
    top = max((k for k in kern if k in FLOPS_PER_ATOM),
              key=lambda k: kern[k]["ms_per_launch"] * kern[k]["launches"], default=top)
    flops_per_atom = FLOPS_PER_ATOM.get(top)
    roof = None
    if flops_per_atom:
        achieved = flops_per_atom * n / (kern[top]["ms_per_launch"] * 1e-3) / 1e12
        roof = {"kernel": top, "bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak, "traffic": TRAFFIC_PER_LAUNCH.get((top, tuned["rebo_task_mode"])),
                "traffic_split": tuned["rebo_task_mode"],
                "peak_source": "measured FP64 FMA probe (mdg_pipe_peak) on this GPU",
                "flops_per_atom": flops_per_atom,
                "step": {"flops_per_atom": STEP_FLOPS_PER_ATOM,
                         "achieved": STEP_FLOPS_PER_ATOM * n / (total_ms / args.steps * 1e-3) / 1e12,
                         "frac": STEP_FLOPS_PER_ATOM * n / (total_ms / args.steps * 1e-3) / 1e12 / fp64_peak}}

    # end to end through the C ABI with host buffers (pinned): each
    # mdg_step_host call takes the state (positions, velocities) from the
    # caller's arrays, advances k steps and returns the state and every step's
    # potential and total energy.  The headline calls k = --e2e-steps-per-call
    # steps at a time; beside it, k = 1 (the state crosses PCIe every step).
    pos = torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    vel = torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    p0, v0, _ = ctx.get_state()
    pos[:] = p0
    vel[:] = v0

    def e2e_rate(k, calls):
        ctx.step_host(k, DT_FS, pos, vel)
        barrier()
        t0 = time.perf_counter()
        for _ in range(calls):
            ctx.step_host(k, DT_FS, pos, vel)
        t = reps.max(time.perf_counter() - t0)
        return world * n * k * calls / t

    kc = max(1, args.e2e_steps_per_call)
    calls = max(1, args.e2e_steps // kc)
    state_bytes = 2 * 24 * n  # [n*3] positions and velocities, FP64
    e2e = {"value": e2e_rate(kc, calls), "unit": "atom-steps/s",
           "h2d_bytes_per_step": state_bytes / kc, "d2h_bytes_per_step": state_bytes / kc + 2 * 8,
           "steps": kc * calls, "steps_per_call": kc,
           "timer": "host wall clock around mdg_step_host calls (each ends synchronised)"}
    e2e["one_step_per_call"] = {"value": e2e_rate(1, args.e2e_steps), "unit": "atom-steps/s",
                                "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes + 2 * 8,
                                "steps": args.e2e_steps}

    # FP32-mixed variant on the same workload, from the FP64 run's final state:
    # device time per step (same protocol) and its force error against the
    # FP64 path at that state
    mixed = None
    if not args.no_variants:
        p1, v1, _ = ctx.get_state()
        _, _, g64 = ctx.compute()
        mx = M.Context(potentials=M.POT_AIREBO, precision=M.PREC_FP32_MIXED, device=local)
        mx.set_system(s["z"], p1, v1, s["box"], s["pbc"], s["fixed"])
        mx.set_stream(stream.cuda_stream)
        _, _, g32 = mx.compute()
        d = g32 - g64
        rel = float(np.linalg.norm(d) / np.linalg.norm(g64))
        maxrms = float(np.abs(d).max() / np.sqrt((g64 ** 2).mean()))
        mx.run(max(args.warmup, 3), DT_FS, energies=False)
        mx.sync()
        kmix = min(args.steps, 200)
        evm = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(kmix)]
        barrier()
        torch.cuda.synchronize()
        for k in range(kmix):
            flush.zero_()
            evm[k][0].record(stream)
            mx.run(1, DT_FS, energies=False)
            evm[k][1].record(stream)
        torch.cuda.synchronize()
        barrier()
        mix_ms = sum(a.elapsed_time(b) for a, b in evm)
        mix_ms = reps.max(mix_ms)
        mixed = {"value": world * n * kmix / (mix_ms * 1e-3), "unit": "atom-steps/s", "steps": kmix,
                 "ms_per_step": mix_ms / kmix,
                 "force_err_vs_fp64": {"norm_rel": rel, "max_abs_over_rms": maxrms},
                 "scope": "FP32 bond orders (REBO, torsion) and plain LJ pairs; FP64 pair exponentials, LJ "
                          "powers and switches, b* of close non-bonded pairs, accumulation, integration"}

    # Batched variant: 256 independent cluster-impact systems of uneven size
    # (AB graphite slabs of 800-6000 atoms, lateral PBC, open z, fixed bottom
    # layer, a 13-atom C cluster at 10-100 eV), FP32-mixed AIREBO, dt 0.2 fs,
    # all systems advanced by the same launches.
    batched = None
    if not args.no_variants:
        from mdtk_b200 import builders as B
        systems = B.impact_batch(BATCH_SYSTEMS, seed=1 + 1000 * rank)
        bx = M.Context(potentials=M.POT_AIREBO, precision=M.PREC_FP32_MIXED, device=local)
        bx.set_batch(systems)
        bx.set_stream(stream.cuda_stream)
        nb_atoms = bx.n
        bx.run(max(args.warmup, 3), BATCH_DT_FS, energies=False)
        bx.sync()
        kb = min(args.steps, 50)
        evb = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(kb)]
        barrier()
        torch.cuda.synchronize()
        for k in range(kb):
            flush.zero_()
            evb[k][0].record(stream)
            bx.run(1, BATCH_DT_FS, energies=False)
            evb[k][1].record(stream)
        torch.cuda.synchronize()
        barrier()
        b_ms = sum(a.elapsed_time(b) for a, b in evb)
        b_ms = reps.max(b_ms)
        bx.sync()
        bx.set_profiling(True)
        for k in range(5):
            flush.zero_()
            bx.run(1, BATCH_DT_FS, energies=False)
        bprof = bx.profile_read()
        bx.set_profiling(False)
        btot = sum(v[0] for v in bprof.values()) or 1.0
        bkern = {k: {"ms_per_launch": v[0] / max(v[1], 1), "launches": v[1], "share": v[0] / btot}
                 for k, v in sorted(bprof.items(), key=lambda kv: -kv[1][0])[:10]}
        batched = {"value": world * nb_atoms * kb / (b_ms * 1e-3), "unit": "atom-steps/s", "steps": kb,
                   "ms_per_step": b_ms / kb, "systems": BATCH_SYSTEMS, "atoms": nb_atoms,
                   "precision": "fp32-mixed", "dt_fs": BATCH_DT_FS, "kernels": bkern,
                   "workload": "cluster impacts: AB graphite slabs 800-6000 atoms (lateral PBC, open z, fixed "
                               "bottom layer) + 13-atom C cluster at 10-100 eV, AIREBO"}
        del bx
        # the same batch in FP64 (batching without the precision change), and
        # the plain FP64 path on the same systems one at a time (a sample of
        # them, scaled by atoms): what running the impacts sequentially costs
        b64 = M.Context(potentials=M.POT_AIREBO, precision=M.PREC_FP64, device=local)
        b64.set_batch(systems)
        b64.set_stream(stream.cuda_stream)
        b64.run(max(args.warmup, 3), BATCH_DT_FS, energies=False)
        b64.sync()
        kb64 = min(args.steps, 20)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        b64_ms = 0.0
        for k in range(kb64):
            flush.zero_()
            e0.record(stream)
            b64.run(1, BATCH_DT_FS, energies=False)
            e1.record(stream)
            e1.synchronize()
            b64_ms += e0.elapsed_time(e1)
        batched["fp64_batched"] = {"value": world * nb_atoms * kb64 / (b64_ms * 1e-3), "unit": "atom-steps/s",
                                   "steps": kb64, "ms_per_step": b64_ms / kb64}
        del b64
        seq_atoms, seq_ms, nseq, kseq = 0, 0.0, 16, 20
        for sysd in systems[:nseq]:
            cx = M.Context(potentials=M.POT_AIREBO, precision=M.PREC_FP64, device=local)
            cx.set_system(sysd["z"], sysd["pos"], sysd["vel"], sysd["box"], sysd["pbc"], sysd["fixed"])
            cx.set_stream(stream.cuda_stream)
            cx.run(max(args.warmup, 3), BATCH_DT_FS, energies=False)
            cx.sync()
            flush.zero_()
            e0.record(stream)
            cx.run(kseq, BATCH_DT_FS, energies=False)
            e1.record(stream)
            e1.synchronize()
            seq_ms += e0.elapsed_time(e1)
            seq_atoms += len(sysd["z"]) * kseq
            del cx
        batched["fp64_sequential"] = {
            "value": world * seq_atoms / (seq_ms * 1e-3), "unit": "atom-steps/s",
            "sample": f"first {nseq} of the {BATCH_SYSTEMS} systems, one context each, {kseq} steps each "
                      f"(graph-replayed), run one after another"}

    # Adjoint variant: gradients of a 200-step trajectory loss with respect to
    # the six C-C pair parameters, x0 and v0 (4,096-atom amorphous carbon at
    # 2.0 g/cm^3, pre-relaxed 500 steps at 3,000 K, dt 0.5 fs, checkpoint every
    # 20 steps, loss = mean |x_200 - x_target|^2 + 1e-5 E_total), FP64
    adjoint = None
    if not args.no_variants:
        from mdtk_b200 import builders as B
        a0 = B.amorphous_carbon(ADJ_ATOMS, density_g_cm3=2.0, min_sep=1.2, seed=81 + rank)
        a5 = B.relax_hot(a0, 500, 3000.0, ADJ_DT_FS, M.POT_AIREBO, seed=82 + rank, device=local)
        ax = M.Context(potentials=M.POT_AIREBO, device=local, task_mode=1)
        ax.set_system(a5["z"], a5["pos"], a5["vel"], a5["box"], a5["pbc"], a5["fixed"])
        ax.set_stream(stream.cuda_stream)
        m = B.masses(a5["z"])[:, None]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

        def grad_once():
            ax.set_state(a5["pos"], a5["vel"])
            e0.record(stream)
            t0 = time.perf_counter()
            xN, vN, _ = ax.adjoint_forward(ADJ_STEPS, ADJ_DT_FS, ADJ_EVERY)
            e1.record(stream)
            t1 = time.perf_counter()
            e1.synchronize()
            fwd_ms = e0.elapsed_time(e1)
            target = xN + 0.01 * np.random.default_rng(83).normal(size=xN.shape)
            sx = 2.0 * (xN - target) / ADJ_ATOMS
            sv = 1e-5 * m * vN / B.EV_PER_AMU_A2FS2
            e0.record(stream)
            t2 = time.perf_counter()
            gp, _, _ = ax.adjoint_backward(sx, sv, 1e-5)
            e1.record(stream)
            t3 = time.perf_counter()
            e1.synchronize()
            return fwd_ms, e0.elapsed_time(e1), (t1 - t0) * 1e3, (t3 - t2) * 1e3, gp

        grad_once()  # buffers, lists, warm-up
        fwd_ms, bwd_ms, fwd_wall, bwd_wall, gp = grad_once()
        ax.set_state(a5["pos"], a5["vel"])
        ax.run(3, ADJ_DT_FS, energies=False)
        ax.sync()
        e0.record(stream)
        ax.run(ADJ_STEPS, ADJ_DT_FS, energies=False)
        e1.record(stream)
        e1.synchronize()
        plain_ms = e0.elapsed_time(e1)
        adjoint = {
            "value": world * ADJ_ATOMS * ADJ_STEPS / ((fwd_ms + bwd_ms) * 1e-3), "unit": "atom-steps/s (gradient)",
            "forward_ms": fwd_ms, "backward_ms": bwd_ms, "forward_wall_ms": fwd_wall, "backward_wall_ms": bwd_wall,
            "plain_fp64_run_ms": plain_ms, "gradient_over_plain": (fwd_ms + bwd_ms) / plain_ms,
            "grad_params": dict(zip(M.PARAM_NAMES, [float(x) for x in gp])),
            "workload": f"{ADJ_ATOMS} C amorphous 2.0 g/cm^3, pre-relaxed 500 steps at 3000 K, {ADJ_STEPS} steps "
                        f"dt {ADJ_DT_FS} fs, checkpoint every {ADJ_EVERY}, AIREBO FP64; gradients w.r.t. eps, "
                        f"sigma, A, B1, alpha, beta1 (C-C), x0, v0",
            "timer": "CUDA events on the library stream around each (host-driven) call"}
        del ax

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "atoms": n, "potentials": "REBO+LJ+ETors", "precision": "fp64",
                       "l2": "flushed between timed steps (256 MiB write, outside the timed events)",
                       "parallelism": f"replicas x{world}"},
            "gpu_launches": launches, "clocks": clk, "kernels": kern, "roofline": roof, "e2e": e2e,
            "autotuner": tuned,
            "fp64_peak_tflops": fp64_peak,
            "variants": {"fp32_mixed": mixed, "batched": batched, "adjoint": adjoint},
        }
        if world == 1 and not args.no_variants:
            line["variants"]["next_rows"] = next_rows(M, s, local, stream, flush, value)
        if world == 1 and not args.no_cpu_baseline:
            try:
                v, res = cpu_baseline(1, args.cpu_steps)
                line["cpu_baseline"] = {
                    "value": v, "unit": "atom-steps/s", "cores": 1, "kind": "reference",
                    "sample": (f"reference MDTK SimLoop (oracle build, g++ -O2, single-threaded) on {cpu_model()}: "
                               f"iterations 1..{args.cpu_steps - 1} of the same workload after its O(N^2) list "
                               f"build ({res[0][3]:.1f} s, excluded)")}
            except Exception as e:  # the oracle is test infrastructure; its absence is reported, not fatal
                line["cpu_baseline"] = {"value": None, "unit": "atom-steps/s", "cores": 1, "kind": "reference",
                                        "sample": f"unavailable: {e}"}
        print(json.dumps(line))
    reps.close()
    return 0


ADJ_ATOMS, ADJ_STEPS, ADJ_DT_FS, ADJ_EVERY = 4096, 200, 0.5, 20


def next_rows(M, s, local, stream, flush, plain_rate, want=None):
    """Throughput of the rows around the step, one GPU:

    * SimLoop's thermal bath (universe, 300 K, 1e13 / s) with adaptive dt on
      the headline ethane liquid;
    * the same liquid writing its files from device snapshots, at
      mdtrajsim's intervals and at ten times their frequency (wall clock, the
      files included);
    * mdtrajsim's impact sequence: 64 impacts of a C projectile on a 256-atom
      graphite slab to 20 fs, one batched context with the application's
      files, against the unmodified mdtrajsim application on the host for
      one impact;
    * metal and ion potentials: ethane molecules and an Ar ion above an
      18,432-atom Cu slab (AIREBO + FBZL + FLJ + Ackland), against the
      reference's own classes on the host (3 steps).
    CUDA events on the library stream unless said otherwise."""
    import torch
    out = {}
    n = len(s["z"])
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(c, k, dt):
        flush.zero_()
        e0.record(stream)
        c.run(k, dt, energies=False)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    def on(name):
        return want is None or name in want

    def rel(v):
        return v / plain_rate if plain_rate else None

    # thermal bath + adaptive dt
    if on("bath"):
        _row_bath(M, s, local, stream, timed, n, out, rel)
    if on("files"):
        _row_files(M, s, local, stream, n, out, rel)
    if on("impacts"):
        _row_impacts(M, local, out)
    if on("metal"):
        _row_metal(M, local, stream, timed, out)
    return out


def _row_bath(M, s, local, stream, timed, n, out, rel):
    c = M.Context(potentials=M.POT_AIREBO, device=local)
    c.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    c.set_stream(stream.cuda_stream)
    c.set_thermal_bath(M.TB_UNIVERSE, 300.0, 1e13 * 1e-15)
    c.set_adaptive_dt(True, 1.0, DT_FS)
    c.run(3, DT_FS, energies=False)
    c.sync()
    ms = timed(c, 100, DT_FS)
    out["bath_adaptive_dt"] = {"value": n * 100 / (ms * 1e-3), "unit": "atom-steps/s", "steps": 100,
                               "over_plain": rel(n * 100 / (ms * 1e-3)),
                               "workload": "headline liquid, universe bath 300 K, gamma 1e13/s, adaptive dt"}
    del c


def _row_files(M, s, local, stream, n, out, rel):
    import shutil
    import tempfile
    tmp = tempfile.mkdtemp(prefix="mdg_out_")
    try:
        c = M.Context(potentials=M.POT_AIREBO, device=local)
        c.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
        c.set_stream(stream.cuda_stream)
        c.run(3, DT_FS, energies=False)
        c.sync()
        for flush_it, traj_fs, label in ((1000, 100.0, "mdtrajsim's intervals: state every 1000 iterations, "
                                                       "XVA every 0.1 ps (400 steps)"),
                                         (100, 10.0, "state every 100 iterations, XVA every 10 fs (40 steps)")):
            c.set_output(os.path.join(tmp, str(flush_it)), flush_it, traj_fs)
            t0 = time.perf_counter()
            c.run(2000, DT_FS, energies=False)
            c.flush_output()
            wall = time.perf_counter() - t0
            c.set_output(None)
            nfiles = len(os.listdir(os.path.join(tmp, str(flush_it))))
            out["files_every_%d" % flush_it] = {
                "value": n * 2000 / wall, "unit": "atom-steps/s (wall clock, files written)", "steps": 2000,
                "files": nfiles, "over_plain": rel(n * 2000 / wall),
                "workload": "headline liquid, " + label}
        del c
    finally:
        shutil.rmtree(tmp, ignore_errors=True)



def _row_impacts(M, local, out):
    import shutil
    import tempfile
    from mdtk_b200 import builders as B
    from mdtk_b200 import trajsim as T
    tmp = tempfile.mkdtemp(prefix="mdg_traj_")
    try:
        slab = B.graphite_slab(2, 8, 4, temp_k=0.0, seed=3)
        top = slab["pos"][:, 2].max()
        base = B.add_atoms(slab, [6], [[slab["box"][0] / 2, slab["box"][1] / 2, top + 3.0]], vel=[[0, 0, -0.04]])
        nb = len(base["z"])
        bc = M.Context(potentials=M.POT_AIREBO | M.POT_METAL, device=local)
        bc.set_system(base["z"], base["pos"], base["vel"], base["box"], (1, 1, 0), base["fixed"])
        tags = np.full(nb, M.TAG_TARGET, np.uint8)
        tags[-1] = M.TAG_PROJECTILE
        bc.set_atom_tags(tags)
        bc.set_adaptive_dt(True, 1.0, 0.2)
        bc.set_time_final(20.0)
        bc.write_state(os.path.join(tmp, "base"))
        del bc
        rng = np.random.default_rng(7)
        nimp = 64
        xy = np.stack([rng.uniform(0, base["box"][0], nimp), rng.uniform(0, base["box"][1], nimp)], 1) * 1e-8
        xy.tofile(os.path.join(tmp, "ionpos.bin"))
        t0 = time.perf_counter()
        T.impact_sequence(os.path.join(tmp, "base"), os.path.join(tmp, "ionpos.bin"), os.path.join(tmp, "dev"),
                          batch=nimp, task_mode=1)
        wall = time.perf_counter() - t0
        iters = []
        for k in range(nimp):
            d = os.path.join(tmp, "dev", "%08d" % k)
            iters += [int(f[2:12]) for f in os.listdir(d) if f.startswith("md") and f.endswith(".r")]
        row = {"value": nimp / wall, "unit": "impacts/s (wall clock, files included)", "impacts": nimp,
               "atoms_per_impact": nb, "atom_steps_per_s": nb * sum(iters) / wall,
               "workload": f"C projectile on a {nb - 1}-atom graphite slab (2 layers) to 20 fs, adaptive dt, "
                           "application potential set, one batched context"}
        # what a persistent fused step could save at most: the floor of a
        # step's 24 dependent phases as graph launches and as one cooperative
        # kernel, beside the wall time per step of this batch
        g_us, c_us = M.launch_floor(local, 24)
        row["per_step"] = {"wall_us": 1e6 * wall / max(iters), "steps": max(iters),
                           "launch_floor_graph_us": g_us, "launch_floor_cooperative_us": c_us, "phases": 24}
        app = os.path.join(ROOT, "oracle", "_ref", "mdtrajsim")
        if os.path.exists(app):
            rd = os.path.join(tmp, "ref")
            os.makedirs(rd)
            for f in os.listdir(tmp):
                if f.startswith("base.") or f == "ionpos.bin":
                    shutil.copy(os.path.join(tmp, f), rd)
            xy[:1].tofile(os.path.join(rd, "ionpos.bin"))
            t0 = time.perf_counter()
            subprocess.run([app, "base", "-i", "0"], cwd=rd, capture_output=True, check=True)
            cw = time.perf_counter() - t0
            row["cpu_baseline"] = {"value": 1.0 / cw, "unit": "impacts/s", "cores": 1, "kind": "reference",
                                   "sample": "the unmodified mdtrajsim application (oracle build) on one impact "
                                             "of the same sequence"}
        out["impact_sequence"] = row
    finally:
        shutil.rmtree(tmp, ignore_errors=True)



def _row_metal(M, local, stream, timed, out):
    from mdtk_b200 import builders as B
    cu = B.fcc(29, 24, 24, 8, pbc=(1, 1, 0), temp_k=300.0, seed=9)
    top = cu["pos"][:, 2].max()
    mol = B.c2h6_example()
    zs, ps = [], []
    for i in range(10):
        for j in range(10):
            zs.append(mol["z"])
            ps.append(mol["pos"] - mol["pos"].mean(axis=0) + [4.0 + 8.5 * i, 4.0 + 8.5 * j, top + 3.0])
    zs.append(np.array([18], np.int32))
    ps.append(np.array([[40.0, 40.0, top + 8.0]]))
    ms_sys = B.add_atoms(cu, np.concatenate(zs), np.concatenate(ps))
    ms_sys["vel"][-1] = [0.0, 0.0, -0.05]
    nm = len(ms_sys["z"])
    c = M.Context(potentials=M.POT_AIREBO | M.POT_METAL, device=local)
    c.set_system(ms_sys["z"], ms_sys["pos"], ms_sys["vel"], ms_sys["box"], ms_sys["pbc"], ms_sys["fixed"])
    c.set_stream(stream.cuda_stream)
    c.run(3, DT_FS, energies=False)
    c.sync()
    ms = timed(c, 100, DT_FS)
    c.set_profiling(True)
    for _ in range(5):
        c.run(1, DT_FS, energies=False)
    prof = c.profile_read()
    c.set_profiling(False)
    ptot = sum(v[0] for v in prof.values()) or 1.0
    mkern = {k: {"ms_per_launch": v[0] / max(v[1], 1), "share": v[0] / ptot}
             for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])[:8]}
    row = {"value": nm * 100 / (ms * 1e-3), "unit": "atom-steps/s", "steps": 100, "atoms": nm, "kernels": mkern,
           "workload": f"{len(cu['z'])} Cu (fcc slab), 100 ethane molecules, an Ar ion; AIREBO + FBZL + FLJ + Ackland, FP64"}
    del c
    try:
        from oracle import ref
        r = ref.RefSystem(ref.POT_AIREBO | ref.POT_METAL)
        r.set_atoms(ms_sys["z"], ms_sys["pos"], ms_sys["vel"], ms_sys["box"], ms_sys["pbc"], ms_sys["fixed"])
        res = r.run(3, DT_FS)
        ts = res["times"]
        step_s = (ts[-1] - ts[2]) / 2.0  # iterations 1 and 2, after the list build of iteration 0
        row["cpu_baseline"] = {"value": nm / step_s, "unit": "atom-steps/s", "cores": 1, "kind": "reference",
                               "sample": "the reference's FBZL, FLJ, REBO, AIREBO, ETors, Ackland (oracle build), "
                                         "iterations 1..2 of the same system"}
    except Exception as e:  # the oracle is test infrastructure; its absence is reported, not fatal
        row["cpu_baseline"] = {"value": None, "sample": f"unavailable: {e}"}
    out["metal_ion"] = row

# 512,000-atom diamond of the precision study (40^3 cells, a = 3.567 A,
# Gaussian displacements sigma 0.05 A, 600 K, dt 0.5 fs)
STUDY_CELLS, STUDY_DT_FS = 40, 0.5


def precision_study(args, local, rank):
    """FP32-mixed against FP64 on the 512,000-atom diamond: force and energy
    error at the start, device time per step of each, and the NVE drift and
    fluctuation of each over --study-steps steps.  Prints one JSON line."""
    import torch
    import mdtk_b200 as M
    from mdtk_b200 import builders as B
    torch.cuda.set_device(local)
    s = B.diamond(STUDY_CELLS, temp_k=600.0, disp_sigma=0.05, seed=7 + rank)
    n = len(s["z"])
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    out = {"study": "precision", "atoms": n, "steps": args.study_steps, "dt_fs": STUDY_DT_FS,
           "workload": f"diamond {STUDY_CELLS}^3 cells ({n} C), Gaussian displacements 0.05 A, 600 K, AIREBO"}
    ctxs, grads, energies = {}, {}, {}
    for name, prec in (("fp64", M.PREC_FP64), ("fp32_mixed", M.PREC_FP32_MIXED)):
        c = M.Context(potentials=M.POT_AIREBO, precision=prec, device=local)
        c.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
        c.set_stream(stream.cuda_stream)
        e, et, g = c.compute()
        ctxs[name], grads[name], energies[name] = c, g, (e, et)
    d = grads["fp32_mixed"] - grads["fp64"]
    out["force_err"] = {"norm_rel": float(np.linalg.norm(d) / np.linalg.norm(grads["fp64"])),
                        "max_abs_over_rms": float(np.abs(d).max() / np.sqrt((grads["fp64"] ** 2).mean()))}
    out["energy_err_rel"] = abs(energies["fp32_mixed"][0] - energies["fp64"][0]) / abs(energies["fp64"][0])
    out["energy_terms"] = {k: [float(x) for x in v[1][:3]] for k, v in energies.items()}
    for name, c in ctxs.items():
        c.run(3, STUDY_DT_FS, energies=False)
        c.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        c.run(50, STUDY_DT_FS, energies=False)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / 50
        c.set_state(s["pos"], s["vel"])
        t0 = time.perf_counter()
        _, etot = c.run(args.study_steps, STUDY_DT_FS)
        wall = time.perf_counter() - t0
        k0 = max(1, len(etot) // 100)
        e = np.asarray(etot[k0:]) / n
        t = (np.arange(k0, len(etot)) + 1) * STUDY_DT_FS * 1e-3
        a, b = np.polyfit(t, e, 1)
        out[name] = {"ms_per_step": ms, "atom_steps_per_s": n / (ms * 1e-3),
                     "nve_drift_ev_per_atom_per_ps": float(a),
                     "nve_rms_fluct_ev_per_atom": float(np.sqrt(np.mean((e - (a * t + b)) ** 2))),
                     "e_total_first_last_ev_per_atom": [float(etot[0] / n), float(etot[-1] / n)],
                     "run_wall_s": wall}
    out["speedup_mixed_over_fp64"] = out["fp64"]["ms_per_step"] / out["fp32_mixed"]["ms_per_step"]
    if rank == 0:
        print(json.dumps(out))
    return 0


# Algorithmic FP64 flops per atom for one launch of each kernel on this
# workload (ethane liquid, 43,688 atoms, step-0 state, seed 1), from the
# op-counting restatement: `python oracle/opcount.py` (add/mul 1, div/sqrt 4,
# exp/cos 12, pow 24; energy + gradient = 3 x energy).  rebo_tors = REBO +
# torsion terms; lj_pairs = the plain LJ pair terms (V_LJ, switches, C_ij
# path products); lj_special = the b*_ij bond orders of close non-bonded pairs.
FLOPS_PER_ATOM = {"rebo_tors": 2541.0 + 504.0, "lj_pairs": 5151.5, "lj_special": 5205.5}
STEP_FLOPS_PER_ATOM = 2541.0 + 504.0 + 10357.0
# DRAM read + write bytes per launch of each kernel on this workload, from
# one ncu capture of the kernel (profiles/, captured with
#   ncu --set full --clock-control none -k regex:<kernel> -c <few> ...
# on one GPU), keyed by the REBO work split the timed step ran (the
# autotuner's choice: "per bond", "directed" or "lane pairs"); None when not
# captured.
TRAFFIC_PER_LAUNCH = {
    ("rebo_tors", "per bond"): 10.88e6, ("rebo_tors", "directed"): 22.83e6,
    ("rebo_tors", "lane pairs"): 13.6e6,
}


if __name__ == "__main__":
    sys.exit(main())
