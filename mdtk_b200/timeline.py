"""Per-kernel timeline of graph-replayed steps of the headline liquid, from
the timeline build of the library (pdl_enter() stamps the global timer):
when each kernel's first block started, when it passed its dependency wait
and when its last warp left, relative to the step's first kernel.  Kernels
are named by the source line of their pdl_enter() in mdg_api.cu; two
launches of one kernel in a step (the two record-sum halves, the cell
kernels of two lists) share a row, from the first start to the last end.

    python -m mdtk_b200.build --timeline
    python -m mdtk_b200.timeline [--task-mode M] [--steps K] [--no-flush]
"""
from __future__ import annotations

import argparse
import ctypes
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SLOTS = 8192


def kernel_names() -> dict:
    """Source line of each pdl_enter() in mdg_api.cu -> the kernel it opens."""
    names, cur = {}, "?"
    pat = re.compile(r"__global__ void (?:__launch_bounds__\([^)]*\) )?(\w+)")
    for ln, text in enumerate(open(os.path.join(HERE, "csrc", "mdg_api.cu")), start=1):
        m = pat.search(text)
        if m:
            cur = m.group(1)
        if "pdl_enter();" in text:
            names[ln % SLOTS] = cur
    return names


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--task-mode", type=int, default=0)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--no-flush", action="store_true")
    args = ap.parse_args(argv)
    sys.path.insert(0, ROOT)
    import torch
    import mdtk_b200 as M
    M.LIB_PATH = os.path.join(HERE, "libmdg_timeline.so")
    if not os.path.exists(M.LIB_PATH):
        raise SystemExit("build the timeline library first: python -m mdtk_b200.build --timeline")
    import bench
    L = M.lib()
    u64p = ctypes.POINTER(ctypes.c_uint64)
    L.mdg_timeline_read.argtypes = [u64p, u64p, u64p, ctypes.c_int]
    names = kernel_names()
    s = bench.build_system(1)
    c = M.Context(potentials=M.POT_AIREBO, task_mode=args.task_mode)
    c.set_system(s["z"], s["pos"], s["vel"], s["box"], s["pbc"], s["fixed"])
    st = torch.cuda.Stream()
    torch.cuda.set_stream(st)
    c.set_stream(st.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    c.run(5, bench.DT_FS, energies=False)
    c.sync()
    print(f"task mode {c.task_mode()[0]}, launch (overlap, REBO blocks) {c.tuned_launch()}, "
          f"L2 {'kept' if args.no_flush else 'flushed'} before each step")
    for k in range(args.steps):
        torch.cuda.synchronize()
        if L.mdg_timeline_reset():
            raise SystemExit(L.mdg_last_error().decode())
        if not args.no_flush:
            flush.zero_()
        torch.cuda.synchronize()
        c.run(1, bench.DT_FS, energies=False)
        c.sync()
        t = [np.zeros(SLOTS, np.uint64) for _ in range(3)]
        if L.mdg_timeline_read(*[a.ctypes.data_as(u64p) for a in t], SLOTS):
            raise SystemExit(L.mdg_last_error().decode())
        start, wait, end = (a.astype(np.int64) for a in t)
        ids = [i for i in range(SLOTS) if end[i] > 0]
        t0, t1 = min(start[i] for i in ids), max(end[i] for i in ids)
        print(f"step {k}: {1e-3 * (t1 - t0):.1f} us (first kernel start to last kernel end)")
        print(f"  {'kernel':26s} {'start':>8s} {'waited':>8s} {'end':>8s} {'run us':>8s}")
        for i in sorted(ids, key=lambda i: start[i]):
            print(f"  {names.get(i, '?'):26s} {1e-3 * (start[i] - t0):8.1f} {1e-3 * (wait[i] - t0):8.1f} "
                  f"{1e-3 * (end[i] - t0):8.1f} {1e-3 * (end[i] - wait[i]):8.1f}")
    c.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
