"""Build libmdg.so in-tree for sm_100a (nvcc cross-compiles without a GPU).

    python -m mdtk_b200.build
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libmdg.so")
# the per-kernel timeline build (MDG_TIMELINE: pdl_enter() stamps the global
# timer; see mdtk_b200/timeline.py), a separate library never loaded by default
OUT_TIMELINE = os.path.join(HERE, "libmdg_timeline.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-O2",
    "-diag-suppress", "177",
]


def sources():
    return [os.path.join(CSRC, f) for f in ("mdg_api.cu", "mdg_noalloc.cu", "mdg_tables.cpp")]


def headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + [
        os.path.join(ROOT, "include", "mdg.h")]


def up_to_date(out: str = OUT) -> bool:
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(f) <= t for f in sources() + headers())


def build(force: bool = False, verbose: bool = False, timeline: bool = False) -> str:
    out = OUT_TIMELINE if timeline else OUT
    if not force and up_to_date(out):
        return out
    nvcc = os.environ.get("NVCC", "nvcc")
    extra = ["-DMDG_TIMELINE"] if timeline else []
    cmd = [nvcc, *NVCC_FLAGS, *extra, "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-shared", *sources(), "-lz",
           "-o", out]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libmdg.so")
    if verbose:
        sys.stderr.write(r.stderr)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv, timeline="--timeline" in sys.argv))
