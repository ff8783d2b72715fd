"""The N > 1 path on the CPU: bench.py runs independent replicas, one
process per GPU, whose only collectives are a barrier and the maximum of the
ranks' device times.  Here two gloo ranks exercise that plumbing, and the
reference arm runs under torchrun with two ranks (rank 0 alone works and
prints one line; the other exits 0)."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from mdtk_b200.replicas import Replicas, aggregate_rate
    r = Replicas("gloo", timeout_s=60)
    r.barrier()
    m = r.max(1.0 + 0.5 * rank)  # rank 1 is the slowest replica
    q.put((rank, m, aggregate_rate(100.0, r.world, m)))
    r.barrier()
    r.close()


def test_replicas_max_over_ranks_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(k, world, port, q)) for k in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, m, rate in out:
        assert m == 1.5
        assert rate == pytest.approx(world * 100.0 / 1.5)


def test_single_process_needs_no_process_group(monkeypatch):
    monkeypatch.setenv("WORLD_SIZE", "1")
    sys.path.insert(0, ROOT)
    from mdtk_b200.replicas import Replicas
    r = Replicas("gloo")
    assert r.dist is None and r.max(3.0) == 3.0
    r.barrier()
    r.close()


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libmdtkref.so")),
                    reason="oracle not built")
def test_reference_arm_under_torchrun_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--cpu-steps", "2", "--cpu-procs", "16", "--steps", "2",
           "--warmup", "3"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["n_gpus"] == 2
    assert d["cpu_baseline"]["cores"] == 16
    assert d["e2e"]["h2d_bytes_per_step"] == 0


def _build_headline(seed):
    sys.path.insert(0, ROOT)
    from bench import build_system
    return seed, len(build_system(seed)["z"])


def test_headline_system_builds_for_every_reference_arm_seed():
    """The reference arm gives its k-th process seed k (1..cores); each must
    build (a jammed lattice site moves to a spare one instead of raising)."""
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(8, os.cpu_count() or 1)) as pool:
        out = pool.map(_build_headline, range(1, 17))
    assert [n for _, n in out] == [43688] * 16
