"""The multi-rank plumbing of bench.py on CPU: one process per rank over
gloo, as torchrun launches them (replicas only: the path has no data
exchange, so the process group carries the barriers and the max / sum of
the timings). No device is used."""

import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    r = bench.Ranks()
    r.barrier()
    mx = r.max(float(rank + 1))
    sm = r.sum(10.0)
    r.close()
    out.put((rank, mx, sm))


def test_ranks_reduce_over_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == [(0, 2.0, 20.0), (1, 2.0, 20.0)]


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_build", "liboracle.so")),
                    reason="the oracle is not built")
def test_reference_arm_under_two_ranks():
    """Rank 0 alone times the reference CPU path and prints one line; rank 1
    exits 0 without work."""
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py",
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
           "--batch", "2"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["cores"] >= 1
    # the arm runs the reference's code alone: nothing of the product mapped
    assert d["config"]["frames_per_step"] == 2
    assert not any("spotfinder_b200" in lib for lib in d["mapped_libraries"])
