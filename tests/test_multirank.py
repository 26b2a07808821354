"""Multi-rank plumbing of bench.py on the host (gloo, world size 2): the
max-over-ranks reduction of the window time, the barrier, and the
reference arm under torchrun (rank 0 alone runs and prints one line)."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    ws, r, local, dist = bench.dist_init()
    assert ws == 2 and r == rank and dist is not None
    bench.barrier(dist)
    m = bench.allmax(dist, 1.5 + rank)
    bench.barrier(dist)
    dist.destroy_process_group()
    with open(out % rank, "w") as fh:
        fh.write(repr(m))


def test_allmax_over_two_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    out = str(tmp_path / "r%d.txt")
    mp.spawn(_rank_main, args=(port, out), nprocs=2, join=True)
    assert [float(open(out % r).read()) for r in (0, 1)] == [2.5, 2.5]


@pytest.mark.timeout(600)
def test_reference_arm_two_ranks():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref
    if not ref.build():
        pytest.skip("reference not built and its sources are absent")
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--workload", "pour", "--particles", "2000", "--steps", "3", "--warmup", "1",
           "--gpus", "2"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["steps"] == 3 and d["warmup"] == 3
