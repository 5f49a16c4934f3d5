"""The multi-rank path of bench.py on CPU (gloo, world size 2): replicas share no
data, so what N > 1 adds is the barrier, the max-over-ranks timing and rank 0
alone printing the reference arm's line."""
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


def _rank_main(rank, world, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank), "WORLD_SIZE": str(world),
                       "LOCAL_RANK": str(rank), "AZK_DIST_BACKEND": "gloo"})
    sys.path.insert(0, ROOT)
    import bench

    w, r, local, dist = bench.dist_setup(None)
    bench.barrier(dist)
    out.put((r, w, bench.max_over_ranks(dist, 1.5 + r, local)))
    dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == [(0, 2, 2.5), (1, 2, 2.5)]


@pytest.mark.slow
def test_reference_arm_prints_once_under_torchrun():
    env = dict(os.environ, AZK_DIST_BACKEND="gloo", OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
           "--master-port", str(_free_port()), "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0", "--instances", "4",
           "--cpu-max-log", "11"]  # the workload's first instance is log 10
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    assert lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2 and lines[0]["value"] > 0
