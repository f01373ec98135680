"""The multi-rank plumbing of bench.py on the CPU: world-size-2 `gloo` ranks for the
max-over-ranks timing and the barrier, and the reference arm launched as a multi-GPU
run is launched (torch.distributed.run, one process per rank), where rank 0 alone
times the host path and prints the one JSON line.  Multi-GPU is replicas only:
no collective touches the data path, so these are all the collectives there are."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch
    import bench
    dist = bench.dist_init("gloo")
    # each rank "measured" a different time; the reported one is the slowest
    ms = bench.reduce_max(10.0 * (rank + 1), torch.device("cpu"), world)
    bench.barrier(world)
    out.put((rank, ms, bench.dist_env()))
    dist.destroy_process_group()


def test_max_over_gloo_ranks_and_barrier():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [20.0, 20.0]
    assert [r[2] for r in res] == [(0, 2, 0), (1, 2, 1)]


def test_reduce_max_is_identity_for_one_rank():
    sys.path.insert(0, ROOT)
    import torch
    import bench
    assert bench.reduce_max(3.5, torch.device("cpu"), 1) == 3.5


def test_reference_arm_under_torchrun_prints_one_line():
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "0", "--cells", "1500"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
