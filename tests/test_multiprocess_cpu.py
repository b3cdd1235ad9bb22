"""The multi-process (replica) path of bench.py on CPU: world_size 2 over
gloo.  Each rank runs its own replica; timing takes the maximum over ranks
and the value aggregates the units of all ranks; the reference arm runs on
rank 0 only and prints one JSON line."""
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
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = 10.0 + 5.0 * rank  # this rank's timed region
    slowest = bench.max_over_ranks(ms, dist)
    value = bench.aggregate_rate(world, 1000.0, slowest)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, slowest, value))


def test_max_over_ranks_and_aggregate_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slowest, value in res:
        assert slowest == 15.0  # the slower rank's time on every rank
        assert value == pytest.approx(2 * 1000.0 / 0.015)


def test_reference_arm_rank0_only_under_torchrun():
    port = _free_port()
    cmd = [
        sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
        "--master-addr", "127.0.0.1", "--master-port", str(port),
        os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1",
        "--h", "0.015625",
    ]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port"
