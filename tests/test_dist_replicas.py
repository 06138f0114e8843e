"""Multi-process (world size 2, gloo, CPU) checks of the replica path of
bench.py: the max-over-ranks timing reduction, and the reference arm under
torch.distributed.run, where rank 0 alone runs and prints one JSON line and
the other rank exits 0 without work."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out[rank] = bench.max_over_ranks(10.0 + 5.0 * rank, dist)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(2, port, out), nprocs=2, join=True)
        assert out[0] == 15.0 and out[1] == 15.0


def test_max_over_ranks_without_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5) == 3.5


def test_reference_arm_two_ranks_prints_one_line():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--size", "4", "--steps", "1", "--warmup", "1"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["value"] > 0 and rec["cpu_baseline"]["kind"] == "port"
    assert rec["e2e"]["h2d_bytes_per_step"] == 0
