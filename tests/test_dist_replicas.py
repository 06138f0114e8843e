"""Multi-process (world size 2, gloo, CPU) checks of the replica path of
bench.py: the max-over-ranks timing reduction; two ranks that evolve distinct
seeded ensemble members through bench.py's own timed region, with the oracle
as the step; and the reference arm under torch.distributed.run (launched by
the caller or by bench.py itself), where rank 0 alone runs and prints one
JSON line and the other rank exits 0 without work."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
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
    assert rec["e2e"]["h2d_bytes_per_step"] == 0 and rec["n_gpus"] == 2


N4, A4 = (4, 4, 4), (0.05, 1.0, 1.0, 1.0)


def _member(seed):
    """The initial fields of one ensemble member at 4^3."""
    from oracle import oracle as oc
    links, ef = oc.transverse_box(N4, A4, 3.0, 1.0, 0.0, seed, identity_links=True)
    q, a = oc.single_point(N4, 1), oc.single_point(N4, 1)
    return links, ef, q, a


def _replica_rank(rank, world, port, out):
    import datetime
    import time

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    from oracle import oracle as oc
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        links, ef, q, a = _member(bench.member_seed(rank))

        def step():
            oc.cn_update(N4, A4, links, ef, 1.0, [1, 1, 1, 1], 1.0, q, a, tol=1e-13)
            oc.gauge_update(N4, A4, links, ef, 1.0)
            if rank == 1:
                time.sleep(0.05)  # the slower rank sets the job's time

        class WallTimer:
            def start(self):
                self.t0 = time.perf_counter()

            def stop(self):
                return 1000.0 * (time.perf_counter() - self.t0)

        steps = 3
        ms = bench.timed_steps(step, steps, dist, WallTimer())
        out[rank] = {"ms": ms, "value": bench.whole_job_rate(world, 64, steps, ms),
                     "energy": oc.energy(N4, A4, links, ef), "q": q.copy(), "seed": bench.member_seed(rank)}
    finally:
        dist.destroy_process_group()


def test_two_ranks_evolve_distinct_members_and_sum_the_rate(oracle):
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_replica_rank, args=(2, port, out), nprocs=2, join=True)
        r0, r1 = dict(out[0]), dict(out[1])
    # both ranks report the slowest rank's time, at least the planted delay
    assert r0["ms"] == r1["ms"] and r0["ms"] >= 3 * 50.0
    # the whole job's rate counts both lattices in that time
    assert abs(r0["value"] - 2 * 64 * 3 / (r0["ms"] / 1000.0)) <= 1e-9 * r0["value"]
    # distinct seeds, distinct members, each equal to a single-process run
    assert (r0["seed"], r1["seed"]) == (1, 2)
    assert abs(r0["energy"] - r1["energy"]) > 1e-6 * abs(r0["energy"])
    for r in (r0, r1):
        links, ef, q, a = _member(r["seed"])
        for _ in range(3):
            oracle.cn_update(N4, A4, links, ef, 1.0, [1, 1, 1, 1], 1.0, q, a, tol=1e-13)
            oracle.gauge_update(N4, A4, links, ef, 1.0)
        assert abs(oracle.energy(N4, A4, links, ef) - r["energy"]) <= 1e-12 * abs(r["energy"])
        assert np.abs(q - r["q"]).max() <= 1e-13


def test_reference_arm_launches_its_own_ranks():
    """`bench.py --gpus 2` without a launcher starts the two ranks itself and
    reports n_gpus 2, as the launcher-started run does."""
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--size", "4",
           "--steps", "1", "--warmup", "1"]
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2
