"""The N > 1 path of bench.py on CPU: two gloo ranks (one process per GPU in
the real run, independent replicas, no data-path collective).  Checks the
max-over-ranks device time, the whole-job throughput built on it, and that
the reference arm runs on rank 0 only."""
import argparse
import io
import os
import sys
from contextlib import redirect_stdout

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _worker(rank, world, port, out):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = 10.0 * (rank + 1)          # rank 1 is the slower replica
        m = bench.max_over_ranks(local_ms, world, "cpu")
        value = bench.job_throughput(world * 4, m)   # 4 solves per rank
        dist.barrier()
        out[rank] = (m, value)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_throughput_gloo():
    world = 2
    port = 29000 + os.getpid() % 1000
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 20.0      # both ranks see the slowest time
    assert abs(res[0][1] - 8 / 0.020) < 1e-9   # 8 solves in 20 ms
    assert res[0] == res[1]


def test_single_process_keeps_its_own_time():
    import bench
    assert bench.max_over_ranks(7.5, 1, "cpu") == 7.5
    assert bench.job_throughput(3, 1500.0) == 2.0


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    import bench
    monkeypatch.setenv("RANK", "1")
    args = argparse.Namespace(workload="helmholtz_fp64_128", steps=1, warmup=0, ref_procs=1)
    buf = io.StringIO()
    with redirect_stdout(buf):
        assert bench.run_reference_arm(args) == 0
    assert buf.getvalue() == ""
