"""bench.py's multi-rank path on CPU: two gloo ranks (127.0.0.1) run the same
barrier and reductions the GPU replicas run over NCCL (max over ranks of the
timed region, whole-job rate = units of all ranks / slowest rank's time)."""
import multiprocessing as mp
import os
import socket
import sys
from datetime import timedelta

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench

    bench.rank_barrier(world)
    mx = bench.max_over_ranks(1.5 + rank, world)  # a rank's timed seconds
    sm = bench.sum_over_ranks(10 * (rank + 1), world)  # completed requests
    rate = bench.job_rate(100, world, mx)
    bench.rank_barrier(world)
    dist.destroy_process_group()
    q.put((rank, mx, sm, rate))


def test_two_gloo_ranks_reduce_like_the_gpu_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, sm, rate in res:
        assert mx == 2.5  # the slowest rank's time, on every rank
        assert sm == 30.0
        assert rate == 2 * 100 / 2.5  # both ranks' units over the slowest time


def test_single_rank_reductions_are_identities():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.25, 1) == 3.25
    assert bench.sum_over_ranks(7, 1) == 7.0
    assert bench.job_rate(50, 1, 2.0) == 25.0


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun the reference arm's other ranks exit without work."""
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        workload, steps, warmup, scale = "suite", 1, 0, 20

    assert bench.run_reference(Args(), rank=1, world=2) is None
