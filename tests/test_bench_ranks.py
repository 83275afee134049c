"""The multi-GPU bench path on the host: two gloo ranks (world_size 2) run the
same rank logic bench.py uses under torchrun -- process group, barrier,
max-over-ranks timing, whole-job rate -- and the reference arm's rule that
only rank 0 works and prints."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    try:
        bench._init_dist(0, backend="gloo")
        bench._barrier()
        # rank r took (r + 1) seconds for 1000 units: the job takes the slowest rank's time
        rate, tmax = bench.whole_job_rate(1000, float(rank + 1))
        m = bench._max_over_ranks(10.0 * rank, 0)
        args = type("A", (), {"count": 4, "seed": 1, "steps": 1, "warmup": 0, "tol": 1e-10,
                              "cpu_budget_s": 0.0})()
        ref = bench.run_batch_reference(args) if rank != 0 else "rank0"
        q.put((rank, rate, tmax, m, ref))
    finally:
        if dist.is_initialized():
            dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_like_the_bench():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        rank, rate, tmax, m, ref = q.get(timeout=120)
        out[rank] = (rate, tmax, m, ref)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in range(world):
        rate, tmax, m, _ = out[rank]
        assert tmax == 2.0  # max over ranks
        assert rate == pytest.approx(world * 1000 / 2.0)
        assert m == 10.0
    assert out[1][3] is None  # the reference arm works on rank 0 only
