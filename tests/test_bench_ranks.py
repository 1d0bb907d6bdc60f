"""The multi-rank plumbing of bench.py on CPU (gloo, world size 2): the whole-job value is world x k increments
over the slowest rank's time, identical on every rank, and the reference arm does no work on ranks other than 0.
The 3D path does not shard, so N GPUs run N replicas; these are the only collectives the bench takes."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        value, ms = bench.whole_job_value(100.0 * (rank + 1), 20, world, device="cpu")
        if rank != 0:
            assert bench.run_reference(None, rank, world) is None  # returns before touching its arguments
        out.put((rank, value, ms))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_whole_job_value_is_the_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), q), nprocs=world, join=True, start_method="spawn")
    got = sorted(q.get() for _ in range(world))
    for rank, value, ms in got:
        assert ms == 200.0  # the slower rank's 200 ms
        assert value == pytest.approx(world * 20 / 0.2)


def test_single_rank_value_needs_no_process_group():
    import bench

    value, ms = bench.whole_job_value(250.0, 10, 1)
    assert ms == 250.0 and value == pytest.approx(40.0)
