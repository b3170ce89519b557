"""The multi-rank path of bench.py on CPU: two gloo ranks, each with its own replica of
the work (no collective on the data path), the slowest rank's time as the result, and
only rank 0 reporting."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, results):
    import sys

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r, w, local = bench.dist_env()
        local_ms = 10.0 + 5.0 * r  # rank 1 is the slower replica
        results[r] = (r, w, local, bench.max_over_ranks(local_ms, w))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_time():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        results = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, results)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(results)
    assert res[0] == (0, 2, 0, 15.0)
    assert res[1] == (1, 2, 1, 15.0)


def test_single_rank_is_a_no_op():
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    assert bench.max_over_ranks(3.5, 1) == 3.5


@pytest.mark.parametrize("rank", [1])
def test_reference_arm_other_ranks_do_no_work(rank, monkeypatch, capsys):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    monkeypatch.setenv("RANK", str(rank))
    monkeypatch.setenv("WORLD_SIZE", "2")

    class Args:
        workload = "p1"
        level = None
        steps = 1
        warmup = 0
        cpu_sample_cells = 8

    bench.run_reference(Args())
    assert capsys.readouterr().out == ""
