"""The multi-GPU path of bench.py is replicas only: each rank solves its own problem, and
the ranks exchange nothing but a barrier around the timed region and the maximum of the
timed duration.  That coordination runs here as two gloo processes on the CPU."""
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


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r = bench.Replicas(dist, "cpu")
        r.barrier()
        t = r.max_over_ranks(1.5 + rank)  # the ranks' own durations differ
        r.barrier()
        out.put((rank, t, bench.Replicas.job_rate(world, 20, t)))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_replica_timing_two_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=100) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every rank sees the slowest rank's time; the job rate counts all ranks' steps
    assert [t for _, t, _ in res] == [2.5, 2.5]
    assert all(abs(v - 2 * 20 / 2.5) < 1e-12 for _, _, v in res)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    r = bench.Replicas(None, "cpu")
    r.barrier()
    assert r.max_over_ranks(3.0) == 3.0


def test_reference_arm_other_ranks_exit_without_work():
    """Under torchrun only rank 0 runs the reference arm; the others return 0 at once."""
    sys.path.insert(0, ROOT)
    import bench
    assert bench.run_reference(None, rank=1, world=2) == 0

