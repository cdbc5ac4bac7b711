"""The multi-GPU form is replicas only: every rank solves its own instances and the ranks meet only in the
timing collectives (max of the times, sum of the counts).  Checked here with two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import sys

    import torch.distributed as dist

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    r, w, local = bench.dist_env()
    maxes, sums = bench.combine_over_ranks(dist, [10.0 + r, 3.0 * (r + 1)], [100 * (r + 1), 7], device="cpu")
    seed = bench.PLAIN["seed"] + r
    out.put((r, w, local, maxes, sums, seed))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_combine_times_by_max_and_counts_by_sum():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, (rank, world, local, maxes, sums, seed) in enumerate(got):
        assert (rank, world, local) == (r, 2, r)
        assert maxes == [11.0, 6.0] and sums == [300.0, 14.0]
        assert seed == 1 + r  # each replica solves its own seed


def test_single_process_combine_is_identity():
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    assert bench.combine_over_ranks(None, [1, 2], [3]) == ([1.0, 2.0], [3.0])
