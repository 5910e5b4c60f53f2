"""Host side of the row-sharded job=1 (CPU, no GPU).

The row split must be the reference's MPI split (kappa.f90:418-428), and
the torch.distributed all-gather adapter that feeds
ald_kappa_pipeline_sharded must concatenate ranks' blocks of different
lengths in rank order.  The adapter runs here on world_size-2 gloo ranks,
the same code path as under torchrun with NCCL.
"""
import os
import socket
import sys

import numpy as np
import pytest

import ald

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("nibz", [1, 7, 85, 276, 1768])
@pytest.mark.parametrize("nranks", [1, 2, 3, 8])
def test_shard_rows_is_the_reference_split(nibz, nranks):
    if nranks > nibz:
        pytest.skip("more ranks than rows")
    local = nibz // nranks
    seen = []
    for r in range(nranks):
        lo, hi = ald.shard_rows(nibz, r, nranks)
        # ksubset(1) = rank*local + 1, ksubset(2) = rank*local + local (+ remainder on the last rank)
        assert lo == r * local + 1
        assert hi == (r * local + local + (nibz % nranks if r == nranks - 1 else 0))
        seen.extend(range(lo, hi + 1))
    assert seen == list(range(1, nibz + 1))


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        counts = [3 * (k + 1) for k in range(world)]  # uneven blocks
        mine = np.arange(counts[rank], dtype=float) + 1000.0 * rank
        allv = ald.torch_allgather()(mine, counts)
        want = np.concatenate([np.arange(c, dtype=float) + 1000.0 * k for k, c in enumerate(counts)])
        out.put((rank, bool(np.array_equal(allv, want))))
        # an empty block on one rank (more ranks than rows)
        counts0 = [0] + counts[1:]
        mine0 = np.zeros(0) if rank == 0 else mine
        allv0 = ald.torch_allgather()(mine0, counts0)
        out.put((rank, bool(np.array_equal(allv0, np.concatenate([np.zeros(0)] + [
            np.arange(c, dtype=float) + 1000.0 * k for k, c in enumerate(counts0) if k > 0])))))
    finally:
        dist.destroy_process_group()


def test_torch_allgather_gloo_two_ranks():
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = [q.get(timeout=5) for _ in range(4)]
    assert all(ok for _, ok in res), res


def _failing_worker(rank, world, port, out):
    """Rank 1 fails before the exchange (a shard lost between steps); rank 0
    must get an error from its all-gather within the process group's
    timeout instead of waiting for good."""
    import datetime
    import time
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    counts = [4, 4]
    if rank == 1:
        dist.barrier()  # both ranks are up
        out.put((rank, "left"))
        out.close()
        out.join_thread()  # the message is out before the process ends
        os._exit(3)  # no destroy_process_group: the peer sees the rank vanish
    dist.barrier()
    t0 = time.time()
    try:
        ald.torch_allgather()(np.ones(4), counts)
        out.put((rank, "no error"))
    except Exception as e:  # the expected path
        out.put((rank, "error after %.1f s: %s" % (time.time() - t0, type(e).__name__)))
    out.close()
    out.join_thread()
    os._exit(0)


def test_torch_allgather_reports_a_lost_rank():
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_failing_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=90)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive, "a rank hung on the lost peer"
    res = dict(q.get(timeout=5) for _ in range(2))
    assert res[1] == "left"
    assert res[0].startswith("error after"), res[0]
    assert procs[0].exitcode == 0 and procs[1].exitcode == 3
