"""The N>1 path of bench.py (replicas only: one independent replica per
GPU, no data-path collective) on CPU: two gloo ranks through the same
process-group set-up and the max-over-ranks timing reduction."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    r, world, local, pg = bench.dist_setup(None, backend="gloo")
    # rank 1 is the slower replica in both measures
    total_s, e2e_s = bench.replica_times(pg, 1.0 + rank, 2.0 + 3.0 * rank, device="cpu")
    pg.barrier()
    q.put((r, world, local, total_s, e2e_s, bench.replica_value(world, 10, total_s)))
    pg.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, (rank, world, local, total_s, e2e_s, value) in enumerate(out):
        assert (rank, world, local) == (r, 2, r)
        assert total_s == 2.0 and e2e_s == 5.0      # the max over the two ranks
        assert value == pytest.approx(10.0)         # 2 replicas x 10 matvecs / 2 s


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        os.environ.pop(k, None)
    rank, world, local, pg = bench.dist_setup(None)
    assert (rank, world, local, pg) == (0, 1, 0, None)
    assert bench.replica_times(pg, 1.5, 2.5) == (1.5, 2.5)
    assert bench.replica_value(world, 20, 0.5) == 40.0
