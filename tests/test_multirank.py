"""The multi-GPU path of bench.py on CPU: two `gloo` ranks (world_size 2).

The map shards with no data exchange: rank r computes the r-th c-stripe of the
grid at full resolution (weak scaling), and the only collectives are the
barriers and the maximum over ranks of the timings.  Checked here: the stripes
tile the c range exactly (no gap, no overlap, the last one ends at the range's
end), every rank sees the same maxima, and ranks that compute different
amounts still agree on the job's time.
"""
import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, q) -> None:
    import datetime

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        w = bench.stripe(bench.SUR_WORKLOAD, rank, world)
        # per-rank "timings": rank 1 is the slow one for the first entry
        t = bench.max_over_ranks([1.0 + rank, 10.0 - rank], dist, "cpu")
        stripes = [None] * world
        dist.all_gather_object(stripes, w["ranges"])
        dist.barrier()
        q.put((rank, t, stripes))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_ranks_tile_the_grid_and_agree_on_time(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sys.path.insert(0, str(ROOT))
    import bench

    full = bench.SUR_WORKLOAD["ranges"]
    for rank, t, stripes in results:
        assert t == [float(world), 10.0]  # the slowest rank's time, on every rank
        assert stripes[0][2] == full[2] and stripes[-1][3] == full[3]
        for a, b in zip(stripes, stripes[1:]):
            assert a[3] == b[2]  # contiguous, no overlap
        assert all(s[:2] == full[:2] for s in stripes)  # the a axis is never split
    assert len({tuple(map(tuple, r[2])) for r in results}) == 1


def test_single_rank_is_the_whole_grid():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.stripe(bench.SUR_WORKLOAD, 0, 1) == dict(bench.SUR_WORKLOAD)
    assert bench.max_over_ranks([3.0, 4.0]) == [3.0, 4.0]
