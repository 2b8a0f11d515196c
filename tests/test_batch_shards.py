"""The many-drape split over GPUs (drape_b200/batch_shards.py) on the host: the row-balanced partition, and the
end-of-job combine over two `gloo` ranks on CPU (the only exchange the split has)."""
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from drape_b200 import batch_shards
from drape_b200.scenes import batch_scenes


def test_partition_covers_every_drape_once_and_balances_rows():
    rows = [n * n for n, _, _, _ in batch_scenes(128)]
    for ranks in (1, 2, 3, 8):
        shares = batch_shards.partition(rows, ranks)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(128))
        loads = [sum(rows[i] for i in s) for s in shares]
        # longest-processing-time bound: no rank exceeds the mean by more than the largest drape
        assert max(loads) - sum(loads) / ranks <= max(rows)
        assert all(s == sorted(s) for s in shares)
    assert batch_shards.partition([5, 3], 4) == [[0], [1], [], []]
    with pytest.raises(ValueError):
        batch_shards.partition([1], 0)


def test_combine_on_one_rank_is_the_identity():
    t, c, s = batch_shards.combine(2.5, {"solved": 2, "newton": 7}, np.array([1.0, 2.0]), [0, 2], 3)
    assert t == 2.5 and c == {"newton": 7, "solved": 2} and np.array_equal(s, [1.0, 0.0, 2.0])


def _rank(rank, world, port, out):
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    shares = batch_shards.partition([4, 9, 1, 16, 25], world)
    mine = shares[rank]
    seconds = np.array([10.0 * i + 1 for i in mine])
    t, c, s = batch_shards.combine(1.0 + rank, {"solved": len(mine), "newton": 3.0 * (rank + 1)}, seconds, mine, 5,
                                   dist)
    out[rank] = (t, c["solved"], c["newton"], list(s))
    dist.destroy_process_group()


def test_combine_over_two_gloo_ranks():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        for r in range(2):
            t, solved, newton, s = out[r]
            assert t == 2.0 and solved == 5 and newton == 9.0
            assert s == [10.0 * i + 1 for i in range(5)]
