"""Multi-rank host path on CPU: world-size-2 gloo ranks each aggregate their own row
partition (with the oracle standing in for the device kernel) and merge the dense group
tables with the same all-reduce bench.py uses; the merged groups equal one aggregate over
the union of the partitions."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from helpers import fact_rows_oracle


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _dense_table(rows):
    """Dense [6, 3] (sum p1, sum p2, count) table of the fact plan for these rows."""
    from helpers import fact_oracle
    keys, sums, counts = fact_oracle(rows)
    t = np.zeros((6, 3), dtype=np.int64)
    for k, s, c in zip(keys, sums, counts):
        g = int(k >> 8) * 2 + int(k & 0xff)
        t[g, 0], t[g, 1], t[g, 2] = s[0], s[1], c
    return t


def _worker(rank, world, port, rows_all, out):
    import torch
    import torch.distributed as dist
    from redfox_b200.partition import merge_group_tables
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    n = len(rows_all) // world
    part = rows_all[rank * n:(rank + 1) * n]
    table = torch.from_numpy(_dense_table(part))
    merge_group_tables(table)
    out[rank] = table.numpy().copy()
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_group_merge_equals_single_aggregate():
    world = 2
    rows = fact_rows_oracle(20000)
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), rows, out), nprocs=world, join=True,
                       start_method="spawn")
    whole = _dense_table(rows)
    assert np.array_equal(out[0], whole) and np.array_equal(out[1], whole)


def test_compact_groups_order():
    from redfox_b200.partition import compact_groups
    t = np.zeros((6, 3), dtype=np.int64)
    t[5] = [7, 8, 2]
    t[1] = [1, 2, 1]
    keys, sums, counts = compact_groups(t, 2, lambda g: ((g // 2) << 8) | (g % 2))
    assert list(keys) == [1, (2 << 8) | 1] and list(counts) == [1, 2] and sums.tolist() == [[1, 2], [7, 8]]
