"""Row partitioning across GPUs for the scan / aggregate plans.

A fact table partitions by rows: rank r owns rows [r * n, (r + 1) * n) of the seeded table
(its own generator stream), runs the plan locally and the group tables are summed with one
all-reduce -- the only exchange the plan has.  Group tables are dense int64 arrays of
groups x (sums + count), so the element-wise sum (wrapping int64) is the exact merge.
"""


def partition_seed(base_seed, rank):
    """Seed of rank `rank`'s partition (rank 0 uses the base seed)."""
    return base_seed + rank


def merge_group_tables(table, group=None):
    """Sum a dense int64 group table over all ranks, in place (NCCL on GPU, gloo on CPU)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(table, group=group)
    return table


def compact_groups(table, nsum, key_of_index):
    """Dense [groups, nsum + 1] table -> (keys, sums, counts) of the non-empty groups in
    group-index order (the packed-key order of the mixed-radix group index)."""
    import numpy as np
    t = np.asarray(table).reshape(-1, nsum + 1)
    nz = np.nonzero(t[:, nsum])[0]
    keys = np.array([key_of_index(int(g)) for g in nz], dtype=np.uint64)
    return keys, t[nz, :nsum].astype(np.int64), t[nz, nsum].astype(np.uint64)
