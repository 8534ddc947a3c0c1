"""Multi-GPU execution of the hot path: one process per GPU (torch.distributed), the fact
table split into row ranges (the reference's morsels, runtime_struct.cpp:856-872, one range
per rank), dimension / build tables replicated, and one exchange step that merges the ranks'
partial aggregates -- the reference's flush2partitions + re-aggregation across threads
(runtime_struct.cpp:1327-1350, relalg_translator.cpp:776-808), here across ranks.

Every aggregate the CUDA flavor emits is a sum or a count, so merging partial rows is a sum
per key (a count re-aggregates as a sum, relalg_translator.cpp:789-792).  Grouped partials are
hash-partitioned so every rank merges a disjoint key range; global partials are reduced.
"""
import numpy as np


EMIT = -1


def plan_group_keys(plan):
    """Number of group keys of the plan's root aggregation: 0 for a global aggregate, EMIT for
    a plan whose root emits rows (no aggregation; the ranks' rows are disjoint and their union
    is the result).  Raises ValueError for text that is not a plan."""
    tokens = plan.replace("(", " ( ").replace(")", " ) ").split()
    if len(tokens) < 2 or tokens[0] != "(":
        raise ValueError("not a plan: " + plan[:40])
    if tokens[1] != "aggr":
        return EMIT
    if len(tokens) < 4 or tokens[2] not in ("hash", "global"):
        raise ValueError("malformed aggregation at the plan root")
    if tokens[2] == "global":
        return 0
    depth, n, i = 0, 0, 3
    while i < len(tokens):  # count the top-level items of the key list
        t = tokens[i]
        if t == "(":
            depth += 1
            if depth == 2:
                n += 1
        elif t == ")":
            depth -= 1
            if depth == 0:
                break
        i += 1
    return n


def load_shard(engine, w, data, rank, world):
    """Declares the workload's tables on `engine` with this rank's row range of the fact table
    (the other tables replicated) and uploads them from host arrays ({table: {col: array}})."""
    b, e = shard_rows(w.fact_rows, rank, world)
    for t, rows in w.tables.items():
        engine.create_table(t, (e - b) if t == w.fact_table else rows)
    for c in w.columns:
        engine.add_column(c.table, c.name, c.type, c.lo, c.hi)
        a = data[c.table][c.name]
        engine.upload(c.table, c.name, a[b:e] if c.table == w.fact_table else a)


def shard_rows(n, rank, world):
    """Row range [begin, end) of the fact table that `rank` of `world` processes."""
    return n * rank // world, n * (rank + 1) // world


def _key_partition(keys, world):
    if keys.shape[1] == 0:
        return np.zeros(len(keys), dtype=np.int64)
    h = np.zeros(len(keys), dtype=np.uint64)
    with np.errstate(over="ignore"):
        for i in range(keys.shape[1]):
            z = keys[:, i].astype(np.int64).view(np.uint64) + h * np.uint64(0x9e3779b97f4a7c15)
            z = (z ^ (z >> np.uint64(30))) * np.uint64(0xbf58476d1ce4e5b9)
            z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94d049bb133111eb)
            h = z ^ (z >> np.uint64(31))
    return (h % np.uint64(world)).astype(np.int64)


def _merge_local(rows, nkeys):
    if len(rows) == 0:
        return rows
    keys = rows[:, :nkeys]
    uniq, inv = np.unique(keys, axis=0, return_inverse=True)
    inv = inv.reshape(-1)
    order = np.argsort(inv, kind="stable")
    bounds = np.concatenate([[0], np.nonzero(np.diff(inv[order]))[0] + 1])
    sums = np.add.reduceat(rows[order][:, nkeys:], bounds, axis=0)
    return np.concatenate([uniq, sums], axis=1).astype(np.int64)


def _all_gather_rows(rows, ncols, group, device):
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    n = torch.tensor([len(rows)], dtype=torch.int64, device=device)
    sizes = [torch.zeros(1, dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    cap = max(int(s.item()) for s in sizes)
    buf = torch.zeros((max(cap, 1), ncols), dtype=torch.int64, device=device)
    if len(rows):
        buf[:len(rows)] = torch.from_numpy(np.ascontiguousarray(rows, dtype=np.int64)).to(device)
    outs = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(outs, buf, group=group)
    return [o[:int(s.item())].cpu().numpy() for o, s in zip(outs, sizes)]


def merge_rows(allrows, nkeys, rank, world):
    """This rank's share of the merged result, given every rank's partial rows (keys then
    aggregates): a disjoint key partition, summed per key, for grouped results; the single
    summed row on rank 0 for a global aggregate (none on the others, and none at all when no
    rank had a row: an aggregate over zero matches emits nothing)."""
    allrows = np.asarray(allrows, dtype=np.int64)
    if nkeys == EMIT:
        raise ValueError("emit plans are not merged: each rank's rows are its share")
    if nkeys == 0:
        if rank != 0 or len(allrows) == 0:
            return allrows[:0]
        return allrows.sum(axis=0, keepdims=True).astype(np.int64)
    mine = allrows[_key_partition(allrows[:, :nkeys], world) == rank]
    return _merge_local(mine, nkeys)


def merge_partials(rows, nkeys, ncols, group=None, device="cpu"):
    """Merges this rank's partial result rows (keys then aggregates, int64) with the other
    ranks' (an all-gather, then merge_rows).  For an emit plan (nkeys == EMIT) there is nothing
    to merge: the rank's own rows are its share of the union."""
    import torch.distributed as dist
    rows = np.asarray(rows, dtype=np.int64).reshape(-1, ncols)
    if nkeys == EMIT:
        return rows
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    parts = _all_gather_rows(rows, ncols, group, device)
    allrows = np.concatenate(parts, axis=0) if parts else rows[:0]
    return merge_rows(allrows, nkeys, rank, world)


def gather_result(rows, ncols, group=None, device="cpu"):
    """All merged rows on every rank (concatenation of the ranks' partitions)."""
    parts = _all_gather_rows(np.asarray(rows, dtype=np.int64).reshape(-1, ncols), ncols, group, device)
    return np.concatenate(parts, axis=0) if parts else np.zeros((0, ncols), dtype=np.int64)
