"""Splitting the configs' independent units across ranks (one process per GPU).

Every workload of the benchmark has units that need no exchange while they
are computed, so N GPUs run them side by side and only the results meet:

* MSSP: the sources.  dist(S, ·) depends on S's own facts and `edge` only,
  so each rank runs the fixpoint for its share of the sources and the union
  of the ranks' relations is the relation of the whole source set.
* batched reachability: the instances (balanced by the n² bit-matrix work).
* probabilistic reachability: the query targets (path(., t) depends only on
  path(., t) and `edge`), so each rank captures its targets' queries.
* triangles: the source vertices of the oriented edges, with the edge list
  replicated; the counts add up.

* Bool transitive closure (one instance): its rows need each other's Δ
  every round, so it has a real exchange step — each rank owns a range of
  path rows (bit rows), and after every round the ranks' Δ' slices are
  all-gathered into the full Δ the next round reads, and their |Δ'| summed
  (`tc_bool_sharded`).

The helpers are plain partition functions plus gather/reduce through
torch.distributed (NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

import numpy as np


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous share [lo, hi) of n units for `rank`."""
    return n * rank // world, n * (rank + 1) // world


def shard_sources(sources, rank: int, world: int):
    """The sources (and their positions) a rank runs: round robin, so every
    rank gets an even share of the id range."""
    idx = np.arange(rank, len(sources), world)
    return np.asarray(sources)[idx], idx


def shard_instances(nodes, rank: int, world: int) -> np.ndarray:
    """Instance indices of `rank`: greedy longest-processing-time assignment
    by the n² bit-matrix cost, deterministic for every rank."""
    cost = np.asarray(nodes, np.float64) ** 2
    order = np.argsort(-cost, kind="stable")
    load = np.zeros(world)
    owner = np.empty(len(cost), np.int64)
    for i in order:
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += cost[i]
    return np.flatnonzero(owner == rank)


def shard_queries(qt, rank: int, world: int) -> np.ndarray:
    """Query indices whose target a rank owns (target id modulo world), so a
    target is captured by one rank only."""
    return np.flatnonzero(np.asarray(qt, np.int64) % world == rank)


def shard_vertices(n_nodes: int, rank: int, world: int) -> tuple[int, int]:
    """The source-vertex range [lo, hi) of the triangle count a rank owns."""
    return shard_range(n_nodes, rank, world)


def batch_subset(wl, idx):
    """The sub-batch of instances `idx` (in that order) of a BatchWorkload."""
    from .gen import BatchWorkload
    idx = np.asarray(idx, np.int64)
    nodes = np.asarray(wl.nodes)[idx]
    lens = (wl.edge_off[idx + 1] - wl.edge_off[idx]).astype(np.uint64)
    off = np.zeros(len(idx) + 1, np.uint64)
    off[1:] = np.cumsum(lens)
    src = np.concatenate([wl.src[int(wl.edge_off[i]):int(wl.edge_off[i + 1])] for i in idx]) if len(idx) else \
        np.zeros(0, np.uint32)
    dst = np.concatenate([wl.dst[int(wl.edge_off[i]):int(wl.edge_off[i + 1])] for i in idx]) if len(idx) else \
        np.zeros(0, np.uint32)
    return BatchWorkload(f"{wl.name}[{len(idx)}]", nodes, off, src, dst, wl.meta)


# ---- meeting of the results (torch.distributed) -----------------------------
def allreduce_sum_u64(dist, value: int, device="cpu") -> int:
    import torch
    t = torch.tensor([int(value)], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return int(t.item())


def allreduce_sum_mod64(dist, value: int, device="cpu") -> int:
    """Sum of unsigned 64-bit values mod 2^64 (fingerprints), through int64."""
    import torch
    v = int(value) & 0xFFFFFFFFFFFFFFFF
    t = torch.tensor([v - (1 << 64) if v >= 1 << 63 else v], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return int(t.item()) & 0xFFFFFFFFFFFFFFFF


def tc_bool_sharded(shards, dist=None, device=None, exchange: str = "auto") -> tuple[int, int, int]:
    """Semi-naive Bool closure with path rows split across ranks.

    `shards` are this process's rank shares (``TcShard`` objects, or any
    object with ``world``, ``shape()``, ``seed``, ``round``, ``summary``,
    ``pack_count``, ``pack`` and ``unpack``): one under torch.distributed
    (`dist` given), whose Δ' meets the other ranks' through an all-gather into
    the full Δ every round (NCCL over NVLink on GPUs); or all `world` shares in
    rank order with `dist` None, the parts then simply concatenated (one
    process standing in for the ranks).

    Each round the ranks first gather every rank's (|Δ'|, nonzero Δ' words),
    one small all-gather.  Then, with `exchange` "auto", a round whose largest
    rank has few nonzero words exchanges only those words — 24 bytes each,
    (word index, 128 bits) — and every rank rebuilds the full Δ from them
    (``pack`` / ``unpack``); a dense round all-gathers the whole Δ' slices and
    row flags.  "dense" and "sparse" force one form.  Every rank takes the
    same collective steps in the same order until the summed |Δ'| is 0.
    Returns (|path|, fingerprint Σ mix64(X)·c^Z mod 2^64, rounds)."""
    import torch
    if exchange not in ("auto", "dense", "sparse"):
        raise ValueError("exchange must be auto, dense or sparse")
    per, _, _, row_bytes = shards[0].shape()
    world = shards[0].world
    words = per * row_bytes // 4
    slice_bytes = per * row_bytes + per
    full = [torch.zeros(world * words, dtype=torch.int32, device=device) for _ in range(2)]
    ffull = [torch.zeros(world * per, dtype=torch.uint8, device=device) for _ in range(2)]
    mine = [torch.zeros(words, dtype=torch.int32, device=device) for _ in shards]
    fmine = [torch.zeros(per, dtype=torch.uint8, device=device) for _ in shards]
    stats = {"dense_rounds": 0, "sparse_rounds": 0, "bytes_per_rank": 0}

    def sparse_wins(m_max: int) -> bool:
        if exchange != "auto":
            return exchange == "sparse"
        return 24 * m_max * 2 <= slice_bytes

    def meet(k: int, counts: list[int]) -> int:
        nnz = [s.pack_count(mine[i]) for i, s in enumerate(shards)]
        if dist is None:
            total, m_max = sum(counts), max(nnz)
        else:
            info = torch.tensor([counts[0], nnz[0]], dtype=torch.int64, device=device)
            every = torch.empty(2 * world, dtype=torch.int64, device=device)
            dist.all_gather_into_tensor(every, info)
            every = every.cpu()
            total, m_max = int(every[0::2].sum()), int(every[1::2].max())
        if m_max == 0:  # no rank has a Δ' word: nothing to exchange
            shards[0].unpack(torch.zeros((0, 3), dtype=torch.int64, device=device), full[k], ffull[k])
        elif sparse_wins(m_max):
            stats["sparse_rounds"] += 1
            stats["bytes_per_rank"] += 24 * m_max
            packs = [s.pack(mine[i], m_max) for i, s in enumerate(shards)]
            if dist is None:
                triples = torch.cat(packs)
            else:
                triples = torch.empty((world * m_max, 3), dtype=torch.int64, device=device)
                dist.all_gather_into_tensor(triples, packs[0].contiguous())
            shards[0].unpack(triples, full[k], ffull[k])
        else:
            stats["dense_rounds"] += 1
            stats["bytes_per_rank"] += slice_bytes
            if dist is None:
                torch.cat(mine, out=full[k])
                torch.cat(fmine, out=ffull[k])
            else:
                dist.all_gather_into_tensor(full[k], mine[0])
                dist.all_gather_into_tensor(ffull[k], fmine[0])
        return total

    total = meet(0, [s.seed(mine[i], fmine[i]) for i, s in enumerate(shards)])
    cur, rounds = 0, 0
    while total:
        rounds += 1
        counts = [s.round(full[cur], ffull[cur], mine[i], fmine[i]) for i, s in enumerate(shards)]
        cur ^= 1
        total = meet(cur, counts)
    tc_bool_sharded.last_stats = stats
    parts = [s.summary() for s in shards]
    count = sum(c for c, _ in parts)
    fp = sum(f for _, f in parts) & 0xFFFFFFFFFFFFFFFF
    if dist is not None:
        count = allreduce_sum_u64(dist, count, device=device or "cpu")
        fp = allreduce_sum_mod64(dist, fp, device=device or "cpu")
    return count, fp, rounds


def gather_objects(dist, obj, world: int) -> list:
    """All ranks' Python objects (small results: per-instance summaries, proof
    lists, relation columns of a test)."""
    out = [None] * world
    dist.all_gather_object(out, obj)
    return out


def merge_by_index(parts: list, n: int) -> list:
    """[(indices, values)] from every rank → values in global index order."""
    out = [None] * n
    for idx, vals in parts:
        for i, v in zip(idx, vals):
            out[int(i)] = v
    return out
