"""Seeded synthetic inputs with the benchmark shapes (no datasets are used).

* ``er_directed``  — Erdős–Rényi directed graph with exactly m distinct
  (u, v), u != v, uniform over n nodes.
* ``rmat``         — R-MAT (a, b, c, d) graph of 2^scale nodes with exactly m
  distinct non-loop edges (directed, or undirected as canonical (lo, hi)).
* ``orient_by_degree`` — orient an undirected simple graph from lower to
  higher (degree, id) rank (a DAG, so e(X,Y),e(Y,Z),e(X,Z) counts each
  triangle once).
* ``intern_first_seen`` — the reference's symbol ids: first-seen order over
  pre-seeded symbols then the TSV cells row by row, column by column
  (strata-ir/src/dict.rs:35-43, strata-k/src/input.rs:109-149).
* ``mssp_workload`` / ``tc_workload`` / ``triangle_workload`` — the configs.

All randomness comes from ``numpy.random.default_rng(seed)`` (PCG64).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def er_directed(n: int, m: int, seed: int) -> tuple[np.ndarray, np.ndarray]:
    if m > n * (n - 1):
        raise ValueError("too many edges for n nodes")
    rng = np.random.default_rng(seed)
    have = np.zeros(0, np.uint64)
    while len(have) < m:
        need = int((m - len(have)) * 1.15) + 64
        u = rng.integers(0, n, size=need, dtype=np.uint64)
        v = rng.integers(0, n, size=need, dtype=np.uint64)
        k = (u << np.uint64(32)) | v
        k = k[u != v]
        have = np.unique(np.concatenate([have, k]))
    pick = rng.choice(len(have), size=m, replace=False)
    k = have[pick]
    return (k >> np.uint64(32)).astype(np.uint32), (k & np.uint64(0xFFFFFFFF)).astype(np.uint32)


def _rmat_batch(rng, scale: int, count: int, a: float, b: float, c: float):
    u = np.zeros(count, np.uint64)
    v = np.zeros(count, np.uint64)
    ab, abc = a + b, a + b + c
    for level in range(scale):
        r = rng.random(count, dtype=np.float32)
        ub = r >= ab
        vb = ((r >= a) & (r < ab)) | (r >= abc)
        bit = np.uint64(1) << np.uint64(scale - 1 - level)
        u |= ub.astype(np.uint64) * bit
        v |= vb.astype(np.uint64) * bit
    return u, v


def rmat(scale: int, m: int, seed: int, a=0.57, b=0.19, c=0.19, undirected=False,
         chunk: int = 1 << 22) -> tuple[np.ndarray, np.ndarray]:
    """Exactly m distinct non-loop R-MAT edges (canonical lo<hi if undirected),
    returned in a random order."""
    rng = np.random.default_rng(seed)
    have = np.zeros(0, np.uint64)
    while len(have) < m:
        need = max(int((m - len(have)) * 1.3), 1024)
        parts = []
        for s in range(0, need, chunk):
            u, v = _rmat_batch(rng, scale, min(chunk, need - s), a, b, c)
            if undirected:
                lo, hi = np.minimum(u, v), np.maximum(u, v)
                u, v = lo, hi
            k = (u << np.uint64(32)) | v
            parts.append(k[u != v])
        have = np.unique(np.concatenate([have] + parts))
    pick = rng.choice(len(have), size=m, replace=False)
    k = have[pick]
    return (k >> np.uint64(32)).astype(np.uint32), (k & np.uint64(0xFFFFFFFF)).astype(np.uint32)


def orient_by_degree(lo: np.ndarray, hi: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Orient undirected simple edges from lower to higher (degree, id) rank."""
    n = int(max(lo.max(initial=0), hi.max(initial=0))) + 1
    deg = np.bincount(lo, minlength=n) + np.bincount(hi, minlength=n)
    dl, dh = deg[lo], deg[hi]
    first = (dl < dh) | ((dl == dh) & (lo < hi))
    return np.where(first, lo, hi).astype(np.uint32), np.where(first, hi, lo).astype(np.uint32)


def intern_first_seen(*cols: np.ndarray, seed_symbols: np.ndarray | None = None):
    """Map raw node names (ints) to first-seen ids.

    Symbols in ``seed_symbols`` are interned first (check-time constants,
    e.g. inline ``src`` facts), then the columns row by row, column by column.
    Returns (ids for seed_symbols or None, [ids per column], n_symbols).
    """
    rows = np.column_stack([np.asarray(c, dtype=np.uint64) for c in cols]).ravel()
    pre = np.zeros(0, np.uint64) if seed_symbols is None else np.asarray(seed_symbols, np.uint64)
    allv = np.concatenate([pre, rows])
    uniq, first, inv = np.unique(allv, return_index=True, return_inverse=True)
    order = np.argsort(first, kind="stable")
    rank = np.empty(len(uniq), np.uint32)
    rank[order] = np.arange(len(uniq), dtype=np.uint32)
    ids = rank[inv]
    seed_ids = ids[:len(pre)] if seed_symbols is not None else None
    body = ids[len(pre):].reshape(-1, len(cols))
    return seed_ids, [np.ascontiguousarray(body[:, k]) for k in range(len(cols))], len(uniq)


@dataclass
class Workload:
    name: str
    src: np.ndarray
    dst: np.ndarray
    w: np.ndarray | None = None
    sources: np.ndarray | None = None
    source_w: np.ndarray | None = None
    n_symbols: int = 0
    meta: dict | None = None


def tc_workload(n=10_000, m=50_000, seed=1) -> Workload:
    """Bool TC on a directed ER graph; ids interned first-seen from the TSV."""
    s, d = er_directed(n, m, seed)
    _, (si, di), ns = intern_first_seen(s, d)
    return Workload(f"tc_er_{n}_{m}", si, di, n_symbols=ns, meta={"nodes": n, "edges": m, "seed": seed})


def mssp_workload(scale=20, edge_factor=8, n_sources=64, seed=2, wmax=100) -> Workload:
    """Trop multi-source shortest paths on R-MAT(scale), i64 weights U[1, wmax].

    Sources are drawn uniformly among nodes with at least one out-edge (a
    source without out-edges derives nothing).  The 64 inline `0 :: src(n)`
    facts are interned before the TSV, so sources get the lowest ids.
    """
    m = edge_factor << scale
    s, d = rmat(scale, m, seed)
    rng = np.random.default_rng(seed + 1000)
    w = rng.integers(1, wmax + 1, size=m, dtype=np.int64)
    cand = np.unique(s)
    srcs = rng.choice(cand, size=min(n_sources, len(cand)), replace=False).astype(np.uint64)
    sid, (si, di), ns = intern_first_seen(s, d, seed_symbols=srcs)
    return Workload(f"mssp_rmat{scale}_{n_sources}src", si, di, w=w, sources=sid,
                    source_w=np.zeros(len(sid), np.int64), n_symbols=ns,
                    meta={"scale": scale, "edges": m, "sources": int(len(sid)), "seed": seed})


def triangle_workload(scale=22, edge_factor=16, seed=3) -> Workload:
    """Undirected R-MAT(scale) with exactly edge_factor*2^scale unique edges,
    oriented by degree; ids interned first-seen from the TSV."""
    m = edge_factor << scale
    lo, hi = rmat(scale, m, seed, undirected=True)
    x, y = orient_by_degree(lo, hi)
    _, (xi, yi), ns = intern_first_seen(x, y)
    return Workload(f"tri_rmat{scale}", xi, yi, n_symbols=ns, meta={"scale": scale, "edges": m, "seed": seed})
