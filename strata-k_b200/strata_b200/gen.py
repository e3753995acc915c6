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
* ``batch_tc_workload`` — many independent directed ER instances (the
  batched reachability config): node counts log-uniform, mean out-degree
  uniform, each instance drawn from its own seed (seed, i).

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


@dataclass
class BatchWorkload:
    """Independent graphs: instance i has nodes [0, nodes[i]) and the edges
    src/dst[edge_off[i]:edge_off[i+1]] (local ids, distinct, no self-loops)."""
    name: str
    nodes: np.ndarray     # u32 [n_inst]
    edge_off: np.ndarray  # u64 [n_inst + 1]
    src: np.ndarray       # u32 [sum m]
    dst: np.ndarray       # u32 [sum m]
    meta: dict | None = None

    def __len__(self) -> int:
        return len(self.nodes)

    def instance(self, i: int) -> tuple[int, np.ndarray, np.ndarray]:
        a, b = int(self.edge_off[i]), int(self.edge_off[i + 1])
        return int(self.nodes[i]), self.src[a:b], self.dst[a:b]


def _er_instance(n: int, m: int, rng) -> tuple[np.ndarray, np.ndarray]:
    have = np.zeros(0, np.int64)
    while len(have) < m:
        need = int((m - len(have)) * 1.1) + 16
        u = rng.integers(0, n, size=need, dtype=np.int64)
        v = rng.integers(0, n, size=need, dtype=np.int64)
        k = u * n + v
        have = np.unique(np.concatenate([have, k[u != v]]))
    k = have[rng.permutation(len(have))[:m]]
    return (k // n).astype(np.uint32), (k % n).astype(np.uint32)


def _batch_chunk(args):
    seed, i0, i1, n_min, n_max, deg_min, deg_max = args
    nodes, ms, srcs, dsts = [], [], [], []
    for i in range(i0, i1):
        rng = np.random.default_rng([seed, i])
        n = int(round(float(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))))
        deg = float(rng.uniform(deg_min, deg_max))
        m = min(int(round(n * deg)), n * (n - 1))
        s_, d_ = _er_instance(n, m, rng)
        nodes.append(n)
        ms.append(m)
        srcs.append(s_)
        dsts.append(d_)
    cat = (lambda xs: np.concatenate(xs) if xs else np.zeros(0, np.uint32))
    return np.array(nodes, np.uint32), np.array(ms, np.uint64), cat(srcs), cat(dsts)


def batch_tc_workload(n_inst=4096, n_min=100, n_max=50_000, deg_min=2.0, deg_max=8.0, seed=4,
                      workers: int = 0) -> BatchWorkload:
    """Instance i: n log-uniform in [n_min, n_max], mean out-degree uniform in
    [deg_min, deg_max], m = round(n * degree) distinct directed non-loop edges
    uniform over the n nodes; every draw of instance i comes from
    default_rng([seed, i]), so the result does not depend on `workers`
    (processes started with spawn; 0 = in this process)."""
    step = 64
    jobs = [(seed, a, min(a + step, n_inst), n_min, n_max, deg_min, deg_max) for a in range(0, n_inst, step)]
    if workers > 1 and len(jobs) > 1:
        import concurrent.futures as cf
        import multiprocessing as mp
        with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            parts = list(ex.map(_batch_chunk, jobs))
    else:
        parts = [_batch_chunk(j) for j in jobs]
    nodes = np.concatenate([p[0] for p in parts]) if parts else np.zeros(0, np.uint32)
    ms = np.concatenate([p[1] for p in parts]) if parts else np.zeros(0, np.uint64)
    off = np.zeros(n_inst + 1, np.uint64)
    off[1:] = np.cumsum(ms)
    src = np.concatenate([p[2] for p in parts]) if parts else np.zeros(0, np.uint32)
    dst = np.concatenate([p[3] for p in parts]) if parts else np.zeros(0, np.uint32)
    return BatchWorkload(f"batch_tc_{n_inst}x_er_{n_min}_{n_max}", nodes, off, src, dst,
                         meta={"instances": n_inst, "n_min": n_min, "n_max": n_max, "deg_min": deg_min,
                               "deg_max": deg_max, "seed": seed, "edges": int(off[-1]),
                               "sum_n2": float((nodes.astype(np.float64) ** 2).sum())})


@dataclass
class ProvWorkload:
    """Probabilistic reachability: edge i has probability p32[i] (fp32; the
    FP64 view p64 is the same value), queries (qs[q], qt[q])."""
    name: str
    n: int
    src: np.ndarray
    dst: np.ndarray
    p32: np.ndarray
    p64: np.ndarray
    qs: np.ndarray
    qt: np.ndarray
    meta: dict | None = None


def prov_workload(n=20_000, m=80_000, n_queries=1024, seed=5) -> ProvWorkload:
    """Directed ER(n, m) with independent edge probabilities ~ Beta(2, 5) drawn
    as fp32, and n_queries (s, t) pairs drawn uniformly."""
    s, d = er_directed(n, m, seed)
    rng = np.random.default_rng(seed + 1)
    p32 = rng.beta(2.0, 5.0, m).astype(np.float32)
    qs = rng.integers(0, n, n_queries).astype(np.uint32)
    qt = rng.integers(0, n, n_queries).astype(np.uint32)
    return ProvWorkload(f"prov_er_{n}_{m}_{n_queries}q", n, s, d, p32, p32.astype(np.float64), qs, qt,
                        meta={"nodes": n, "edges": m, "queries": n_queries, "seed": seed})
