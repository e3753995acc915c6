"""The multi-rank split of every workload, run as two gloo ranks on the CPU.

Each rank computes its share with the oracle (the device path is covered by
the GPU tests) and the shares meet through torch.distributed exactly as they
do under NCCL; rank 0 checks the merged result against the single-process
result.  One exchange per workload, no data-path collective inside."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class NumpyTcShard:
    """CPU stand-in of one rank's ``TcShard`` with the same buffer layout
    (bit rows of ceil(n / 128) · 16 bytes, bit Z of a row at word Z / 32, bit
    Z % 32), so the orchestrator moves the same bytes as on GPUs."""

    def __init__(self, n, src, dst, rank, world):
        self.n, self.rank, self.world = n, rank, world
        self.per = -(-n // world)
        self.lo = min(rank * self.per, n)
        self.hi = min(self.lo + self.per, n)
        self.w4 = max(1, -(-n // 128))
        self.row_bytes = self.w4 * 16
        self.out = [[] for _ in range(self.hi - self.lo)]
        for a, b in zip(np.asarray(src).tolist(), np.asarray(dst).tolist()):
            if self.lo <= a < self.hi:
                self.out[a - self.lo].append(b)
        self.F = np.zeros((self.hi - self.lo, self.w4 * 128), bool)

    def shape(self):
        return self.per, self.lo, self.hi, self.row_bytes

    def _emit(self, delta, mine, fmine):
        import torch
        rows = np.zeros((self.per, self.w4 * 128), bool)
        rows[: len(delta)] = delta
        packed = np.packbits(rows, axis=1, bitorder="little")
        mine.copy_(torch.from_numpy(packed.reshape(-1).view(np.int32).copy()))
        fmine.copy_(torch.from_numpy(rows.any(axis=1).astype(np.uint8)))
        return int(delta.sum())

    def seed(self, mine, fmine):
        for x, ys in enumerate(self.out):
            self.F[x, ys] = True
        return self._emit(self.F.copy(), mine, fmine)

    def round(self, full, ffull, mine, fmine):
        D = np.unpackbits(full.numpy().view(np.uint8).reshape(-1, self.row_bytes), axis=1, bitorder="little")
        D = D.astype(bool)
        flags = ffull.numpy().astype(bool)
        delta = np.zeros_like(self.F)
        for x, ys in enumerate(self.out):
            ys = [y for y in ys if flags[y]]
            if ys:
                delta[x] = D[ys].any(axis=0) & ~self.F[x]
        self.F |= delta
        return self._emit(delta, mine, fmine)

    def summary(self):
        import oracle as O
        x, z = np.nonzero(self.F)
        return int(len(x)), O.poly_fingerprint(x + self.lo, z, self.n)

    def _words(self, mine):
        return mine.numpy().view(np.uint32).reshape(-1, 4)

    def pack_count(self, mine):
        return int(self._words(mine).any(axis=1).sum())

    def pack(self, mine, cap):
        """(word index, low 64, high 64) of the nonzero 128-bit words, as the
        device pack writes them, padded with index -1."""
        import torch
        w = self._words(mine).astype(np.uint64)
        nz = np.nonzero(w.any(axis=1))[0]
        out = np.full((cap, 3), -1, np.int64)
        out[: len(nz), 0] = nz + self.rank * self.per * self.w4
        out[: len(nz), 1] = (w[nz, 0] | (w[nz, 1] << np.uint64(32))).view(np.int64)
        out[: len(nz), 2] = (w[nz, 2] | (w[nz, 3] << np.uint64(32))).view(np.int64)
        return torch.from_numpy(out)

    def unpack(self, triples, full, ffull):
        t = triples.numpy()
        t = t[t[:, 0] >= 0]
        w = np.zeros((full.numel() // 4, 4), np.uint32)
        lo, hi = t[:, 1].view(np.uint64), t[:, 2].view(np.uint64)
        idx = t[:, 0]
        w[idx, 0], w[idx, 1] = lo & np.uint64(0xFFFFFFFF), lo >> np.uint64(32)
        w[idx, 2], w[idx, 3] = hi & np.uint64(0xFFFFFFFF), hi >> np.uint64(32)
        full.copy_(torch_from(w.reshape(-1).view(np.int32)))
        f = np.zeros(ffull.numel(), np.uint8)
        f[idx // self.w4] = 1
        ffull.copy_(torch_from(f))


def torch_from(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a))


def _closure_graph(seed):
    rng = np.random.default_rng(seed)
    n = 300
    s = rng.integers(0, n, 700)
    d = rng.integers(0, n, 700)
    s[:5], d[:5] = 7, 7  # self-loops and a duplicate
    return n, s.astype(np.uint32), d.astype(np.uint32)


def _worker(rank: int, world: int, port: int, out_dir: str):
    for p in (ROOT / "strata-k_b200", ROOT / "oracle"):
        sys.path.insert(0, str(p))
    import datetime

    import torch.distributed as dist

    import oracle as O
    from strata_b200 import gen, shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    res = {}
    try:
        # MSSP: sources
        wl = gen.mssp_workload(scale=9, n_sources=8, seed=13)
        mine, idx = shard.shard_sources(wl.sources, rank, world)
        s, d, w, inf, _ = O.fast_trop(1, wl.src, wl.dst, wl.w, sources=mine, source_w=wl.source_w[idx])
        parts = shard.gather_objects(dist, (s.tolist(), d.tolist(), w.tolist()), world)
        if rank == 0:
            rows = sorted(r for p in parts for r in zip(*p))
            fs, fd, fw, _, _ = O.fast_trop(1, wl.src, wl.dst, wl.w, sources=wl.sources, source_w=wl.source_w)
            res["mssp"] = rows == sorted(zip(fs.tolist(), fd.tolist(), fw.tolist()))
        # batched reachability: instances
        bw = gen.batch_tc_workload(n_inst=24, n_min=20, n_max=400, seed=14)
        idx = shard.shard_instances(bw.nodes, rank, world)
        sub = shard.batch_subset(bw, idx)
        c, f = O.closure_batch(sub.nodes, sub.edge_off, sub.src, sub.dst, threads=2)
        parts = shard.gather_objects(dist, (idx.tolist(), list(zip(c.tolist(), f.tolist()))), world)
        if rank == 0:
            merged = shard.merge_by_index(parts, len(bw))
            fc, ff = O.closure_batch(bw.nodes, bw.edge_off, bw.src, bw.dst, threads=2)
            res["batch"] = merged == list(zip(fc.tolist(), ff.tolist()))
        # probabilistic reachability: query targets
        pw = gen.prov_workload(n=300, m=1200, n_queries=12, seed=15)
        qi = shard.shard_queries(pw.qt, rank, world)
        pr, _ = O.prov_tc(pw.n, pw.src, pw.dst, pw.p64, 8, pw.qs[qi], pw.qt[qi], threads=2) if len(qi) else ([], {})
        parts = shard.gather_objects(dist, (qi.tolist(), pr), world)
        if rank == 0:
            merged = shard.merge_by_index(parts, len(pw.qs))
            full, _ = O.prov_tc(pw.n, pw.src, pw.dst, pw.p64, 8, pw.qs, pw.qt, threads=2)
            res["prov"] = merged == full
        # triangles: source-vertex ranges over a replicated edge list
        tw = gen.triangle_workload(scale=8, edge_factor=8, seed=16)
        n = int(max(tw.src.max(), tw.dst.max())) + 1
        lo, hi = shard.shard_vertices(n, rank, world)
        out = [set() for _ in range(n)]
        for a, b in zip(tw.src.tolist(), tw.dst.tolist()):
            out[a].add(b)
        mine = sum(len(out[x] & out[y]) for x in range(lo, hi) for y in out[x])
        total = shard.allreduce_sum_u64(dist, mine)
        if rank == 0:
            res["tri"] = total == O.count_pattern(tw.src, tw.dst)
        # Bool closure: path rows per rank, Δ' exchanged every round (dense
        # slices, sparse nonzero words, or whichever is smaller)
        n, cs, cd = _closure_graph(17)
        got = {x: shard.tc_bool_sharded([NumpyTcShard(n, cs, cd, rank, world)], dist, exchange=x)
               for x in ("auto", "dense", "sparse")}
        if rank == 0:
            c, f = O.closure_batch([n], [0, len(cs)], cs, cd, threads=2)
            want = (int(c[0]), int(f[0]), O.fast_tc(cs, cd)[2])
            res["tc"] = all(g == want for g in got.values())
    finally:
        dist.destroy_process_group()
    if rank == 0:
        Path(out_dir, "result.txt").write_text(repr(res))


def test_two_gloo_ranks_split_every_workload(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    res = eval((tmp_path / "result.txt").read_text())
    assert res == {"mssp": True, "batch": True, "prov": True, "tri": True, "tc": True}, res


def test_sharded_closure_emulated_ranks():
    """All ranks' shares in one process (slices concatenated): uneven row
    splits, more ranks than rows, and an edge-free rank give the closure's
    count, fingerprint and rounds."""
    sys.path.insert(0, str(ROOT / "strata-k_b200"))
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    from strata_b200 import shard
    n, cs, cd = _closure_graph(18)
    c, f = O.closure_batch([n], [0, len(cs)], cs, cd, threads=2)
    want = (int(c[0]), int(f[0]), O.fast_tc(cs, cd)[2])
    forms = set()
    for world in (1, 3, 7):
        for x in ("auto", "dense", "sparse"):
            got = shard.tc_bool_sharded([NumpyTcShard(n, cs, cd, r, world) for r in range(world)], exchange=x)
            assert got == want, (world, x)
            st = shard.tc_bool_sharded.last_stats
            if x == "auto":
                forms |= {k for k in ("dense_rounds", "sparse_rounds") if st[k]}
    assert forms == {"dense_rounds", "sparse_rounds"}  # auto used both forms
    for x in ("auto", "dense", "sparse"):
        tiny = shard.tc_bool_sharded([NumpyTcShard(2, [0], [1], r, 4) for r in range(4)], exchange=x)
        assert tiny == (1, O.poly_fingerprint([0], [1], 2), 1)


def test_partitions_cover_every_unit_once():
    sys.path.insert(0, str(ROOT / "strata-k_b200"))
    from strata_b200 import shard
    for world in (1, 2, 3, 8):
        src = np.arange(64)
        got = np.sort(np.concatenate([shard.shard_sources(src, r, world)[1] for r in range(world)]))
        assert np.array_equal(got, np.arange(64))
        nodes = np.random.default_rng(world).integers(100, 50_000, 300)
        got = np.sort(np.concatenate([shard.shard_instances(nodes, r, world) for r in range(world)]))
        assert np.array_equal(got, np.arange(300))
        loads = [float((nodes[shard.shard_instances(nodes, r, world)].astype(float) ** 2).sum()) for r in range(world)]
        assert max(loads) <= 1.05 * (sum(loads) / world) + float(nodes.max()) ** 2
        qt = np.random.default_rng(5).integers(0, 1000, 200)
        got = np.sort(np.concatenate([shard.shard_queries(qt, r, world) for r in range(world)]))
        assert np.array_equal(got, np.arange(200))
        spans = [shard.shard_vertices(1001, r, world) for r in range(world)]
        assert spans[0][0] == 0 and spans[-1][1] == 1001
        assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
