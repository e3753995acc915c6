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
    finally:
        dist.destroy_process_group()
    if rank == 0:
        Path(out_dir, "result.txt").write_text(repr(res))


def test_two_gloo_ranks_split_every_workload(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    res = eval((tmp_path / "result.txt").read_text())
    assert res == {"mssp": True, "batch": True, "prov": True, "tri": True}, res


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
