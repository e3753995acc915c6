"""Batched Bool reachability and the bit-row closure plan against the oracle.

Every instance's |path| and row-polynomial fingerprint must equal the SCC
oracle's, and its round count the semi-naive restatement's (the reference's
`run_semi_naive` schedule, strata-eval/src/seminaive.rs:29-106)."""
import numpy as np
import pytest

import oracle as O
import strata_b200 as S
from strata_b200 import gen

pytestmark = pytest.mark.gpu


def _check(res, wl, rounds_sample=16):
    counts, fps = O.closure_batch(wl.nodes, wl.edge_off, wl.src, wl.dst, threads=8)
    assert np.array_equal(res.counts, counts)
    assert np.array_equal(res.fps, fps)
    for i in range(min(rounds_sample, len(wl))):
        n, s, d = wl.instance(i)
        if n > 3000:  # the tuple-materialising restatement stays at small sizes
            continue
        if len(s):
            _, _, r = O.fast_tc(s, d)
            assert int(res.rounds[i]) == r, i
        else:
            assert int(res.rounds[i]) == 0


def test_batch_matches_oracle(engine):
    wl = gen.batch_tc_workload(n_inst=384, n_min=20, n_max=3000, seed=21)
    res = engine.tc_bool_batch(wl.nodes, wl.edge_off, wl.src, wl.dst, mode=0)
    _check(res, wl)
    assert res.stats["instances"] == 384 and res.stats["graph_launches"] >= 1
    assert res.stats["result_tuples"] == int(res.counts.sum())


def test_batch_large_instances(engine):
    """Rows wider than a warp's 32 × 128 bits (lanes loop over chunks)."""
    wl = gen.batch_tc_workload(n_inst=5, n_min=9000, n_max=50_000, deg_min=1.5, deg_max=3.0, seed=5)
    res = engine.tc_bool_batch(wl.nodes, wl.edge_off, wl.src, wl.dst, mode=0)
    _check(res, wl, rounds_sample=2)


def test_batch_one_per_launch_agrees(engine):
    wl = gen.batch_tc_workload(n_inst=64, n_min=50, n_max=2000, seed=22)
    a = engine.tc_bool_batch(wl.nodes, wl.edge_off, wl.src, wl.dst, mode=0)
    b = engine.tc_bool_batch(wl.nodes, wl.edge_off, wl.src, wl.dst, mode=1)
    assert np.array_equal(a.counts, b.counts) and np.array_equal(a.fps, b.fps)
    assert np.array_equal(a.rounds, b.rounds)
    assert b.stats["graph_launches"] == 0 and b.stats["waves"] == 64


@pytest.mark.parametrize("knob,value", [(4, 2), (4, 32), (5, 1), (6, 1)])
def test_batch_knobs_identical(engine, knob, value):
    """Graph rounds, resident blocks and a 1 MiB wave budget (many waves)
    change speed only."""
    wl = gen.batch_tc_workload(n_inst=96, n_min=30, n_max=1500, seed=23)
    base = engine.tc_bool_batch(wl.nodes, wl.edge_off, wl.src, wl.dst, mode=0)
    engine.set_knob(knob, value)
    try:
        got = engine.tc_bool_batch(wl.nodes, wl.edge_off, wl.src, wl.dst, mode=0)
    finally:
        engine.set_knob(knob, 0)
    assert np.array_equal(base.counts, got.counts) and np.array_equal(base.fps, got.fps)
    assert np.array_equal(base.rounds, got.rounds)
    if knob == 6:
        assert got.stats["waves"] > 1


def test_batch_edge_cases(engine):
    """Empty instances, one node, self-loops, duplicate edges, a cycle (n^2
    pairs), a chain (n(n-1)/2 pairs, n-1 rounds)."""
    inst = [
        (1, [], []),
        (7, [], []),
        (1, [0], [0]),
        (3, [0, 0, 1], [1, 1, 2]),
        (200, list(range(200)), [(i + 1) % 200 for i in range(200)]),
        (300, list(range(299)), list(range(1, 300))),
        (129, [0, 128, 64], [128, 64, 0]),
    ]
    nodes = np.array([n for n, _, _ in inst], np.uint32)
    off = np.zeros(len(inst) + 1, np.uint64)
    for i, (_, s, _) in enumerate(inst):
        off[i + 1] = off[i] + len(s)
    src = np.array([x for _, s, _ in inst for x in s], np.uint32)
    dst = np.array([x for _, _, d in inst for x in d], np.uint32)
    wl = gen.BatchWorkload("edge", nodes, off, src, dst)
    res = engine.tc_bool_batch(nodes, off, src, dst, mode=0)
    _check(res, wl, rounds_sample=len(inst))
    assert res.counts.tolist()[:6] == [0, 0, 1, 3, 200 * 200, 300 * 299 // 2]
    assert int(res.rounds[5]) == 299


def test_batch_rejects_ids_outside_instance(engine):
    with pytest.raises(S.InvalidArgument):
        engine.tc_bool_batch([3, 3], [0, 1, 2], [0, 1], [1, 3])
    with pytest.raises(S.InvalidArgument):
        engine.tc_bool_batch([3], [0, 5], [0, 1], [1, 2])


def test_batch_device_inputs(engine):
    import torch
    wl = gen.batch_tc_workload(n_inst=40, n_min=20, n_max=800, seed=24)
    ds = torch.from_numpy(wl.src.astype(np.int32)).cuda()
    dd = torch.from_numpy(wl.dst.astype(np.int32)).cuda()
    res = engine.tc_bool_batch(wl.nodes, wl.edge_off, ds, dd, mode=0)
    _check(res, wl, rounds_sample=4)


def test_bit_row_plan_selected_and_exclusive(engine):
    """Automatic planning uses bit rows for Bool closure; forcing them on a
    tropical program is an error, and forcing them on closure is exact."""
    s, d = gen.er_directed(3000, 9000, 31)
    a, b, r = O.fast_tc(s, d)
    got = engine.transitive_closure_bool((s, d))
    assert got.stats["plan"] == 3 and got.stats["rounds"] == r
    assert np.array_equal(got.src, a) and np.array_equal(got.dst, b)
    engine.set_plan(3)
    try:
        got3 = engine.transitive_closure_bool((s, d))
        assert np.array_equal(got3.src, a) and np.array_equal(got3.dst, b)
        with pytest.raises(S.Unsupported):
            engine.shortest_paths_trop([(0, 1, 1), (1, 2, 1)])
    finally:
        engine.set_plan(0)


@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_sharded_closure_ranks_on_one_gpu(engine, world):
    """The sharded closure's device rounds, with every rank's share run in
    this process (no rank waits on another; the Δ' slices are concatenated
    where ranks would all-gather them): count, fingerprint and rounds equal
    the oracle's and the single-device batch's, whether Δ' moves as whole
    slices, as packed nonzero words, or as the smaller of the two."""
    import torch

    from strata_b200 import shard
    for (n, m, seed), x in zip(((3000, 9000, 41), (777, 2500, 42), (129, 400, 43), (2000, 2600, 44)),
                               ("auto", "sparse", "dense", "auto")):
        s, d = gen.er_directed(n, m, seed)
        s, d = np.concatenate([s, s[:10]]), np.concatenate([d, d[:10]])  # duplicate edges
        c, f = O.closure_batch([n], [0, len(s)], s, d, threads=8)
        rounds = O.fast_tc(s, d)[2]
        ts = torch.from_numpy(s.astype(np.int32)).cuda()
        td = torch.from_numpy(d.astype(np.int32)).cuda()
        parts = [engine.tc_shard(n, ts, td, r, world) for r in range(world)]
        try:
            got = shard.tc_bool_sharded(parts, device="cuda", exchange=x)
        finally:
            for p in parts:
                p.free()
        assert got == (int(c[0]), int(f[0]), rounds), (n, world)
        one = engine.tc_bool_batch([n], [0, len(s)], s, d)
        assert (int(one.counts[0]), int(one.fps[0]), int(one.rounds[0])) == got


def test_sharded_closure_rejects_bad_input(engine):
    import torch
    ts = torch.tensor([0, 5], dtype=torch.int32, device="cuda")
    td = torch.tensor([1, 1], dtype=torch.int32, device="cuda")
    with pytest.raises(S.InvalidArgument):  # endpoint outside [0, n)
        engine.tc_shard(3, ts, td, 0, 2)
    with pytest.raises(S.InvalidArgument):  # rank >= world
        engine.tc_shard(8, ts, td, 2, 2)
    sh = engine.tc_shard(8, ts, td, 0, 2)
    try:
        per, _, _, rb = sh.shape()
        full = torch.zeros(2 * per * rb // 4, dtype=torch.int32, device="cuda")
        flags = torch.zeros(2 * per, dtype=torch.uint8, device="cuda")
        mine = torch.zeros(per * rb // 4, dtype=torch.int32, device="cuda")
        fmine = torch.zeros(per, dtype=torch.uint8, device="cuda")
        with pytest.raises(S.InvalidArgument):  # a round before the seed
            sh.round(full, flags, mine, fmine)
        with pytest.raises(S.InvalidArgument):  # a summary before the seed
            sh.summary()
        with pytest.raises(S.InvalidArgument):  # a pack before the seed
            sh.pack_count(mine)
        sh.seed(mine, fmine)
        assert sh.pack_count(mine) >= 1  # row 0 holds its edge to 1
        with pytest.raises(S.InvalidArgument):  # more nonzero words than the capacity
            sh.pack(mine, 0)
        trip = sh.pack(mine, sh.pack_count(mine) + 2)
        assert int((trip[:, 0] < 0).sum()) == 2  # padding
        with pytest.raises(S.InvalidArgument):  # triples inside the gathered Δ
            sh.unpack(full.view(torch.int64)[: 3 * 2].view(2, 3), full, flags)
        with pytest.raises(S.InvalidArgument):  # a second seed (its edge columns are gone)
            sh.seed(mine, fmine)
        with pytest.raises(S.InvalidArgument):  # the slice inside the gathered Δ
            sh.round(full, flags, full[: per * rb // 4], fmine)
        with pytest.raises(S.InvalidArgument):  # the row flags inside the gathered flags
            sh.round(full, flags, mine, flags[per:])
        assert sh.round(full, flags, mine, fmine) == 0  # an empty gathered Δ derives nothing
    finally:
        sh.free()
