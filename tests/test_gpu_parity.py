"""Parity of the CUDA engine (through the C ABI) with the CPU oracle.

Bit-exact for every relation, count and error: integers and Trop i64 weights
with a distinct +inf leave no tolerance to state.
"""
import numpy as np
import pytest

import oracle as O
import strata_b200 as S
from strata_b200 import gen

pytestmark = pytest.mark.gpu

I64_MAX = 2**63 - 1


def _pairs(rel):
    return list(zip(rel.src.tolist(), rel.dst.tolist()))


def _trop(rel):
    return [(a, b, O.POS_INF if i else w) for a, b, w, i in
            zip(rel.src.tolist(), rel.dst.tolist(), rel.w.tolist(), rel.inf.tolist())]


def _otrop(cols):
    s, d, w, i = cols[:4]
    return [(a, b, O.POS_INF if x else y) for a, b, y, x in zip(s.tolist(), d.tolist(), w.tolist(), i.tolist())]


# ------------------------------------------------------------------ Bool TC
@pytest.mark.parametrize("edges", [
    [(0, 1), (1, 2), (2, 3)], [(0, 1), (1, 0)], [(5, 5), (5, 5), (5, 6)], [],
])
def test_tc_fixed_cases(tceng, edges):
    engine = tceng
    got = engine.transitive_closure_bool(edges)
    s = [e[0] for e in edges]
    d = [e[1] for e in edges]
    a, b, _ = O.fast_tc(s, d)
    assert _pairs(got) == list(zip(a.tolist(), b.tolist()))


def test_tc_random_small(tceng, lcg):
    engine = tceng
    rng = lcg(0x123456789ABCDEF0)
    for trial in range(200):
        nodes = 3 + rng.upto(8)
        m = rng.upto(nodes * 2 + 1)
        edges = [(rng.upto(nodes), rng.upto(nodes)) for _ in range(m)]
        a, b, r = O.fast_tc([e[0] for e in edges], [e[1] for e in edges])
        got = engine.transitive_closure_bool(edges)
        assert _pairs(got) == list(zip(a.tolist(), b.tolist())), (trial, edges)
        if edges:
            assert got.stats["rounds"] == r


def test_tc_chain_400(tceng):
    engine = tceng
    n = 400
    got = engine.transitive_closure_bool((np.arange(n), np.arange(1, n + 1)))
    assert len(got) == (n + 1) * n // 2
    want = [(i, j) for i in range(n + 1) for j in range(i + 1, n + 1)]
    assert _pairs(got) == want
    assert got.stats["rounds"] == n


@pytest.mark.parametrize("n,m,seed", [(200, 600, 1), (2000, 6000, 2), (5000, 12000, 3)])
def test_tc_er_medium_exact(tceng, n, m, seed):
    engine = tceng
    s, d = gen.er_directed(n, m, seed)
    a, b, r = O.fast_tc(s, d)
    got = engine.transitive_closure_bool((s, d))
    assert np.array_equal(got.src, a) and np.array_equal(got.dst, b)
    assert got.stats["rounds"] == r


def test_tc_wide_keys(peng):
    """Ids above 2^16 force 64-bit packed keys."""
    engine = peng
    rng = np.random.default_rng(4)
    s = rng.integers(0, 1 << 31, 3000).astype(np.uint32)
    d = rng.choice(s, 3000).astype(np.uint32)
    a, b, _ = O.fast_tc(s, d)
    got = engine.transitive_closure_bool((s, d))
    assert got.stats["key_bits"] > 32
    assert np.array_equal(got.src, a) and np.array_equal(got.dst, b)


def test_tc_config_size_fingerprint(tceng):
    """ER(10 000, 50 000): count + fingerprint equal a per-source BFS closure."""
    engine = tceng
    w = gen.tc_workload()
    cnt, fp = O.bfs_closure(w.src, w.dst)
    import torch
    ds = torch.from_numpy(w.src.astype(np.int32)).cuda()
    dd = torch.from_numpy(w.dst.astype(np.int32)).cuda()
    rel = engine.tc_bool_dev(ds, dd)
    assert len(rel) == cnt
    assert rel.fingerprint() == fp
    host = engine.transitive_closure_bool((w.src, w.dst))
    assert len(host) == cnt and O.fingerprint(host.src, host.dst) == fp
    rel.free()


# ------------------------------------------------------------------ Trop all-pairs
def test_trop_fixed_case(peng):
    engine = peng
    got = engine.shortest_paths_trop([(0, 2, 10), (0, 1, 2), (1, 2, 3)])
    assert _trop(got) == [(0, 1, 2), (0, 2, 5), (1, 2, 3)]


def test_trop_random_small(peng, lcg):
    engine = peng
    rng = lcg(0xDEADBEEFCAFE1234)
    for trial in range(200):
        nodes = 3 + rng.upto(6)
        m = rng.upto(nodes * 2 + 1)
        edges = [(rng.upto(nodes), rng.upto(nodes), rng.upto(10)) for _ in range(m)]
        s, d, w = ([e[k] for e in edges] for k in range(3))
        want = O.fast_trop(0, s, d, w)
        got = engine.shortest_paths_trop(edges)
        assert _trop(got) == _otrop(want), (trial, edges)


def test_trop_weighted_chain_300(peng):
    engine = peng
    n = 300
    got = engine.shortest_paths_trop((np.arange(n), np.arange(1, n + 1), np.arange(1, n + 1)))
    want = []
    for i in range(n + 1):
        acc = 0
        for j in range(i + 1, n + 1):
            acc += j
            want.append((i, j, acc))
    assert _trop(got) == want


def test_trop_overflow_is_error(peng):
    engine = peng
    with pytest.raises(S.TropOverflow):
        engine.shortest_paths_trop([(0, 1, I64_MAX - 5), (1, 2, 6)])
    # the context stays usable afterwards
    assert _trop(engine.shortest_paths_trop([(0, 1, 1)])) == [(0, 1, 1)]


def test_trop_negative_cycle(peng):
    engine = peng
    with pytest.raises(S.NegativeWeightCycle):
        engine.shortest_paths_trop([(0, 1, 1), (1, 0, -2)])


def test_trop_pos_inf(peng):
    engine = peng
    got = engine.shortest_paths_trop([(0, 1, O.POS_INF), (1, 2, 4), (0, 2, O.POS_INF)])
    assert _trop(got) == [(0, 1, O.POS_INF), (0, 2, O.POS_INF), (1, 2, 4)]
    # a finite derivation improves a +inf tuple
    got = engine.shortest_paths_trop([(0, 1, 3), (1, 2, 4), (0, 2, O.POS_INF)])
    assert _trop(got) == [(0, 1, 3), (0, 2, 7), (1, 2, 4)]


@pytest.mark.parametrize("plan", [0, 1, 2], ids=["auto", "sortmerge", "dense"])
def test_trop_finite_i64_max_is_a_value(engine, plan):
    """Finite(i64::MAX) is a legal weight distinct from +inf
    (strata-ir/src/trop.rs:35-62): it is kept, ⊗ 0 keeps it, ⊗ 1 overflows."""
    engine.set_plan(plan)
    try:
        for edges in ([(0, 1, I64_MAX)], [(0, 1, I64_MAX), (1, 2, 0)],
                      [(0, 1, I64_MAX - 3), (1, 2, 3), (0, 3, O.POS_INF), (3, 2, 5)],
                      [(0, 1, I64_MAX), (1, 2, 0), (2, 0, 0)], [(0, 1, I64_MAX), (1, 2, 0), (2, 1, 0)]):
            s = [e[0] for e in edges]
            d = [e[1] for e in edges]
            w = [0 if e[2] == O.POS_INF else e[2] for e in edges]
            inf = [1 if e[2] == O.POS_INF else 0 for e in edges]
            try:
                want = O.fast_trop(0, s, d, w, np.array(inf, np.uint8))
            except O.OracleError as e:  # a cycle through i64::MAX overflows in the reference too
                assert e.kind == "overflow"
                with pytest.raises(S.TropOverflow):
                    engine.shortest_paths_trop(edges)
                continue
            got = engine.shortest_paths_trop(edges)
            assert _trop(got) == _otrop(want), edges
            assert got.stats["weight_bytes"] == 8
        with pytest.raises(S.TropOverflow):
            engine.shortest_paths_trop([(0, 1, I64_MAX), (1, 2, 1)])
        # MSSP: a source weight of 1 plus an edge of i64::MAX - 1 is finite i64::MAX
        got = engine.mssp_trop([0], [(0, 1, I64_MAX - 1), (1, 2, 0)], source_weights=[1])
        assert _trop(got) == [(0, 1, I64_MAX), (0, 2, I64_MAX)]
        with pytest.raises(S.TropOverflow):
            engine.mssp_trop([0], [(0, 1, I64_MAX - 1), (1, 2, 1)], source_weights=[1])
    finally:
        engine.set_plan(0)


def test_weight_lanes_knob_forces_int64_with_identical_results(engine):
    wl = gen.mssp_workload(scale=12, n_sources=16, seed=19)
    narrow = engine.mssp_trop(wl.sources, (wl.src, wl.dst, wl.w), source_weights=wl.source_w)
    engine.set_knob(9, 8)
    try:
        wide = engine.mssp_trop(wl.sources, (wl.src, wl.dst, wl.w), source_weights=wl.source_w)
    finally:
        engine.set_knob(9, 0)
    assert narrow.stats["weight_bytes"] == 4 and wide.stats["weight_bytes"] == 8
    assert wide.stats["plan"] == narrow.stats["plan"] == 2
    for a in ("src", "dst", "w", "inf"):
        assert np.array_equal(getattr(narrow, a), getattr(wide, a))
    assert narrow.stats["rounds"] == wide.stats["rounds"]
    with pytest.raises(S.InvalidArgument):
        engine.set_knob(9, 4)


def test_trop_weights_spanning_all_of_i64_are_refused(engine):
    """Sums that can reach both i64::MIN and i64::MAX within the round cap leave
    no 64-bit code for +inf: reported, never mixed up."""
    with pytest.raises(S.WeightRange):
        engine.shortest_paths_trop([(0, 1, I64_MAX), (1, 2, -2**63)])


@pytest.mark.parametrize("plan", [0, 1, 2], ids=["auto", "sortmerge", "dense"])
def test_mssp_wide_lanes_exact(engine, plan):
    """Weights too large for int32 lanes (U[1, 2^40]) on every plan: exact rows
    and rounds against the semi-naive restatement."""
    wl = gen.mssp_workload(scale=13, n_sources=32, seed=17)
    w = np.random.default_rng(18).integers(1, 1 << 40, len(wl.w), dtype=np.int64)
    want = O.fast_trop(1, wl.src, wl.dst, w, sources=wl.sources, source_w=wl.source_w)
    engine.set_plan(plan)
    try:
        got = engine.mssp_trop(wl.sources, (wl.src, wl.dst, w), source_weights=wl.source_w)
    finally:
        engine.set_plan(0)
    assert got.stats["weight_bytes"] == 8
    assert got.stats["plan"] == (1 if plan == 1 else 2)
    assert np.array_equal(got.src, want[0]) and np.array_equal(got.dst, want[1])
    assert np.array_equal(got.w, want[2]) and not got.inf.any()
    assert got.stats["rounds"] == want[4]


@pytest.mark.parametrize("scale_w", [100, 10**12])
def test_trop_medium_narrow_and_wide(peng, scale_w):
    """Small weights run in int32 lanes, huge ones in int64 lanes: same answers."""
    engine = peng
    rng = np.random.default_rng(11)
    n, m = 300, 1500
    s = rng.integers(0, n, m)
    d = rng.integers(0, n, m)
    w = rng.integers(0, scale_w, m)
    want = O.fast_trop(0, s, d, w)
    got = engine.shortest_paths_trop((s, d, w))
    assert got.stats["weight_bytes"] == (4 if scale_w == 100 else 8)
    assert _trop(got) == _otrop(want)
    assert got.stats["rounds"] == want[4]


def test_trop_negative_weights_no_cycle(peng):
    engine = peng
    rng = np.random.default_rng(12)
    n = 60
    s = rng.integers(0, n, 200)
    d = rng.integers(0, n, 200)
    keep = s < d  # a DAG: negative weights but no cycle
    s, d = s[keep], d[keep]
    w = rng.integers(-50, 50, len(s))
    want = O.fast_trop(0, s, d, w)
    assert _trop(engine.shortest_paths_trop((s, d, w))) == _otrop(want)


# ------------------------------------------------------------------ MSSP (bench shape)
def test_mssp_random_small(peng):
    engine = peng
    rng = np.random.default_rng(7)
    for trial in range(60):
        n = int(rng.integers(4, 14))
        m = int(rng.integers(1, 3 * n))
        s = rng.integers(0, n, m)
        d = rng.integers(0, n, m)
        w = rng.integers(0, 9, m)
        srcs = rng.integers(0, n, 3)
        sw = rng.integers(0, 5, 3)
        want = O.fast_trop(1, s, d, w, sources=srcs, source_w=sw)
        got = engine.mssp_trop(srcs, (s, d, w), source_weights=sw)
        assert _trop(got) == _otrop(want), trial
        assert got.stats["rounds"] == want[4]


def test_mssp_rmat_scale12_exact(peng):
    engine = peng
    wl = gen.mssp_workload(scale=12, n_sources=64, seed=5)
    want = O.fast_trop(1, wl.src, wl.dst, wl.w, sources=wl.sources, source_w=wl.source_w)
    got = engine.mssp_trop(wl.sources, (wl.src, wl.dst, wl.w), source_weights=wl.source_w)
    assert np.array_equal(got.src, want[0]) and np.array_equal(got.dst, want[1])
    assert np.array_equal(got.w, want[2]) and not got.inf.any()
    assert got.stats["rounds"] == want[4]


@pytest.mark.parametrize("members", [1, 20, 33])
def test_mssp_dense_word_paths_identical(engine, members):
    """Direct-addressed rounds: the bit-lane path for dense Δ words (from 1
    member: every word; 33: none) gives the oracle's relation and rounds,
    with sources spread over both marks words of an index row."""
    wl = gen.mssp_workload(scale=13, n_sources=64, seed=8)
    want = O.fast_trop(1, wl.src, wl.dst, wl.w, sources=wl.sources, source_w=wl.source_w)
    engine.set_plan(2)
    engine.set_knob(8, members)
    try:
        got = engine.mssp_trop(wl.sources, (wl.src, wl.dst, wl.w), source_weights=wl.source_w)
        assert np.array_equal(got.src, want[0]) and np.array_equal(got.dst, want[1])
        assert np.array_equal(got.w, want[2])
        assert got.stats["rounds"] == want[4] and got.stats["plan"] == 2
        # Bool closure on the direct-addressed index (rows padded to 32 columns)
        s, d = gen.er_directed(777, 3000, members)
        a, b, r = O.fast_tc(s, d)
        tc = engine.transitive_closure_bool((s, d))
        assert np.array_equal(tc.src, a) and np.array_equal(tc.dst, b) and tc.stats["rounds"] == r
    finally:
        engine.set_knob(8, 0)
        engine.set_plan(0)
    with pytest.raises(S.InvalidArgument):
        engine.set_knob(8, 34)


def test_mssp_rmat_scale16_matches_dijkstra(peng):
    engine = peng
    import torch
    wl = gen.mssp_workload(scale=16, n_sources=64, seed=6)
    cnt, fp = O.dijkstra_mssp(wl.sources, wl.src, wl.dst, wl.w, wl.source_w)
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a).astype(dt)).cuda()
    rel = engine.mssp_dev(t(wl.sources, np.int32), t(wl.src, np.int32), t(wl.dst, np.int32),
                          t(wl.w, np.int64), source_weights=t(wl.source_w, np.int64))
    assert len(rel) == cnt
    assert rel.fingerprint() == fp
    rel.free()


def test_mssp_overflow(peng):
    engine = peng
    with pytest.raises(S.TropOverflow):
        engine.mssp_trop([0], [(0, 1, 5), (1, 2, I64_MAX - 2)])


# ------------------------------------------------------------------ WCOJ counts
def test_triangles_fixed_and_complete(engine):
    k4 = [(0, 1), (1, 0), (0, 2), (0, 3), (1, 2), (2, 3), (1, 3), (1, 3), (2, 2)]
    assert engine.count_triangles(k4) == 4
    assert engine.count_triangles([]) == 0
    assert engine.count_triangles([(0, 1), (1, 2), (0, 2)]) == 1
    for n in (3, 10, 30, 64):
        e = [(a, b) for a in range(n) for b in range(a + 1, n)]
        assert engine.count_triangles(e) == n * (n - 1) * (n - 2) // 6


def test_triangles_random_vs_brute(engine, lcg):
    rng = lcg(0x7EA12345678)
    for trial in range(200):
        n = 5 + rng.upto(30)
        m = rng.upto(n * 3)
        e = np.array([(rng.upto(n), rng.upto(n)) for _ in range(m)]).reshape(-1, 2)
        assert engine.count_triangles(e) == O.brute_triangles(e[:, 0], e[:, 1], n), trial


def test_triangle_pattern_random(engine):
    rng = np.random.default_rng(21)
    for trial in range(40):
        n = int(rng.integers(5, 300))
        m = int(rng.integers(1, 8 * n))
        x = rng.integers(0, n, m)
        y = rng.integers(0, n, m)
        assert engine.count_triangle_pattern((x, y)) == O.count_pattern(x, y), trial


def test_triangle_pattern_rmat_oriented(engine):
    wl = gen.triangle_workload(scale=14, edge_factor=16, seed=9)
    want = O.count_pattern(wl.src, wl.dst)
    assert engine.count_triangle_pattern((wl.src, wl.dst)) == want
    # the undirected entry point orients internally and agrees
    assert engine.count_triangles((wl.src, wl.dst)) == want


@pytest.mark.parametrize("probe", [1, 2, 3])
def test_triangle_probe_knob(engine, probe):
    """Every membership test (shared-memory hash set, binary search, bitmap
    filter with queued searches) gives the oracle's count, including a vertex
    whose out-list exceeds the staged list (it falls back to the binary
    search), R-MAT skew and a dense graph whose warps fill the search queue
    many times over."""
    engine.set_knob(3, probe)
    try:
        big = 3000  # X=0 -> 1..3000, i -> i+1: 2999 triangles through the wide vertex
        x = np.concatenate([np.zeros(big, np.int64), np.arange(1, big)])
        y = np.concatenate([np.arange(1, big + 1), np.arange(2, big + 1)])
        assert engine.count_triangle_pattern((x, y)) == O.count_pattern(x, y) == big - 1
        wl = gen.triangle_workload(scale=13, edge_factor=16, seed=4)
        assert engine.count_triangle_pattern((wl.src, wl.dst)) == O.count_pattern(wl.src, wl.dst)
        rng = np.random.default_rng(probe)
        a, b = rng.integers(0, 400, 40_000), rng.integers(0, 400, 40_000)
        assert engine.count_triangle_pattern((a, b)) == O.count_pattern(a, b)
        for _ in range(10):
            n = int(rng.integers(5, 2000))
            m = int(rng.integers(1, 20 * n))
            a, b = rng.integers(0, n, m), rng.integers(0, n, m)
            assert engine.count_triangle_pattern((a, b)) == O.count_pattern(a, b)
    finally:
        engine.set_knob(3, 0)


def test_hub_graph_closed_form(engine):
    h, b = 16, 20000
    e = [(i, j) for i in range(h) for j in range(i + 1, h)]
    e += [(hub, h + k) for k in range(b) for hub in range(h)]
    a = np.array(e)
    want = b * h * (h - 1) // 2 + h * (h - 1) * (h - 2) // 6
    assert engine.count_triangles(a) == want


def test_4cliques(engine, lcg):
    assert engine.count_4cliques([(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]) == 1
    assert engine.count_4cliques([(0, 1), (1, 2), (0, 2)]) == 0
    for n in (4, 10, 20, 40):
        e = [(a, b) for a in range(n) for b in range(a + 1, n)]
        assert engine.count_4cliques(e) == n * (n - 1) * (n - 2) * (n - 3) // 24
    # a wide vertex (oriented out-degree above the small launch's 512-entry
    # lists) goes through the second launch: K_600 has C(600, 4) 4-cliques
    n = 600
    e = np.stack(np.triu_indices(n, 1), 1)
    assert engine.count_4cliques(e) == n * (n - 1) * (n - 2) * (n - 3) // 24
    # K_40 planted in a random sparse graph, checked by brute force
    rng0 = np.random.default_rng(44)
    sp = rng0.integers(0, 300, (1500, 2))
    e = np.concatenate([np.stack(np.triu_indices(40, 1), 1) * 7, sp])
    assert engine.count_4cliques(e) == O.brute_4cliques(e[:, 0], e[:, 1], 300)
    rng = lcg(0x4C19999)
    for trial in range(100):
        n = 6 + rng.upto(18)
        m = rng.upto(n * 4)
        e = np.array([(rng.upto(n), rng.upto(n)) for _ in range(m)]).reshape(-1, 2)
        assert engine.count_4cliques(e) == O.brute_4cliques(e[:, 0], e[:, 1], n), trial


def test_binary_plan_intermediate(engine):
    rng = np.random.default_rng(3)
    e = rng.integers(0, 50, (400, 2))
    lo, hi = np.minimum(e[:, 0], e[:, 1]), np.maximum(e[:, 0], e[:, 1])
    keep = lo != hi
    pairs = np.unique(np.stack([lo[keep], hi[keep]], 1), axis=0)
    deg = np.bincount(pairs[:, 0], minlength=50)
    assert engine.binary_plan_intermediate(e) == int((deg.astype(np.int64) ** 2).sum())


def test_intern_terms(engine):
    """Equal keys get equal ids, ids are dense ranks (strata-gpu/tests/intern_diff.rs:24-63)."""
    rng = np.random.default_rng(5)
    keys = rng.integers(0, 2**63, 5000, dtype=np.uint64)
    keys = np.concatenate([keys, keys[:1000]])
    rng.shuffle(keys)
    ids = engine.intern_terms(keys)
    uniq = np.unique(keys)
    assert np.array_equal(ids, np.searchsorted(uniq, keys).astype(np.uint32))


# ------------------------------------------------------------------ operator surface
def _dev(a, dtype):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(dtype)).cuda()


@pytest.mark.parametrize("n", [0, 1, 3839, 3840, 3841, 2303, 2304, 2305, 200_003])
@pytest.mark.parametrize("kb,vb", [(4, 0), (4, 4), (4, 8), (8, 0), (8, 8)])
def test_op_sort_stable(engine, n, kb, vb):
    import ctypes as C
    import torch
    rng = np.random.default_rng(n + kb + vb)
    kdt = np.uint32 if kb == 4 else np.uint64
    bits = 27 if kb == 4 else 45
    keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(kdt)
    vals = np.arange(n, dtype=np.uint32 if vb == 4 else np.uint64) if vb else None
    tdt = torch.int32 if kb == 4 else torch.int64
    ki = _dev(keys, np.int32 if kb == 4 else np.int64)
    ko = torch.empty(max(n, 1), dtype=tdt, device="cuda")
    vi = _dev(vals, np.int32 if vb == 4 else np.int64) if vb else None
    vo = torch.empty(max(n, 1), dtype=torch.int32 if vb == 4 else torch.int64, device="cuda") if vb else None
    rc = engine.lib.strata_op_sort(engine.ctx, kb, vb, C.c_void_p(ki.data_ptr() if n else 0),
                                   C.c_void_p(vi.data_ptr() if vb and n else 0), C.c_void_p(ko.data_ptr()),
                                   C.c_void_p(vo.data_ptr() if vb else 0), n, bits)
    engine._check(rc)
    order = np.argsort(keys, kind="stable")
    got = ko.cpu().numpy().view(kdt)[:n]
    assert np.array_equal(got, keys[order])
    if vb:
        assert np.array_equal(vo.cpu().numpy().view(vals.dtype)[:n], vals[order])


def test_op_sort_beyond_2_30_keys(engine):
    """A sort of 2^30 + 4,097 keys whose most frequent digit occurs more than
    2^30 times (the look-back then needs its 64-bit words): keys and the
    values riding along come out in stable order."""
    import ctypes as C
    import torch
    n = (1 << 30) + 4097
    tail = 100
    keys = torch.zeros(n, dtype=torch.int32, device="cuda")
    keys[n - tail:] = torch.arange(tail, dtype=torch.int32, device="cuda") % 4
    vals = torch.arange(n, dtype=torch.int32, device="cuda")
    ko, vo = torch.empty_like(keys), torch.empty_like(vals)
    engine._check(engine.lib.strata_op_sort(engine.ctx, 4, 4, C.c_void_p(keys.data_ptr()), C.c_void_p(vals.data_ptr()),
                                            C.c_void_p(ko.data_ptr()), C.c_void_p(vo.data_ptr()), n, 2))
    j = torch.arange(tail, dtype=torch.int32, device="cuda")
    want_v = torch.cat([torch.arange(n - tail, dtype=torch.int32, device="cuda")] +
                       [(n - tail + j[j % 4 == d]).to(torch.int32) for d in range(4)])
    want_k = torch.cat([torch.zeros(n - tail + 25, dtype=torch.int32, device="cuda")] +
                       [torch.full((25,), d, dtype=torch.int32, device="cuda") for d in (1, 2, 3)])
    assert int((want_k == 0).sum()) > (1 << 30)
    assert torch.equal(ko, want_k)
    assert torch.equal(vo, want_v)
    del keys, vals, ko, vo, want_v, want_k
    torch.cuda.empty_cache()
    small = torch.zeros(16, dtype=torch.int32, device="cuda")
    with pytest.raises(S.InvalidArgument):  # past 2^32 - 1 keys (refused before any key is read)
        engine._check(engine.lib.strata_op_sort(engine.ctx, 4, 0, C.c_void_p(small.data_ptr()), None,
                                                C.c_void_p(small.data_ptr()), None, 1 << 32, 32))


def test_op_dedup_diff_and_min_improve(engine):
    import ctypes as C
    import torch
    rng = np.random.default_rng(8)
    cand = np.sort(rng.integers(0, 5000, 20000).astype(np.uint32))
    full = np.unique(rng.integers(0, 5000, 3000).astype(np.uint32))
    out = torch.empty(len(cand), dtype=torch.int32, device="cuda")
    n = C.c_uint64()
    cand_d, full_d = _dev(cand, np.int32), _dev(full, np.int32)  # kept alive across the calls
    engine._check(engine.lib.strata_op_dedup_diff(engine.ctx, 4, C.c_void_p(cand_d.data_ptr()),
                                                  len(cand), C.c_void_p(full_d.data_ptr()), len(full),
                                                  C.c_void_p(out.data_ptr()), C.byref(n)))
    want = np.setdiff1d(np.unique(cand), full)
    assert np.array_equal(out.cpu().numpy().view(np.uint32)[:n.value], want)
    # Trop: min per key, keep new or strictly better, improve full in place
    cw = rng.integers(0, 100, len(cand)).astype(np.int64)
    fw = rng.integers(0, 100, len(full)).astype(np.int64)
    fw_dev = _dev(fw, np.int64)
    cw_d = _dev(cw, np.int64)
    ok = torch.empty(len(cand), dtype=torch.int32, device="cuda")
    ow = torch.empty(len(cand), dtype=torch.int64, device="cuda")
    engine._check(engine.lib.strata_op_min_improve(
        engine.ctx, 4, C.c_void_p(cand_d.data_ptr()), C.c_void_p(cw_d.data_ptr()),
        len(cand), C.c_void_p(full_d.data_ptr()), C.c_void_p(fw_dev.data_ptr()), len(full),
        C.c_void_p(ok.data_ptr()), C.c_void_p(ow.data_ptr()), C.byref(n)))
    best = {}
    for k, w in zip(cand.tolist(), cw.tolist()):
        best[k] = min(w, best.get(k, w))
    fmap = dict(zip(full.tolist(), fw.tolist()))
    want_rows = [(k, w) for k, w in sorted(best.items()) if k not in fmap or w < fmap[k]]
    got_rows = list(zip(ok.cpu().numpy().view(np.uint32)[:n.value].tolist(), ow.cpu().numpy()[:n.value].tolist()))
    assert got_rows == want_rows
    new_fw = {k: min(v, best.get(k, v)) for k, v in fmap.items()}
    assert fw_dev.cpu().numpy().tolist() == [new_fw[k] for k in full.tolist()]


def test_op_merge(engine):
    import ctypes as C
    import torch
    rng = np.random.default_rng(9)
    allk = rng.permutation(100000)[:30000].astype(np.uint64)
    a = np.sort(allk[:20000])
    b = np.sort(allk[20000:])
    out = torch.empty(len(allk), dtype=torch.int64, device="cuda")
    a_d, b_d = _dev(a, np.int64), _dev(b, np.int64)  # kept alive across the call
    engine._check(engine.lib.strata_op_merge(engine.ctx, 8, C.c_void_p(a_d.data_ptr()), None, len(a),
                                             C.c_void_p(b_d.data_ptr()), None, len(b),
                                             C.c_void_p(out.data_ptr()), None))
    assert np.array_equal(out.cpu().numpy().view(np.uint64), np.sort(allk))


def test_launch_counter_and_memory_returned(engine):
    before = engine.launches()
    engine.transitive_closure_bool([(0, 1), (1, 2)])
    assert engine.launches() > before
    in_use, peak = engine.mem()
    assert in_use == 0 and peak > 0


def test_plans_pick_and_agree(engine):
    """Automatic planning picks the direct-addressed plan for the benchmark
    shapes; forcing sort-merge gives the same relation and round count."""
    wl = gen.mssp_workload(scale=11, n_sources=32, seed=8)
    res = {}
    for plan in (0, 1, 2):
        engine.set_plan(plan)
        r = engine.mssp_trop(wl.sources, (wl.src, wl.dst, wl.w), source_weights=wl.source_w)
        res[plan] = r
    engine.set_plan(0)
    assert res[0].stats["plan"] == 2 and res[1].stats["plan"] == 1 and res[2].stats["plan"] == 2
    for p in (1, 2):
        assert np.array_equal(res[0].src, res[p].src) and np.array_equal(res[0].dst, res[p].dst)
        assert np.array_equal(res[0].w, res[p].w) and res[0].stats["rounds"] == res[p].stats["rounds"]
    # wide weights use the direct-addressed plan with int64 lanes
    engine.set_plan(2)
    got = engine.shortest_paths_trop([(0, 1, 10**13), (1, 2, 1)])
    assert got.stats["plan"] == 2 and got.stats["weight_bytes"] == 8
    assert _trop(got) == [(0, 1, 10**13), (0, 2, 10**13 + 1), (1, 2, 1)]
    engine.set_plan(0)
    assert engine.shortest_paths_trop([(0, 1, 10**13), (1, 2, 1)]).stats["plan"] == 2


@pytest.mark.parametrize("kb,choices", [(4, (11, 15, 19, 23)), (8, (7, 9, 13))])
def test_sort_knobs_identical(engine, kb, choices):
    """Every keys-per-thread choice of the radix tile sorts identically
    (stable, with values) on sizes that end mid-tile for every choice."""
    import ctypes as C
    import torch
    knob = 1 if kb == 4 else 2
    for n in (1, 4097, 300_001):
        rng = np.random.default_rng(n + kb)
        kdt = np.uint32 if kb == 4 else np.uint64
        bits = 26 if kb == 4 else 41
        keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(kdt)
        keys[: n // 3] = keys[0]  # a long run of one key (histogram fast path)
        vals = np.arange(n, dtype=np.uint32)
        order = np.argsort(keys, kind="stable")
        ki, vi = _dev(keys, np.int32 if kb == 4 else np.int64), _dev(vals, np.int32)
        for v in choices:
            engine.set_knob(knob, v)
            ko, vo = torch.empty_like(ki), torch.empty_like(vi)
            engine._check(engine.lib.strata_op_sort(engine.ctx, kb, 4, C.c_void_p(ki.data_ptr()),
                                                    C.c_void_p(vi.data_ptr()), C.c_void_p(ko.data_ptr()),
                                                    C.c_void_p(vo.data_ptr()), n, bits))
            assert np.array_equal(ko.cpu().numpy().view(kdt), keys[order]), v
            assert np.array_equal(vo.cpu().numpy().view(np.uint32), vals[order]), v
    engine.set_knob(knob, 0)
    with pytest.raises(S.InvalidArgument):
        engine.set_knob(knob, 12)
    with pytest.raises(S.InvalidArgument):
        engine.set_knob(99, 0)


def test_sort_knobs_fixpoint_identical(engine):
    """A sort-merge fixpoint gives the same relation under every knob value."""
    wl = gen.mssp_workload(scale=10, n_sources=8, seed=5)
    engine.set_plan(1)
    base = engine.mssp_trop(wl.sources, (wl.src, wl.dst, wl.w), source_weights=wl.source_w)
    for v in (11, 19, 23):
        engine.set_knob(1, v)
        r = engine.mssp_trop(wl.sources, (wl.src, wl.dst, wl.w), source_weights=wl.source_w)
        assert np.array_equal(base.src, r.src) and np.array_equal(base.dst, r.dst)
        assert np.array_equal(base.w, r.w)
    engine.set_knob(1, 0)
    engine.set_plan(0)


@pytest.mark.parametrize("rank", [1, 2, 3])
def test_sort_rank_methods_identical(engine, rank):
    """Ballot, match-instruction and shared-mask digit ranking sort identically (stable)."""
    import ctypes as C
    engine.set_knob(7, rank)
    try:
        for n, kb, bits in ((5000, 4, 27), (300_001, 4, 26), (70_001, 8, 45)):
            rng = np.random.default_rng(n + rank)
            kdt = np.uint32 if kb == 4 else np.uint64
            keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(kdt)
            keys[: n // 4] = keys[1]
            vals = np.arange(n, dtype=np.uint32)
            order = np.argsort(keys, kind="stable")
            ki, vi = _dev(keys, np.int32 if kb == 4 else np.int64), _dev(vals, np.int32)
            import torch
            ko, vo = torch.empty_like(ki), torch.empty_like(vi)
            engine._check(engine.lib.strata_op_sort(engine.ctx, kb, 4, C.c_void_p(ki.data_ptr()),
                                                    C.c_void_p(vi.data_ptr()), C.c_void_p(ko.data_ptr()),
                                                    C.c_void_p(vo.data_ptr()), n, bits))
            assert np.array_equal(ko.cpu().numpy().view(kdt), keys[order])
            assert np.array_equal(vo.cpu().numpy().view(np.uint32), vals[order])
    finally:
        engine.set_knob(7, 0)


def test_triangle_pattern_vertex_ranges_add_up(engine):
    """Shares of the source-vertex range (one per rank) add up to the count."""
    import torch
    wl = gen.triangle_workload(scale=12, edge_factor=16, seed=12)
    x = torch.from_numpy(wl.src.astype(np.int32)).cuda()
    y = torch.from_numpy(wl.dst.astype(np.int32)).cuda()
    n = int(max(wl.src.max(), wl.dst.max())) + 1
    total = engine.count_triangle_pattern_dev(x, y)
    assert total == O.count_pattern(wl.src, wl.dst)
    for world in (2, 3, 8):
        parts = [engine.count_triangle_pattern_range_dev(x, y, n * r // world, n * (r + 1) // world)
                 for r in range(world)]
        assert sum(parts) == total
    assert engine.count_triangle_pattern_range_dev(x, y, 5, 5) == 0
