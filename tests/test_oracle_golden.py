"""CPU checks of the oracle against the reference's own known answers.

Every constant here is a golden value from the reference's tests or workloads
(file:line in each test's docstring).  These tests pin the oracle before it is
trusted as the checker of the CUDA engine.
"""
import itertools
import json
from pathlib import Path

import numpy as np
import pytest

import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"


def _pairs(db_rows):
    return [t for t, _ in db_rows]


def _set_fixpoint(edges):
    """Closure by repeated composition (strata-gpu/tests/tc_diff.rs:12-29)."""
    s = set(edges)
    while True:
        add = {(x, z) for (x, y) in s for (y2, z) in s if y2 == y} - s
        if not add:
            return sorted(s)
        s |= add


def _floyd(edges, n):
    """Floyd–Warshall with the `reach` convention (trop_diff.rs:14-45)."""
    INF = None
    d = [[INF] * n for _ in range(n)]
    for x, y, w in edges:
        if d[x][y] is None or w < d[x][y]:
            d[x][y] = w
    for k in range(n):
        for i in range(n):
            if d[i][k] is None:
                continue
            for j in range(n):
                if d[k][j] is not None and (d[i][j] is None or d[i][k] + d[k][j] < d[i][j]):
                    d[i][j] = d[i][k] + d[k][j]
    return sorted((i, j, d[i][j]) for i in range(n) for j in range(n) if d[i][j] is not None)


# ---------------------------------------------------------------- Bool TC
def test_chain_closure_interp_naive_and_semi():
    """a→b→c→d closes to 6 pairs (strata-eval/tests/interp.rs:61-114)."""
    p = O.tc_program([0, 1, 2], [1, 2, 3])
    semi, rounds = p.run(semi_naive=True)
    naive, _ = p.run(semi_naive=False)
    want = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
    assert _pairs(semi["path"]) == want
    assert semi == naive
    a, b, r = O.fast_tc([0, 1, 2], [1, 2, 3])
    assert list(zip(a.tolist(), b.tolist())) == want and r == rounds


@pytest.mark.parametrize("edges", [
    [(0, 1), (1, 0)],             # 2-cycle closes to the full 2×2 (tc_diff.rs:54-56)
    [(5, 5), (5, 5), (5, 6)],     # self-loop + duplicates (tc_diff.rs:58-60)
    [],                           # empty (tc_diff.rs:62-66)
])
def test_tc_fixed_cases(edges):
    s = [e[0] for e in edges]
    d = [e[1] for e in edges]
    db, _ = O.tc_program(s, d).run()
    assert _pairs(db["path"]) == _set_fixpoint(edges)
    a, b, _ = O.fast_tc(s, d)
    assert list(zip(a.tolist(), b.tolist())) == _set_fixpoint(edges)


def test_tc_random_matches_set_fixpoint(lcg):
    """200 random graphs on 3..10 nodes (tc_diff.rs:69-84), interpreter and fast path."""
    rng = lcg(0x123456789ABCDEF0)
    for trial in range(200):
        nodes = 3 + rng.upto(8)
        m = rng.upto(nodes * 2 + 1)
        edges = [(rng.upto(nodes), rng.upto(nodes)) for _ in range(m)]
        want = _set_fixpoint(edges)
        s, d = [e[0] for e in edges], [e[1] for e in edges]
        db, _ = O.tc_program(s, d).run()
        assert _pairs(db["path"]) == want, trial
        a, b, _ = O.fast_tc(s, d)
        assert list(zip(a.tolist(), b.tolist())) == want, trial


def test_chain_400_closed_form():
    """A 400-edge chain closes to {(i,j): i<j} in 400 rounds (tc_diff.rs:86-102)."""
    n = 400
    a, b, rounds = O.fast_tc(np.arange(n), np.arange(1, n + 1))
    assert len(a) == (n + 1) * n // 2
    want = [(i, j) for i in range(n + 1) for j in range(i + 1, n + 1)]
    assert list(zip(a.tolist(), b.tolist())) == want
    assert rounds == n  # the last round finds nothing new
    cnt, fp = O.bfs_closure(np.arange(n), np.arange(1, n + 1))
    assert cnt == len(a) and fp == O.fingerprint(a, b)


def test_interp_chain_40_rounds_match_fast():
    n = 40
    db, rounds = O.tc_program(np.arange(n), np.arange(1, n + 1)).run()
    a, b, r2 = O.fast_tc(np.arange(n), np.arange(1, n + 1))
    assert _pairs(db["path"]) == list(zip(a.tolist(), b.tolist()))
    assert rounds == r2


# ---------------------------------------------------------------- Trop
def test_trop_fixed_case():
    """min(10, 2+3) = 5 (trop_diff.rs:69-81; strata-cli/src/main.rs:605-618)."""
    p = O.trop_paths_program([0, 0, 1], [2, 1, 2], [10, 2, 3])
    db, _ = p.run()
    assert ((0, 2), 5) in db["reach"]
    assert [(t[0], t[1], w) for t, w in db["reach"]] == _floyd([(0, 2, 10), (0, 1, 2), (1, 2, 3)], 3)
    s, d, w, inf, _ = O.fast_trop(0, [0, 0, 1], [2, 1, 2], [10, 2, 3])
    assert list(zip(s.tolist(), d.tolist(), w.tolist())) == [(0, 1, 2), (0, 2, 5), (1, 2, 3)]


def test_trop_random_matches_floyd_warshall(lcg):
    """200 random non-negative graphs on 3..8 nodes (trop_diff.rs:84-101)."""
    rng = lcg(0xDEADBEEFCAFE1234)
    for trial in range(200):
        nodes = 3 + rng.upto(6)
        m = rng.upto(nodes * 2 + 1)
        edges = [(rng.upto(nodes), rng.upto(nodes), rng.upto(10)) for _ in range(m)]
        n = 1 + max((max(x, y) for x, y, _ in edges), default=-1)
        want = _floyd(edges, n)
        s = [e[0] for e in edges]
        d = [e[1] for e in edges]
        w = [e[2] for e in edges]
        db, _ = O.trop_paths_program(s, d, w).run()
        assert [(t[0], t[1], x) for t, x in db["reach"]] == want, trial
        fs, fd, fw, fi, _ = O.fast_trop(0, s, d, w)
        assert list(zip(fs.tolist(), fd.tolist(), fw.tolist())) == want, trial


def test_weighted_chain_300_closed_form():
    """Edge i→i+1 of weight i+1: reach(i,j) = Σ_{k=i+1..j} k (trop_diff.rs:103-118)."""
    n = 300
    s, d, w, inf, _ = O.fast_trop(0, np.arange(n), np.arange(1, n + 1), np.arange(1, n + 1))
    want = []
    for i in range(n + 1):
        acc = 0
        for j in range(i + 1, n + 1):
            acc += j
            want.append((i, j, acc))
    assert list(zip(s.tolist(), d.tolist(), w.tolist())) == want
    assert not inf.any()


def test_trop_overflow_is_error_not_wrap():
    """i64::MAX + 1 is EvalError::Overflow in both engines (interp.rs:173-209)."""
    p = O.trop_paths_program([0, 1], [1, 2], [2**63 - 1, 1])
    for semi in (True, False):
        with pytest.raises(O.OracleError) as e:
            p.run(semi_naive=semi)
        assert e.value.kind == "overflow"
    with pytest.raises(O.OracleError) as e:
        O.fast_trop(0, [0, 1], [1, 2], [2**63 - 1, 1])
    assert e.value.kind == "overflow"


def test_negative_weight_cycle_detected():
    """a→b (1), b→a (-2) diverges (interp.rs:407-446)."""
    p = O.trop_paths_program([0, 1], [1, 0], [1, -2])
    for semi in (True, False):
        with pytest.raises(O.OracleError) as e:
            p.run(semi_naive=semi)
        assert e.value.kind == "negative_cycle"
    with pytest.raises(O.OracleError) as e:
        O.fast_trop(0, [0, 1], [1, 0], [1, -2])
    assert e.value.kind == "negative_cycle"


def test_pos_inf_weights_absorb():
    """+inf ⊗ x = +inf and min(x, +inf) = x (strata-ir/src/trop.rs:136-175)."""
    s, d, w, inf = [0, 1, 0], [1, 2, 2], [0, 4, 0], [1, 0, 1]
    db, _ = O.trop_paths_program(s, d, w, inf).run()
    got = {t: x for t, x in db["reach"]}
    assert got[(0, 1)] == O.POS_INF and got[(1, 2)] == 4 and got[(0, 2)] == O.POS_INF
    fs, fd, fw, fi, _ = O.fast_trop(0, s, d, w, inf)
    assert [(a, b, O.POS_INF if i else x) for a, b, x, i in zip(fs.tolist(), fd.tolist(), fw.tolist(), fi.tolist())] \
        == [(0, 1, O.POS_INF), (0, 2, O.POS_INF), (1, 2, 4)]


def test_mssp_shape_interp_matches_fast_and_dijkstra():
    rng = np.random.default_rng(7)
    for trial in range(40):
        n = int(rng.integers(4, 12))
        m = int(rng.integers(0, 3 * n))
        s = rng.integers(0, n, m)
        d = rng.integers(0, n, m)
        w = rng.integers(0, 9, m)
        srcs = np.unique(rng.integers(0, n, 3))
        db, r1 = O.mssp_program(srcs, s, d, w).run()
        fs, fd, fw, fi, r2 = O.fast_trop(1, s, d, w, sources=srcs)
        assert [(t[0], t[1], x) for t, x in db["dist"]] == list(zip(fs.tolist(), fd.tolist(), fw.tolist())), trial
        assert r1 == r2
        c, fp = O.dijkstra_mssp(srcs, s, d, w)
        assert c == len(fs) and fp == O.fingerprint(fs, fd, fw, fi), trial
        rs, rd, rw = O.dijkstra_mssp_rows(srcs, s, d, w)
        assert np.array_equal(rs, fs) and np.array_equal(rd, fd) and np.array_equal(rw, fw), trial


def test_routing_workload_pinned_lines():
    """The routing workload prints route(n0_0, n7_7) = 5, … (strata-cli/tests/workloads.rs:26-32)."""
    from strata_b200.textio import SymbolDict, load_tsv, render_db
    g = json.loads((GOLDEN / "routing.json").read_text())
    sd = SymbolDict()
    # The plain queries are interned at check time, before the TSV
    # (strata-check/src/lib.rs:418-437).
    for a, b in g["queries"]:
        sd.intern(a), sd.intern(b)
    (s, d), w = load_tsv(g["rows"], 2, sd, trop=True)
    db, _ = O.trop_paths_program(s, d, w).run()
    rows = db["reach"]
    cols = [np.array([t[0] for t, _ in rows]), np.array([t[1] for t, _ in rows])]
    ws = np.array([x for _, x in rows])
    out = render_db({"route": (cols, ws, np.zeros(len(ws)))}, sd,
                    queries=[("route", q) for q in g["queries"]])
    assert out.splitlines() == g["pinned"]


# ---------------------------------------------------------------- counts
def test_stratified_negation_complement():
    """reach(Y) :- edge(X,Y), reach(X).  unreach(X) :- node(X), not reach(X).
    with nodes a, b, c, edge(a, b), reach(a): only c is unreachable and reach
    saturates to {a, b} (strata-eval/tests/interp.rs:241-293; symbols
    interned first-seen, so a, b, c = 0, 1, 2)."""
    for semi in (True, False):
        p = (O.Prog().pred("node", 1).pred("edge", 2).pred("reach", 1).pred("unreach", 1, stratum=1))
        p.rule(("reach", ["Y"]), ("edge", ["X", "Y"]), ("reach", ["X"]))
        p.rule(("unreach", ["X"]), ("node", ["X"]), ("not", "reach", ["X"]))
        for v in (0, 1, 2):
            p.fact("node", [v])
        p.fact("edge", [0, 1]).fact("reach", [0])
        db, _ = p.run(semi_naive=semi)
        assert _pairs(db["unreach"]) == [(2,)]
        assert len(db["reach"]) == 2


def test_negation_against_same_stratum_is_rejected():
    """p(X) :- q(X), not p(X) in one stratum is an error, naive and
    semi-naive (strata-eval/tests/interp.rs:295-324)."""
    for semi in (True, False):
        p = O.Prog().pred("q", 1).pred("p", 1)
        p.rule(("p", ["X"]), ("q", ["X"]), ("not", "p", ["X"]))
        p.fact("q", [0])
        with pytest.raises(O.OracleError) as e:
            p.run(semi_naive=semi)
        assert e.value.kind == "neg_not_stratified"


def test_count_aggregate_outdegree():
    """outdeg(X, count<Y>) :- edge(X,Y) (interp.rs:327-362)."""
    p = O.Prog().pred("edge", 2).pred("outdeg", 2, stratum=1)
    p.rule(("outdeg", ["X", "N"]), ("edge", ["X", "Y"]), agg=("count", "Y", 1))
    for a, b in [(0, 1), (0, 2), (1, 2)]:
        p.fact("edge", [a, b])
    db, _ = p.run()
    assert db["outdeg"] == [((0, ("i", 2)), None), ((1, ("i", 1)), None)]


def test_sum_aggregate():
    """total(X, sum<V>) :- w(X,V) (interp.rs:364-405)."""
    p = O.Prog().pred("w", 2).pred("total", 2, stratum=1)
    p.rule(("total", ["X", "S"]), ("w", ["X", "V"]), agg=("sum", "V", 1))
    p.fact("w", [0, ("i", 3)]).fact("w", [0, ("i", 4)]).fact("w", [1, ("i", 5)])
    db, _ = p.run()
    assert db["total"] == [((0, ("i", 7)), None), ((1, ("i", 5)), None)]


def test_triangles_fixed_and_complete():
    """K4 fed both ways + dup + self-loop = 4; K_n has C(n,3) (wcoj_diff.rs:56-88)."""
    k4 = np.array([(0, 1), (1, 0), (0, 2), (0, 3), (1, 2), (2, 3), (1, 3), (1, 3), (2, 2)])
    assert O.brute_triangles(k4[:, 0], k4[:, 1], 4) == 4
    for n in (3, 10, 30, 64):
        e = np.array([(a, b) for a in range(n) for b in range(a + 1, n)])
        assert O.brute_triangles(e[:, 0], e[:, 1], n) == n * (n - 1) * (n - 2) // 6
        # the count aggregate over the id-oriented DAG counts each triangle once
        assert O.count_pattern(e[:, 0], e[:, 1]) == n * (n - 1) * (n - 2) // 6


def test_count_aggregate_interp_matches_merge_count(lcg):
    rng = lcg(0x7EA12345678)
    for trial in range(60):
        n = 5 + rng.upto(12)
        m = rng.upto(n * 3)
        e = [(rng.upto(n), rng.upto(n)) for _ in range(m)]
        x = [a for a, _ in e]
        y = [b for _, b in e]
        db, _ = O.count_program(x, y).run()
        want = O.count_pattern(x, y)
        got = db["ntri"][0][0][0][1] if db["ntri"] else 0
        assert got == want, trial


def test_hub_graph_closed_form():
    """b·C(h,2) + C(h,3) triangles on the hub/bridge graph (strata-gpu/examples/tri.rs:29-72)."""
    h, b = 6, 50
    e = [(i, j) for i in range(h) for j in range(i + 1, h)]
    e += [(hub, h + k) for k in range(b) for hub in range(h)]
    a = np.array(e)
    want = b * h * (h - 1) // 2 + h * (h - 1) * (h - 2) // 6
    assert O.brute_triangles(a[:, 0], a[:, 1], h + b) == want
    assert O.count_pattern(a[:, 0], a[:, 1]) == want


def test_4cliques_complete():
    """K_n has C(n,4) 4-cliques (wcoj_diff.rs:136-155)."""
    for n in (4, 10, 20):
        e = np.array([(a, b) for a in range(n) for b in range(a + 1, n)])
        assert O.brute_4cliques(e[:, 0], e[:, 1], n) == n * (n - 1) * (n - 2) * (n - 3) // 24


# ---------------------------------------------------------------- engine equivalence
class _Xorshift:
    """The fuzzer's PRNG (strata-eval/tests/fuzz.rs:16-41)."""

    def __init__(self, seed):
        self.s = (seed * 0x9E3779B97F4A7C15 + 0x12345678) & 0xFFFFFFFFFFFFFFFF

    def next(self):
        x = self.s
        x ^= (x << 13) & 0xFFFFFFFFFFFFFFFF
        x ^= x >> 7
        x ^= (x << 17) & 0xFFFFFFFFFFFFFFFF
        self.s = x
        return x

    def below(self, n):
        return self.next() % n

    def range(self, lo, hi):
        return lo + self.below(hi - lo + 1)

    def chance(self, pct):
        return self.next() % 100 < pct


def _fuzz_program(seed):
    """Random safe program + EDB with the generator's shape (fuzz.rs:46-150)."""
    r = _Xorshift(seed)
    trop = r.chance(50)
    domain = r.range(2, 4)
    n_pred = r.range(2, 3)
    nvars = r.range(2, 3)
    p = O.Prog()
    for i in range(n_pred):
        p.pred(f"p{i}", 2, trop=trop)
    for _ in range(r.range(2, 5)):
        body, bvars = [], []
        for _ in range(r.range(1, 3)):
            q = r.below(n_pred)
            a, b = r.below(nvars), r.below(nvars)
            bvars += [a, b]
            body.append((f"p{q}", [f"V{a}", f"V{b}"]))
        h1 = bvars[r.below(len(bvars))]
        h2 = bvars[r.below(len(bvars))]
        p.rule((f"p{r.below(n_pred)}", [f"V{h1}", f"V{h2}"]), *body)
    if not trop and n_pred >= 2 and r.chance(35):
        p.pred(f"p{n_pred}", 2, stratum=1)
        pos, neg = r.below(n_pred), r.below(n_pred)
        p.rule((f"p{n_pred}", ["V0", "V1"]), (f"p{pos}", ["V0", "V1"]), ("not", f"p{neg}", ["V0", "V1"]))
    for _ in range(r.range(2, 8)):
        q = f"p{r.below(n_pred)}"
        a, b = r.below(domain), r.below(domain)
        p.fact(q, [a, b], weight=r.range(0, 4) if trop else None)
    return p


def test_naive_equals_semi_naive_fuzz():
    """naive == semi-naive on random programs (strata-eval/tests/fuzz.rs:161-177)."""
    for seed in range(1500):
        p = _fuzz_program(seed)
        try:
            a = p.run(semi_naive=False)[0]
            ea = None
        except O.OracleError as e:
            a, ea = None, e.kind
        try:
            b = p.run(semi_naive=True)[0]
            eb = None
        except O.OracleError as e:
            b, eb = None, e.kind
        assert (a, ea) == (b, eb), seed


def test_closure_count_fp_matches_tuples(lcg):
    """The batched-reachability summary oracle (SCC + DAG closure, count and
    row-polynomial fingerprint) agrees with the reference's set fixpoint
    (strata-gpu/tests/tc_diff.rs:12-29) and the interpreter-shaped fast TC."""
    rng = lcg(0xC10541)
    for trial in range(120):
        n = 2 + rng.upto(40)
        m = rng.upto(3 * n)
        edges = sorted({(rng.upto(n), rng.upto(n)) for _ in range(m)})
        s = np.array([e[0] for e in edges], np.uint32)
        d = np.array([e[1] for e in edges], np.uint32)
        want = _set_fixpoint(edges) if edges else []
        wx = np.array([t[0] for t in want], np.uint64)
        wz = np.array([t[1] for t in want], np.int64)
        got = O.closure_count_fp(n, s, d)
        assert got == (len(want), O.poly_fingerprint(wx, wz, n)), trial
        if edges:
            fx, fz, _ = O.fast_tc(s, d)
            assert (len(fx), O.poly_fingerprint(fx, fz.astype(np.int64), n)) == got


def test_closure_count_closed_forms():
    """Chain of n nodes: n(n-1)/2 pairs (tc_diff.rs:86-102); a cycle: n^2."""
    for n in (2, 17, 400):
        s = np.arange(n - 1, dtype=np.uint32)
        assert O.closure_count_fp(n, s, s + 1)[0] == n * (n - 1) // 2
        c = np.arange(n, dtype=np.uint32)
        assert O.closure_count_fp(n, c, (c + 1) % n)[0] == n * n


def test_closure_batch_equals_per_instance():
    import sys
    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "strata-k_b200"))
    from strata_b200 import gen
    wl = gen.batch_tc_workload(n_inst=48, n_min=20, n_max=600, seed=11)
    counts, fps = O.closure_batch(wl.nodes, wl.edge_off, wl.src, wl.dst, threads=4)
    for i in range(len(wl)):
        n, s, d = wl.instance(i)
        assert (int(counts[i]), int(fps[i])) == O.closure_count_fp(n, s, d)
        if i < 6:
            fx, fz, _ = O.fast_tc(s, d)
            assert int(counts[i]) == len(fx)
            assert int(fps[i]) == O.poly_fingerprint(fx, fz.astype(np.int64), n)


def _aml_program(fx):
    """The AML workload program (examples/workloads/aml/aml.strata) over its
    TSV inputs: symbols interned first-seen — the query constants at check
    time, then the inputs in declaration order (strata-check/src/lib.rs:863-870,
    strata-k/src/input.rs:109-149); flags are the probabilistic leaves in row
    order."""
    from strata_b200.textio import SymbolDict
    d = SymbolDict()
    for _, c in fx["queries"]:
        d.intern(c)
    p = (O.Prog().pred("entity", 1).pred("owns", 2).pred("sanctioned", 1).pred("flag", 1)
         .pred("control", 2).pred("investigate", 1).pred("cleared", 1, stratum=1))
    p.rule(("control", ["X", "Y"]), ("owns", ["X", "Y"]))
    p.rule(("control", ["X", "Z"]), ("owns", ["X", "Y"]), ("control", ["Y", "Z"]))
    p.rule(("investigate", ["X"]), ("flag", ["X"]))
    p.rule(("investigate", ["X"]), ("control", ["X", "Y"]), ("flag", ["Y"]))
    p.rule(("investigate", ["X"]), ("control", ["Y", "X"]), ("sanctioned", ["Y"]))
    p.rule(("cleared", ["X"]), ("entity", ["X"]), ("not", "investigate", ["X"]))
    for name in ("entity", "owns", "sanctioned"):
        for row in fx[name]:
            p.fact(name, [d.intern(v) for v in row])
    probs, flags = [], []
    for row in fx["flag"]:
        p.fact("flag", [d.intern(row[0])], O.PROB)
        probs.append(float(row[1]))
        flags.append(row)
    return p, d, probs, flags


def test_aml_workload_pinned_lines():
    """Provenance capture (Prov_k(4) with stratified negation over soft
    evidence), exact compilation and the gradient reproduce the reference
    CLI's pinned AML lines (crates/strata-cli/tests/workloads.rs:17-23)."""
    from strata_b200.textio import grad_line, prob_line
    fx = json.loads((GOLDEN / "aml.json").read_text())
    p, d, probs, flags = _aml_program(fx)
    db = O.ProvDb(p, probs, {"investigate": 4, "cleared": 4})
    lines = []
    for pred, c in fx["queries"]:
        proofs = db.proofs(pred, [d.get(c)])
        pr, g, _ = O.compile_grad(proofs, probs)
        lines.append(prob_line(pr, pred, [c], top_k=4).rstrip("\n"))
        if pred == "investigate":
            for (name, fp), gv in zip(flags, g):
                lines.append(grad_line(float(fp), "flag", [name], gv, model="aml_gnn").rstrip("\n"))
    for want in fx["pinned"]:
        assert want in lines, (want, lines)


def test_prov_facade_and_bridge_values():
    """path over {a->c, a->b, b->c}: 0.625 and d/d(direct) = 0.75
    (strata-k/tests/facade.rs:38-52); owns acme->shell->target with a direct
    0.3 stake: 0.804 (facade.rs:56-76); the DIAMOND 0.86 and dP/dp(ac) = 0.28
    (strata-py/tests/test_bridge.py:42-54) — as Prov captures of path."""
    def run(edges):
        p = O.Prog().pred("edge", 2).pred("path", 2)
        p.rule(("path", ["X", "Y"]), ("edge", ["X", "Y"]))
        p.rule(("path", ["X", "Z"]), ("edge", ["X", "Y"]), ("path", ["Y", "Z"]))
        for a, b, _ in edges:
            p.fact("edge", [a, b], O.PROB)
        db = O.ProvDb(p, [w for _, _, w in edges], {"path": 0})
        return O.compile_grad(db.proofs("path", [0, 2]), [w for _, _, w in edges])
    pr, g, _ = run([(0, 2, 0.5), (0, 1, 0.5), (1, 2, 0.5)])
    assert abs(pr - 0.625) < 1e-12 and abs(g[0] - 0.75) < 1e-12
    pr, _, _ = run([(0, 1, 0.9), (1, 2, 0.8), (0, 2, 0.3)])
    assert abs(pr - 0.804) < 1e-12
    pr, g, _ = run([(0, 1, 0.9), (1, 2, 0.8), (0, 2, 0.5)])
    assert pr == pytest.approx(0.86) and g[2] == pytest.approx(0.28)


def test_prov_tc_fast_matches_interpreter_capture():
    """The target-restricted TC-shaped Prov_k capture equals the interpreter's
    full capture (provenance.rs:286-362) on random graphs, for every k."""
    rng = np.random.default_rng(5)
    for trial in range(30):
        n = int(rng.integers(3, 12))
        m = int(rng.integers(1, 3 * n))
        src = rng.integers(0, n, m)
        dst = rng.integers(0, n, m)
        probs = rng.uniform(0.05, 0.95, m)
        k = int(rng.integers(1, 5))
        p = O.Prog().pred("edge", 2).pred("path", 2)
        p.rule(("path", ["X", "Y"]), ("edge", ["X", "Y"]))
        p.rule(("path", ["X", "Z"]), ("edge", ["X", "Y"]), ("path", ["Y", "Z"]))
        for a, b in zip(src, dst):
            p.fact("edge", [int(a), int(b)], O.PROB)
        db = O.ProvDb(p, probs, {"path": k})
        rel = db.relation("path")
        qs = np.repeat(np.arange(n), n)
        qt = np.tile(np.arange(n), n)
        got, _ = O.prov_tc(n, src, dst, probs, k, qs, qt, threads=2)
        for q in range(len(qs)):
            want = rel.get((int(qs[q]), int(qt[q])), [])
            assert got[q] == want, (trial, qs[q], qt[q])


def test_asp_simplify_filter_reference_case():
    """crates/strata-gpu/src/asp.rs tests: r :- p, not s  keeps an empty body;
    r :- q, s  dies (s impossible)."""
    poss, cert = [1, 1, 0, 1], [1, 1, 0, 0]
    h, s, l = O.asp_simplify_filter([3, 3], [0, 2, 4], [1, -3, 2, 3], poss, cert)
    assert h == [3] and s == [0, 0] and l == []
