"""The operator surface (strata_op_join / _project / _select / _intersect /
_semijoin / _reduce / _merge_diff / _aggregate) against numpy restatements
of the interpreter's operators, and whole programs composed from it
(strata_b200.ops.Program) against oracle layer A — the restated
interpreter — on random programs from the fuzz generator
(strata-eval/tests/fuzz.rs:46-177).  Integer results: exact."""
import numpy as np
import pytest

import oracle as O
import strata_b200 as S
from strata_b200 import gen
from strata_b200.ops import INF, SH, DevRel, Operators, Program

pytestmark = pytest.mark.gpu

M32 = np.uint64(0xFFFFFFFF)


@pytest.fixture(scope="module")
def ops(engine):
    o = Operators(engine)
    yield o
    engine.set_stream(None)


def _keys(a, b):
    return (np.asarray(a, np.uint64) << np.uint64(SH)) | np.asarray(b, np.uint64)


def _cols(k):
    return (k >> np.uint64(SH)).astype(np.int64), (k & M32).astype(np.int64)


def _trop_mul(x, y):
    if x == INF or y == INF:
        return INF
    return x + y


def test_join_bool_and_trop_match_nested_loop(ops):
    rng = np.random.default_rng(1)
    for trial in range(12):
        n = int(rng.integers(2, 60))
        ma, mb = int(rng.integers(0, 400)), int(rng.integers(0, 400))
        a = np.unique(_keys(rng.integers(0, n, ma), rng.integers(0, n, ma)))
        b = np.unique(_keys(rng.integers(0, n, mb), rng.integers(0, n, mb)))
        trop = trial % 2 == 1
        aw = rng.integers(0, 1000, len(a)) if trop else None
        bw = rng.integers(0, 1000, len(b)) if trop else None
        if trop and len(a):
            aw[0] = INF  # a +inf row
        ra, rb = ops.upload(a, aw), ops.upload(b, bw)
        k, w, m = ops.join(ra.keys, ra.w, ra.n, rb)
        got = sorted(zip(k[:m].cpu().numpy().view(np.uint64).tolist(),
                         (w[:m].cpu().numpy().tolist() if trop else [None] * m)))
        ax, ay = _cols(a)
        bx, by = _cols(b)
        want = []
        for i in range(len(a)):
            for j in np.flatnonzero(bx == ay[i]):
                key = (int(ax[i]) << SH) | int(by[j])
                want.append((key, _trop_mul(int(aw[i]), int(bw[j])) if trop else None))
        assert got == sorted(want), trial


def test_join_overflow_and_capacity(ops, engine):
    import ctypes as C
    a = ops.upload(_keys([0], [1]), np.array([INF - 10], np.int64))
    b = ops.upload(_keys([1], [2]), np.array([100], np.int64))
    with pytest.raises(S.TropOverflow):
        ops.join(a.keys, a.w, a.n, b)
    # an output capacity below the binding count is refused, and the count returned
    a = ops.upload(_keys([0, 0], [1, 2]))
    b = ops.upload(_keys([1, 1, 2], [5, 6, 7]))
    out = ops._new(2)
    m = C.c_uint64()
    rc = engine.lib.strata_op_join(engine.ctx, 8, C.c_void_p(a.keys.data_ptr()), None, 2, SH,
                                   C.c_void_p(b.keys.data_ptr()), None, 3, SH, SH, C.c_void_p(out.data_ptr()),
                                   None, 2, C.byref(m))
    assert rc == 1 and m.value == 3


def test_project_select_intersect_semijoin(ops):
    rng = np.random.default_rng(2)
    k = np.unique(_keys(rng.integers(0, 20, 300), rng.integers(0, 20, 300)))
    w = rng.integers(0, 50, len(k))
    r = ops.upload(k, w)
    c0, c1 = _cols(k)
    # project: swap; (c0, const 7); unary c1
    for sh, sl, ch, cl, want in ((1, 0, 0, 0, (c1 << SH) | c0), (0, 2, 0, 7, (c0 << SH) | 7),
                                 (1, 2, 0, 0, c1 << SH)):
        got = ops.project(r.keys, r.n, sh, sl, ch, cl)[:r.n].cpu().numpy()
        assert np.array_equal(got, want.astype(np.int64))
    # select: c0 == c1, c0 == 3, c1 == 5 (rows and weights kept in order)
    for mode, val, keep in ((0, 0, c0 == c1), (1, 3, c0 == 3), (2, 5, c1 == 5)):
        kk, ww, m = ops.select(r.keys, r.w, r.n, mode, val)
        assert np.array_equal(kk[:m].cpu().numpy().view(np.uint64), k[keep])
        assert np.array_equal(ww[:m].cpu().numpy(), w[keep])
    # intersect with weights multiplied; semijoin / anti-join
    b = np.unique(_keys(rng.integers(0, 20, 200), rng.integers(0, 20, 200)))
    bw = rng.integers(0, 50, len(b))
    rb = ops.upload(b, bw)
    kk, ww, m = ops.intersect(r.keys, r.w, r.n, rb)
    inb = np.isin(k, b)
    assert np.array_equal(kk[:m].cpu().numpy().view(np.uint64), k[inb])
    pos = np.searchsorted(b, k[inb])
    assert np.array_equal(ww[:m].cpu().numpy(), w[inb] + bw[pos])
    for anti in (False, True):
        kk, ww, m = ops.semijoin(r.keys, r.w, r.n, None, rb, anti)
        sel = ~inb if anti else inb
        assert np.array_equal(kk[:m].cpu().numpy().view(np.uint64), k[sel])
    # probe keys: negation of a unary atom over c1
    u = np.unique(rng.integers(0, 20, 8)).astype(np.uint64) << np.uint64(SH)
    probe = ops.project(r.keys, r.n, 1, 2, 0, 0)
    kk, _, m = ops.semijoin(r.keys, None, r.n, probe, ops.upload(u), True)
    assert np.array_equal(kk[:m].cpu().numpy().view(np.uint64), k[~np.isin(c1 << SH, u.astype(np.int64))])


def test_reduce_long_runs_across_tiles(ops):
    """Runs longer than a reduction tile, runs ending exactly at tile ends,
    tiles without a run head, unsorted weights inside a run and +inf
    weights: one row per key, the minimum weight (Trop) or the distinct keys
    (Bool)."""
    rng = np.random.default_rng(11)
    lens = [1, 3, 1279, 1280, 1281, 2303, 2304, 2305, 40_000, 1, 1, 7, 100_000, 2, 4608, 1]
    keys = np.repeat(np.arange(len(lens), dtype=np.uint64) * np.uint64(7) + np.uint64(5), lens)
    w = rng.integers(-10**12, 10**12, len(keys))
    w[rng.random(len(keys)) < 0.01] = np.iinfo(np.int64).max  # +inf
    r = ops.upload(keys, w)
    red = ops.reduce(r.keys, r.w, r.n)
    kk, ww = ops.download(red)
    starts = np.concatenate([[0], np.cumsum(lens)[:-1]])
    assert np.array_equal(kk, keys[starts])
    assert np.array_equal(ww, np.minimum.reduceat(w, starts))
    b = ops.reduce(ops.upload(keys).keys, None, len(keys))
    assert b.n == len(lens)
    assert np.array_equal(ops.download(b)[0], keys[starts])
    # in place is refused: tiles write while other tiles still read
    import ctypes as C
    m = C.c_uint64()
    rc = ops.lib.strata_op_reduce(ops.eng.ctx, 8, C.c_void_p(r.keys.data_ptr()), None, len(keys),
                                  C.c_void_p(r.keys.data_ptr()), None, C.byref(m))
    assert rc == S._lib.E_INVALID
    nf, nd = C.c_uint64(), C.c_uint64()
    rc = ops.lib.strata_op_merge_diff(ops.eng.ctx, 8, C.c_void_p(r.keys.data_ptr()), C.c_void_p(r.w.data_ptr()), 10,
                                      C.c_void_p(r.keys.data_ptr() + 80), C.c_void_p(r.w.data_ptr() + 80), 10,
                                      C.c_void_p(r.keys.data_ptr() + 80), C.c_void_p(r.w.data_ptr() + 800),
                                      C.c_void_p(r.keys.data_ptr() + 1600), C.c_void_p(r.w.data_ptr() + 1600),
                                      C.byref(nf), C.byref(nd))
    assert rc == S._lib.E_INVALID  # full_out over cand


def test_reduce_merge_diff_and_aggregate(ops):
    rng = np.random.default_rng(3)
    cand = np.sort(_keys(rng.integers(0, 30, 2000), rng.integers(0, 30, 2000)))
    cw = rng.integers(0, 100, len(cand))
    order = np.lexsort((cw, cand))
    cand, cw = cand[order], cw[order]
    rc = ops.upload(cand, cw)
    red = ops.reduce(rc.keys, rc.w, rc.n)
    uk, first = np.unique(cand, return_index=True)
    kk, ww = ops.download(red)
    assert np.array_equal(kk, uk) and np.array_equal(ww, cw[first])  # min per key
    full_k = np.unique(_keys(rng.integers(0, 30, 300), rng.integers(0, 30, 300)))
    full_w = rng.integers(0, 100, len(full_k))
    f2, d = ops.merge_diff(ops.upload(full_k, full_w), red)
    fk, fw = ops.download(f2)
    dk, dw = ops.download(d)
    ref = dict(zip(full_k.tolist(), full_w.tolist()))
    changed = {}
    for key, wv in zip(uk.tolist(), cw[first].tolist()):
        if key not in ref or wv < ref[key]:
            ref[key] = wv
            changed[key] = wv
    assert fk.tolist() == sorted(ref) and fw.tolist() == [ref[x] for x in sorted(ref)]
    assert dk.tolist() == sorted(changed) and dw.tolist() == [changed[x] for x in sorted(changed)]
    # aggregates per group (key >> 32) and over everything
    vals = rng.integers(-1000, 1000, len(cand))
    rv = ops.upload(cand, vals)
    g0 = (cand >> np.uint64(SH)).astype(np.int64)
    for op, fn in ((0, len), (1, np.sum), (2, np.min), (3, np.max)):
        gr, out, m = ops.aggregate(rv.keys, rv.w, rv.n, SH, op)
        groups = np.unique(g0)
        assert np.array_equal(gr[:m].cpu().numpy(), groups)
        want = [fn(vals[g0 == g]) for g in groups]
        assert out[:m].cpu().numpy().tolist() == [int(x) for x in want]
    _, out, m = ops.aggregate(rv.keys, None, rv.n, 64, 0)
    assert m == 1 and int(out[0]) == len(cand)
    # unsorted keys are refused
    bad = ops.upload(cand[::-1].copy())
    with pytest.raises(S.Cuda):
        ops.aggregate(bad.keys, None, bad.n, SH, 0)


def _mirror(p: O.Prog) -> Program:
    """The same program for the device executor."""
    q = Program()
    for name, ar, trop, st in p.preds:
        q.pred(name, ar, trop=trop, stratum=st)
    for head, body, agg in p.rules:
        q.rule(head, *body, agg=agg)
    for f in p.facts:
        if f[0] == "__bulk__":
            _, name, cols, weights, inf = f
            q.facts_bulk(name, cols, weights, inf)
        else:
            q.fact(*f)
    return q


def _fuzz(seed):
    from test_oracle_golden import _fuzz_program
    return _fuzz_program(seed)


def test_fuzz_programs_equal_the_interpreter(engine):
    """Random programs of the fuzz generator's shape: every program the
    executor accepts gives the restated interpreter's relations, errors
    included; programs outside its fragment raise Unsupported."""
    run, skipped = 0, 0
    for seed in range(300):
        p = _fuzz(seed)
        try:
            want, _ = p.run(semi_naive=True)
            werr = None
        except O.OracleError as e:
            want, werr = None, e.kind
        try:
            got, _ = _mirror(p).run(engine)
            gerr = None
        except S.Unsupported:
            skipped += 1
            continue
        except S.NegativeWeightCycle:
            got, gerr = None, "negative_cycle"
        if werr == "unsafe_head":
            skipped += 1
            continue
        assert (got, gerr) == (want, werr), seed
        run += 1
    print(f"fuzz programs run: {run}, outside the executor's fragment: {skipped}")
    assert run >= 150


def test_composed_closure_and_shortest_paths_equal_the_drivers(engine):
    """The TC and MSSP programs composed from operators: same relations and
    rounds as the interpreter restatement and as the fused drivers."""
    s, d = gen.er_directed(300, 1200, 3)
    want, wr = O.tc_program(s, d).run()
    got, gr = _mirror(O.tc_program(s, d)).run(engine)
    assert got == want and gr == wr
    wl = gen.mssp_workload(scale=9, n_sources=8, seed=4)
    p = O.mssp_program(wl.sources, wl.src, wl.dst, wl.w, wl.source_w)
    want, wr = p.run()
    got, gr = _mirror(p).run(engine)
    assert got == want and gr == wr
    fused = engine.mssp_trop(wl.sources, (wl.src, wl.dst, wl.w), source_weights=wl.source_w)
    assert [((a, b), w) for a, b, w in zip(fused.src.tolist(), fused.dst.tolist(), fused.w.tolist())] == got["dist"]
