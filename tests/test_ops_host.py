"""Host logic of the operator-composed interpreter (strata_b200.ops.Program):
the schedule, body planning and head building, run on the CPU against a
numpy stand-in of the device operator surface with the operators' documented
semantics, and compared with oracle layer A (the restated interpreter) on
random programs of the fuzz generator.  The device operators themselves are
checked in tests/test_gpu_ops.py."""
import numpy as np
import pytest

import oracle as O
import strata_b200 as S
from strata_b200.ops import INF, SH, DevRel, Program

M32 = np.uint64(0xFFFFFFFF)


class NumpyOps:
    """strata_op_* semantics on numpy arrays (test stand-in, not the product)."""

    @staticmethod
    def upload(keys, w=None):
        return DevRel(np.asarray(keys, np.uint64).copy(), None if w is None else np.asarray(w, np.int64).copy(),
                      len(keys))

    @staticmethod
    def download(r):
        return r.keys[:r.n], None if r.w is None else r.w[:r.n]

    @staticmethod
    def to_host(t, n):
        return np.asarray(t[:n])

    @staticmethod
    def zeros(n):
        return np.zeros(max(n, 1), np.int64)

    @staticmethod
    def empty_rel(trop):
        return DevRel(np.zeros(1, np.uint64), np.zeros(1, np.int64) if trop else None, 0)

    @staticmethod
    def concat(parts):
        return np.concatenate([t[:n] for t, n in parts])

    @staticmethod
    def sort(keys, w, n):
        o = np.argsort(keys[:n], kind="stable")
        return keys[:n][o], None if w is None else w[:n][o]

    @staticmethod
    def reduce(keys, w, n):
        k, first = np.unique(keys[:n], return_index=True)
        if w is None:
            return DevRel(k, None, len(k))
        mins = np.minimum.reduceat(w[:n], first) if n else np.zeros(0, np.int64)
        return DevRel(k, mins, len(k))

    @staticmethod
    def merge_diff(full, cand):
        trop = cand.w is not None
        ref = {int(k): (int(full.w[i]) if trop else None) for i, k in enumerate(full.keys[:full.n])}
        ch = {}
        for i, k in enumerate(cand.keys[:cand.n]):
            k = int(k)
            v = int(cand.w[i]) if trop else None
            if k not in ref or (trop and v < ref[k]):
                ref[k] = v
                ch[k] = v
        fk = np.array(sorted(ref), np.uint64)
        dk = np.array(sorted(ch), np.uint64)
        return (DevRel(fk, np.array([ref[int(x)] for x in fk], np.int64) if trop else None, len(fk)),
                DevRel(dk, np.array([ch[int(x)] for x in dk], np.int64) if trop else None, len(dk)))

    @staticmethod
    def _split(k):
        return k >> np.uint64(SH), k & M32

    def project(self, keys, n, sh, sl, ch=0, cl=0):
        c0, c1 = self._split(keys[:n])
        pick = lambda s, c: c0 if s == 0 else c1 if s == 1 else np.full(n, c, np.uint64)
        lo = pick(sl, cl)
        return lo if sh == 3 else (pick(sh, ch) << np.uint64(SH)) | lo

    def select(self, keys, w, n, mode, value=0):
        c0, c1 = self._split(keys[:n])
        m = (c0 == c1) if mode == 0 else (c0 == value) if mode == 1 else (c1 == value)
        return keys[:n][m], None if w is None else w[:n][m], int(m.sum())

    @staticmethod
    def _mul(x, y):
        if x == INF or y == INF:
            return INF
        r = x + y
        if r > INF - 2 or r < -2**63:
            raise S.TropOverflow("overflow")
        return r

    def join(self, a, aw, na, b):
        ac0, ac1 = self._split(a[:na])
        bc0, bc1 = self._split(b.keys[:b.n])
        ok, ow = [], []
        for i in range(na):
            for j in np.flatnonzero(bc0 == ac1[i]):
                ok.append((int(ac0[i]) << SH) | int(bc1[j]))
                if aw is not None:
                    ow.append(self._mul(int(aw[i]), int(b.w[j])))
        return (np.array(ok, np.uint64), np.array(ow, np.int64) if aw is not None else None, len(ok))

    def intersect(self, a, aw, na, b):
        bk = b.keys[:b.n]
        pos = np.searchsorted(bk, a[:na])
        hit = (pos < len(bk)) & (bk[np.minimum(pos, max(len(bk) - 1, 0))] == a[:na]) if len(bk) else np.zeros(na, bool)
        w = None
        if aw is not None:
            w = np.array([self._mul(int(aw[i]), int(b.w[pos[i]])) for i in np.flatnonzero(hit)], np.int64)
        return a[:na][hit], w, int(hit.sum())

    def semijoin(self, rows, w, n, probe, b, anti):
        p = rows[:n] if probe is None else probe[:n]
        hit = np.isin(p, b.keys[:b.n])
        keep = ~hit if anti else hit
        return rows[:n][keep], None if w is None else w[:n][keep], int(keep.sum())

    def aggregate(self, keys, vals, n, gshift, op):
        g = (keys[:n] >> np.uint64(gshift)) if gshift < 64 else np.zeros(n, np.uint64)
        groups, first = np.unique(g, return_index=True)
        bounds = list(first) + [n]
        out = []
        for i in range(len(groups)):
            seg = slice(bounds[i], bounds[i + 1])
            out.append(bounds[i + 1] - bounds[i] if op == 0 else
                       int([np.sum, np.min, np.max][op - 1](vals[seg])))
        return groups, np.array(out, np.int64), len(groups)


def _mirror(p):
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


def test_executor_schedule_on_fuzz_programs_matches_the_interpreter():
    from test_oracle_golden import _fuzz_program
    run, skipped = 0, 0
    for seed in range(600):
        p = _fuzz_program(seed)
        try:
            want, _ = p.run(semi_naive=True)
            werr = None
        except O.OracleError as e:
            want, werr = None, e.kind
        try:
            got, _ = _mirror(p).run(ops=NumpyOps())
            gerr = None
        except S.Unsupported:
            skipped += 1
            continue
        except S.NegativeWeightCycle:
            got, gerr = None, "negative_cycle"
        except S.TropOverflow:
            got, gerr = None, "overflow"
        if werr == "unsafe_head":
            skipped += 1
            continue
        assert (got, gerr) == (want, werr), seed
        run += 1
    assert run >= 450, (run, skipped)


def test_executor_rounds_and_aggregates():
    from strata_b200 import gen
    s, d = gen.er_directed(60, 150, 3)
    want, wr = O.tc_program(s, d).run()
    got, gr = _mirror(O.tc_program(s, d)).run(ops=NumpyOps())
    assert got == want and gr == wr
    p = O.Prog().pred("e", 2).pred("deg", 2, stratum=1).pred("tot", 1, stratum=1)
    p.rule(("deg", ["X", "N"]), ("e", ["X", "Y"]), agg=("count", "Y", 1))
    p.rule(("tot", ["N"]), ("e", ["X", "Y"]), ("e", ["Y", "Z"]), agg=("count", "Z", 0))
    p.facts_bulk("e", [s, d])
    want, _ = p.run()
    got, _ = _mirror(p).run(ops=NumpyOps())
    assert got == want


def test_executor_refuses_what_it_cannot_run():
    # a cross product that must keep both variables of one side
    p = Program().pred("a", 2).pred("b", 2).pred("h", 2, stratum=1)
    p.rule(("h", ["X", "Y"]), ("a", ["X", "Y"]), ("b", ["Z", "W"]))
    p.fact("a", [0, 1]).fact("b", [1, 2])
    with pytest.raises(S.Unsupported):
        p.run(ops=NumpyOps())
    # three variables live across a join step (a triangle whose head keeps X, Y)
    q = Program().pred("a", 2).pred("h", 2, stratum=1)
    q.rule(("h", ["X", "Y"]), ("a", ["X", "Y"]), ("a", ["Y", "Z"]), ("a", ["Z", "X"]))
    q.fact("a", [0, 1])
    with pytest.raises(S.Unsupported):
        q.run(ops=NumpyOps())
    # the same triangle with the head on X alone runs (Y drops after the closing atom)
    t = Program().pred("a", 2).pred("h", 1, stratum=1)
    t.rule(("h", ["X"]), ("a", ["X", "Y"]), ("a", ["Y", "Z"]), ("a", ["Z", "X"]))
    for e in ((0, 1), (1, 2), (2, 0), (2, 3)):
        t.fact("a", list(e))
    got, _ = t.run(ops=NumpyOps())
    assert got["h"] == [((0,), None), ((1,), None), ((2,), None)]
