"""Rule evaluation composed from the device operator surface (strata_op_*).

This is the interpreter's schedule (crates/strata-eval/src/seminaive.rs:70-210:
per stratum the aggregate rules once, a bootstrap full step, then delta
rounds until nothing changes, with the Bellman-Ford cap universe + 2 for Trop
strata) with every rule body evaluated on the device:

    body bindings  ->  strata_op_select / _join / _intersect / _semijoin
    head tuples    ->  strata_op_project
    one round      ->  strata_op_sort, strata_op_reduce (⊕ of a batch),
                       strata_op_merge_diff (combine + the changed tuples)
    aggregates     ->  strata_op_sort + strata_op_aggregate

Relations live on the device as sorted unique packed keys (c0 << 32) | c1 in
64-bit lanes (a unary tuple (v) is v << 32), with an int64 weight column for
Trop (INT64_MAX = +inf).  Supported rules: positive atoms of arity 1 or 2
(variables or symbol constants) that a left-deep chain of joins can bind
with at most two live variables per step, negated atoms over variables the
positive atoms bind, heads of arity 1 or 2 over body variables or symbol
constants, count aggregates.  Other shapes raise ``strata_b200.Unsupported``
(the engine's whole-program drivers run the benchmark programs: closure,
shortest paths, the triangle pattern through its worst-case-optimal join).

The program API mirrors the CPU oracle's: ``pred``, ``rule``, ``fact``,
``facts_bulk``; ``run`` returns ``({pred: [(tuple, weight)]}, rounds)`` with
tuples in id order, weights None (Bool), an int or ``float('inf')``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .gpu import Engine, NegativeWeightCycle, Unsupported, _dp

INF = 2**63 - 1
POS_INF = float("inf")
SH = 32  # bits of the low column of a packed key
OPS = {"count": 0, "sum": 1, "min": 2, "max": 3}


class DevRel:
    """Sorted unique packed keys (int64 tensor holding u64 bits) and weights."""

    def __init__(self, keys, w=None, n: int | None = None):
        self.keys, self.w = keys, w
        self.n = len(keys) if n is None else n

    def __len__(self) -> int:
        return self.n


class Operators:
    """The operator surface on one engine, on torch tensors (64-bit keys)."""

    def __init__(self, eng: Engine):
        import torch
        self.eng, self.lib, self.torch = eng, eng.lib, torch
        self.stream = torch.cuda.Stream()
        eng.set_stream(self.stream.cuda_stream)

    def _new(self, n, dt=None):
        t = self.torch
        with t.cuda.stream(self.stream):
            return t.empty(max(int(n), 1), dtype=dt or t.int64, device="cuda")

    def _ok(self, rc):
        self.eng._check(rc)

    def upload(self, keys: np.ndarray, w: np.ndarray | None = None) -> DevRel:
        t = self.torch
        with t.cuda.stream(self.stream):
            k = t.from_numpy(np.ascontiguousarray(keys, np.uint64).view(np.int64)).cuda()
            ww = None if w is None else t.from_numpy(np.ascontiguousarray(w, np.int64)).cuda()
        self.stream.synchronize()
        return DevRel(k, ww, len(keys))

    def download(self, r: DevRel) -> tuple[np.ndarray, np.ndarray | None]:
        k = r.keys[:r.n].cpu().numpy().view(np.uint64)
        w = None if r.w is None else r.w[:r.n].cpu().numpy()
        return k, w

    def to_host(self, t, n) -> np.ndarray:
        return t[:n].cpu().numpy()

    def zeros(self, n):
        t = self._new(n)
        with self.torch.cuda.stream(self.stream):
            t.zero_()
        return t

    def empty_rel(self, trop: bool) -> DevRel:
        return DevRel(self._new(0), self._new(0) if trop else None, 0)

    def concat(self, parts):
        """[(tensor, n)] -> one tensor of the first n entries of each."""
        with self.torch.cuda.stream(self.stream):
            return self.torch.cat([t[:n] for t, n in parts])

    def sort(self, keys, w, n):
        out_k, out_w = self._new(n), (self._new(n) if w is not None else None)
        self._ok(self.lib.strata_op_sort(self.eng.ctx, 8, 8 if w is not None else 0, _dp(keys), _dp(w),
                                         _dp(out_k), _dp(out_w), n, 64))
        return out_k, out_w

    def reduce(self, keys, w, n):
        out_k, out_w = self._new(n), (self._new(n) if w is not None else None)
        m = C.c_uint64()
        self._ok(self.lib.strata_op_reduce(self.eng.ctx, 8, _dp(keys), _dp(w), n, _dp(out_k), _dp(out_w),
                                           C.byref(m)))
        return DevRel(out_k, out_w, m.value)

    def merge_diff(self, full: DevRel, cand: DevRel) -> tuple[DevRel, DevRel]:
        trop = cand.w is not None
        fk, dk = self._new(full.n + cand.n), self._new(cand.n)
        fw = self._new(full.n + cand.n) if trop else None
        dw = self._new(cand.n) if trop else None
        nf, nd = C.c_uint64(), C.c_uint64()
        self._ok(self.lib.strata_op_merge_diff(self.eng.ctx, 8, _dp(full.keys), _dp(full.w), full.n, _dp(cand.keys),
                                               _dp(cand.w), cand.n, _dp(fk), _dp(fw), _dp(dk), _dp(dw),
                                               C.byref(nf), C.byref(nd)))
        return DevRel(fk, fw, nf.value), DevRel(dk, dw, nd.value)

    def project(self, keys, n, sel_hi, sel_lo, const_hi=0, const_lo=0):
        out = self._new(n)
        self._ok(self.lib.strata_op_project(self.eng.ctx, 8, _dp(keys), n, SH, sel_hi, sel_lo, const_hi, const_lo, 8,
                                            SH, _dp(out)))
        return out

    def select(self, keys, w, n, mode, value=0):
        out_k, out_w = self._new(n), (self._new(n) if w is not None else None)
        m = C.c_uint64()
        self._ok(self.lib.strata_op_select(self.eng.ctx, 8, _dp(keys), _dp(w), n, SH, mode, value, _dp(out_k),
                                           _dp(out_w), C.byref(m)))
        return out_k, out_w, m.value

    def join(self, a, aw, na, b: DevRel):
        m = C.c_uint64()
        self._ok(self.lib.strata_op_join(self.eng.ctx, 8, _dp(a), _dp(aw), na, SH, _dp(b.keys), _dp(b.w), b.n, SH, SH,
                                          None, None, 0, C.byref(m)))
        out_k = self._new(m.value)
        out_w = self._new(m.value) if aw is not None else None
        self._ok(self.lib.strata_op_join(self.eng.ctx, 8, _dp(a), _dp(aw), na, SH, _dp(b.keys), _dp(b.w), b.n, SH, SH,
                                          _dp(out_k), _dp(out_w), m.value, C.byref(m)))
        return out_k, out_w, m.value

    def intersect(self, a, aw, na, b: DevRel):
        out_k, out_w = self._new(na), (self._new(na) if aw is not None else None)
        m = C.c_uint64()
        self._ok(self.lib.strata_op_intersect(self.eng.ctx, 8, _dp(a), _dp(aw), na, _dp(b.keys), _dp(b.w), b.n,
                                              _dp(out_k), _dp(out_w), C.byref(m)))
        return out_k, out_w, m.value

    def semijoin(self, rows, w, n, probe, b: DevRel, anti: bool):
        out_k, out_w = self._new(n), (self._new(n) if w is not None else None)
        m = C.c_uint64()
        self._ok(self.lib.strata_op_semijoin(self.eng.ctx, 8, _dp(rows), _dp(w), n, _dp(probe), _dp(b.keys), b.n,
                                             1 if anti else 0, _dp(out_k), _dp(out_w), C.byref(m)))
        return out_k, out_w, m.value

    def aggregate(self, keys, vals, n, group_shift, op):
        groups, out = self._new(n), self._new(n)
        m = C.c_uint64()
        self._ok(self.lib.strata_op_aggregate(self.eng.ctx, 8, _dp(keys), _dp(vals), n, group_shift, op,
                                              _dp(groups), _dp(out), C.byref(m)))
        return groups, out, m.value


def _is_var(a) -> bool:
    return isinstance(a, str)


def _const(a) -> int:
    if isinstance(a, tuple) and a[0] == "s":
        return int(a[1])
    if isinstance(a, (int, np.integer)):
        return int(a)
    raise Unsupported(f"only variables and symbol constants are supported, not {a!r}")


class Program:
    """A Core-IR program over unary / binary relations, evaluated on the device."""

    def __init__(self):
        self.preds: dict[str, tuple[int, bool, int]] = {}
        self.order: list[str] = []
        self.rules: list = []
        self.facts: list = []

    def pred(self, name, arity, trop=False, stratum=0):
        if arity not in (1, 2):
            raise Unsupported("relations of arity 1 or 2 only")
        self.preds[name] = (arity, trop, stratum)
        self.order.append(name)
        return self

    def rule(self, head, *body, agg=None):
        self.rules.append((head, body, agg))
        return self

    def fact(self, name, values, weight=None):
        self.facts.append((name, [np.array([_const(v)], np.uint64) for v in values],
                           None if weight is None else np.array([INF if weight == POS_INF else int(weight)], np.int64),
                           None if weight is None else np.array([weight == POS_INF], bool)))
        return self

    def facts_bulk(self, name, cols, weights=None, inf=None):
        w = None
        infm = None
        if weights is not None:
            w = np.asarray(weights, np.int64).copy()
            infm = np.zeros(len(w), bool) if inf is None else np.asarray(inf).astype(bool)
            w[infm] = INF
        self.facts.append((name, [np.asarray(c, np.uint64) for c in cols], w, infm))
        return self

    # ---- host side of the schedule ------------------------------------------------
    @staticmethod
    def _pack(cols) -> np.ndarray:
        k = cols[0].astype(np.uint64) << np.uint64(SH)
        if len(cols) == 2:
            k |= cols[1].astype(np.uint64)
        return k

    def _edb(self, ops: Operators):
        """Every relation from its facts, ⊕-combined on the device."""
        per: dict[str, list] = {p: [] for p in self.order}
        for name, cols, w, infm in self.facts:
            if name not in self.preds:
                raise Unsupported(f"unknown predicate {name}")
            per[name].append((self._pack(cols), w, infm))
        db, universe = {}, set()
        for p in self.order:
            ar, trop, _ = self.preds[p]
            parts = per[p]
            keys = np.concatenate([k for k, _, _ in parts]) if parts else np.zeros(0, np.uint64)
            if trop:
                ws = [np.zeros(len(k), np.int64) if w is None else w for k, w, _ in parts]
                w = np.concatenate(ws) if ws else np.zeros(0, np.int64)
            else:
                w = None
            for k, _, _ in parts:
                universe.update((k >> np.uint64(SH)).tolist())
                if ar == 2:
                    universe.update((k & np.uint64(0xFFFFFFFF)).tolist())
            if len(keys):
                r = ops.upload(keys, w)
                sk, sw = ops.sort(r.keys, r.w, r.n)
                db[p] = ops.reduce(sk, sw, r.n)
            else:
                db[p] = ops.empty_rel(trop)
        return db, len(universe)

    def _atom_rows(self, ops, rel: DevRel, args, trop_head: bool):
        """The bindings of one positive atom (unify, naive.rs:407-455): packed
        keys of the atom's rows, constants and repeated variables filtered by
        select, with cols = {variable: column (0 = high, 1 = low)}."""
        keys, w, n = rel.keys, rel.w, rel.n
        if trop_head and w is None:
            w = ops.zeros(n)  # a Bool atom in a Trop rule contributes the ⊗ identity Finite(0)
        if not trop_head:
            w = None
        if len(args) == 1:
            a = args[0]
            if not _is_var(a):
                keys, w, n = ops.select(keys, w, n, 1, _const(a))
                return keys, w, n, {}
            return keys, w, n, {a: 0}
        a, b = args
        if not _is_var(a):
            keys, w, n = ops.select(keys, w, n, 1, _const(a))
        if not _is_var(b):
            keys, w, n = ops.select(keys, w, n, 2, _const(b))
        if _is_var(a) and _is_var(b) and a == b:
            keys, w, n = ops.select(keys, w, n, 0)
            return keys, w, n, {a: 0}
        cols = {}
        if _is_var(a):
            cols[a] = 0
        if _is_var(b):
            cols[b] = 1
        return keys, w, n, cols

    @staticmethod
    def _pair(ops, keys, n, cols, hi, lo):
        """Re-pack rows so the columns are (hi, lo) (two body variables)."""
        return ops.project(keys, n, cols[hi], cols[lo])

    def _body(self, ops, db, delta, rule, pos, trop_head):
        """Bindings of a rule body with the positive atom at `pos` over Δ (None:
        every atom over its full relation) — `solve` (seminaive.rs:215-298) as a
        left-deep chain of device operators over rows of at most two live
        variables: (keys, weights, n, cols) with cols = {variable: column}.

        Each step joins the rows so far with the next positive atom: on one
        shared variable a join (the output keeps the two variables still needed
        — later atoms, negated atoms, the head; a dropped variable keeps its
        multiplicity, one row per binding), on two an intersect, on none a
        cross product of the needed columns (not for aggregates, whose counts
        need every binding).  Negated atoms filter the final rows (anti-join)."""
        head, body, agg = rule
        posl = [(i, b) for i, b in enumerate(body) if b[0] != "not"]
        negl = [b for b in body if b[0] == "not"]
        if not posl:
            raise Unsupported("a rule body without a positive atom")
        head_vars = [a for i, a in enumerate(head[1]) if _is_var(a) and (agg is None or i != agg[2])]
        neg_vars = [v for b in negl for v in b[2] if _is_var(v)]

        def rel_of(i, name):
            if name not in self.preds:
                raise Unsupported(f"unknown predicate {name}")
            return delta[name] if i == pos else db[name]

        # join order: the planner's cost-based variable order (plan.body_order,
        # over the atoms' current sizes) when a chain of two live variables
        # can follow it, else the written order; bindings do not depend on it
        from .plan import body_order
        sizes = [rel_of(i, b[0]).n for i, b in posl]
        universe = getattr(self, "_universe", 1)
        planned = [posl[j] for j in body_order([[v for v in b[1] if _is_var(v)] for _, b in posl], sizes, universe)]
        if planned != posl and self._chain_ok(planned, head_vars, neg_vars, agg is not None):
            posl = planned

        def needed(after):
            vs = set(head_vars) | set(neg_vars)
            for _, (_, args) in posl[after:]:
                vs |= {v for v in args if _is_var(v)}
            return vs

        i0, (n0, a0) = posl[0]
        k, w, n, cols = self._atom_rows(ops, rel_of(i0, n0), a0, trop_head)
        for step, (i1, (n1, a1)) in enumerate(posl[1:], start=1):
            k1, w1, m1, cols1 = self._atom_rows(ops, rel_of(i1, n1), a1, trop_head)
            need = needed(step + 1)
            shared = [v for v in cols if v in cols1]
            if len(shared) == 1:
                y = shared[0]
                x = next((v for v in cols if v != y), y)
                z = next((v for v in cols1 if v != y), y)
                keep = [v for v in dict.fromkeys((x, y, z)) if v in need]
                if len(keep) > 2:
                    raise Unsupported("a join step whose three variables are all still needed")
                p = x if x in keep else y
                q = z if z in keep else y
                a = ops.project(k, n, cols[p], cols[y]) if p in cols else ops.project(k, n, cols[y], cols[y])
                bk = ops.project(k1, m1, cols1[y], cols1[q])
                bs, bw = ops.sort(bk, w1, m1)
                k, w, n = ops.join(a, w, n, DevRel(bs, bw, m1))
                cols = {p: 0} if p == q else {p: 0, q: 1}
            elif len(shared) == 2:
                if len(cols1) != 2 or len(cols) != 2:
                    raise Unsupported("an intersect over a partly bound atom")
                x, y = shared
                a = ops.project(k, n, cols[x], cols[y])
                bk = ops.project(k1, m1, cols1[x], cols1[y])
                bs, bw = ops.sort(bk, w1, m1)
                k, w, n = ops.intersect(a, w, n, DevRel(bs, bw, m1))
                cols = {x: 0, y: 1}
            else:
                if agg is not None:
                    raise Unsupported("a cross product in an aggregate body")
                kl = [v for v in cols if v in need]
                kr = [v for v in cols1 if v in need]
                if len(kl) > 1 or len(kr) > 1:
                    raise Unsupported("a cross product keeping two variables of one side")
                # each side reduced to its needed variable (⊕ over the rest),
                # then paired through a constant join column
                left = ops.project(k, n, cols[kl[0]] if kl else 2, 2, 0, 0)
                ls, lw = ops.sort(left, w, n)
                lr = ops.reduce(ls, lw, n)
                right = ops.project(k1, m1, 2, cols1[kr[0]] if kr else 2, 0, 0)
                rs, rw = ops.sort(right, w1, m1)
                rr = ops.reduce(rs, rw, m1)
                k, w, n = ops.join(ops.project(lr.keys, lr.n, 0, 2, 0, 0), lr.w, lr.n, rr)
                cols = {}
                if kl:
                    cols[kl[0]] = 0
                if kr:
                    cols[kr[0]] = 1
        for _, name, args in negl:
            if name not in self.preds:
                raise Unsupported(f"unknown predicate {name}")
            if not all(_is_var(v) and v in cols for v in args):
                raise Unsupported("negated atoms over variables the positive atoms bind")
            if len(args) == 2:
                probe = ops.project(k, n, cols[args[0]], cols[args[1]])
            else:
                probe = ops.project(k, n, cols[args[0]], 2, 0, 0)
            k, w, n = ops.semijoin(k, w, n, probe, db[name], True)
        return k, w, n, cols

    @staticmethod
    def _chain_ok(posl, head_vars, neg_vars, is_agg) -> bool:
        """Whether the left-deep chain over `posl` keeps at most two live
        variables per step (host-side dry run of _body's cases)."""
        def atom_vars(args):
            return list(dict.fromkeys(v for v in args if _is_var(v)))

        state = atom_vars(posl[0][1][1])
        for step in range(1, len(posl)):
            nxt = atom_vars(posl[step][1][1])
            need = set(head_vars) | set(neg_vars)
            for _, (_, args) in posl[step + 1:]:
                need |= {v for v in args if _is_var(v)}
            shared = [v for v in state if v in nxt]
            if len(shared) == 1:
                y = shared[0]
                x = next((v for v in state if v != y), y)
                z = next((v for v in nxt if v != y), y)
                keep = [v for v in dict.fromkeys((x, y, z)) if v in need]
                if len(keep) > 2:
                    return False
                p = x if x in keep else y
                q = z if z in keep else y
                state = [p] if p == q else [p, q]
            elif len(shared) == 2:
                if len(state) != 2 or len(nxt) != 2:
                    return False
                state = shared
            else:
                kl = [v for v in state if v in need]
                kr = [v for v in nxt if v in need]
                if is_agg or len(kl) > 1 or len(kr) > 1:
                    return False
                state = kl + kr
        return all(v in state for v in neg_vars) and all(v in state for v in head_vars)

    def _head(self, ops, k, n, cols, hargs):
        """Head tuples (build_head, naive.rs:526) from body rows."""

        def sel(a):
            if _is_var(a):
                if a not in cols:
                    raise Unsupported(f"head variable {a} is not bound by the body")
                return cols[a], 0
            return 2, _const(a)

        if len(hargs) == 1:
            s0, c0 = sel(hargs[0])
            return ops.project(k, n, s0, 2, c0, 0)
        (s0, c0), (s1, c1) = sel(hargs[0]), sel(hargs[1])
        return ops.project(k, n, s0, s1, c0, c1)

    def run(self, eng: Engine | None = None, ops=None):
        """Evaluate on `eng` (or on a given operator object with the same
        methods as Operators)."""
        ops = ops if ops is not None else Operators(eng)
        db, universe = self._edb(ops)
        self._universe = universe
        strata = sorted({st for _, _, st in self.preds.values()})
        total_rounds = 0
        agg_out: dict[str, list] = {}
        for st in strata:
            rules = [r for r in self.rules if self.preds[r[0][0]][2] == st]
            for r in rules:
                if r[2] is not None:
                    agg_out.setdefault(r[0][0], []).extend(self._aggregate(ops, db, r))
            plain = [r for r in rules if r[2] is None]
            idb = {r[0][0] for r in plain}
            is_trop = any(self.preds[p][1] for p in idb)
            delta = self._round(ops, db, plain, None, idb)
            rounds = 0
            while any(d.n for d in delta.values()):
                delta = self._round(ops, db, plain, delta, idb)
                rounds += 1
                if is_trop and rounds > universe + 2:
                    raise NegativeWeightCycle("negative-weight cycle: tropical stratum diverges")
            total_rounds = max(total_rounds, rounds)
        out = {}
        for p in self.order:
            if p in agg_out:
                out[p] = sorted(agg_out[p])
                continue
            ar, trop, _ = self.preds[p]
            k, w = ops.download(db[p])
            hi = (k >> np.uint64(SH)).astype(np.int64)
            lo = (k & np.uint64(0xFFFFFFFF)).astype(np.int64)
            rows = []
            for i in range(len(k)):
                t = (int(hi[i]),) if ar == 1 else (int(hi[i]), int(lo[i]))
                rows.append((t, None if not trop else (POS_INF if w[i] == INF else int(w[i]))))
            out[p] = rows
        return out, total_rounds

    def _round(self, ops, db, rules, delta, idb):
        """apply_round (seminaive.rs:114-210): derive with the db as it was at
        the round's start, then combine per head relation."""
        cands: dict[str, list] = {}
        for rule in rules:
            head, body, _ = rule
            hp = head[0]
            trop = self.preds[hp][1]
            positions = [None] if delta is None else [
                i for i, b in enumerate(body) if b[0] != "not" and b[0] in idb and delta.get(b[0]) is not None
                and delta[b[0]].n]
            for pos in positions:
                k, w, n, vs = self._body(ops, db, delta, rule, pos, trop)
                if n:
                    cands.setdefault(hp, []).append((self._head(ops, k, n, vs, head[1]), w, n))
        nxt = {}
        for hp, parts in cands.items():
            n = sum(p[2] for p in parts)
            keys = ops.concat([(p[0], p[2]) for p in parts])
            w = ops.concat([(p[1], p[2]) for p in parts]) if parts[0][1] is not None else None
            sk, sw = ops.sort(keys, w, n)
            red = ops.reduce(sk, sw, n)
            db[hp], nxt[hp] = ops.merge_diff(db[hp], red)
        return nxt

    def _aggregate(self, ops, db, rule):
        """eval_aggregate_rule (naive.rs:300-391) for count: the number of body
        bindings per value of the head's other argument (or one group)."""
        head, body, agg = rule
        op, var, apos = agg
        if op != "count":
            raise Unsupported("sum / min / max need integer aggregands; the device relations hold symbols")
        k, w, n, cols = self._body(ops, db, None, rule, None, False)
        groups = [a for i, a in enumerate(head[1]) if i != apos]
        if len(groups) > 1:
            raise Unsupported("one group column at most")
        if n == 0:
            return []
        if groups:
            g = groups[0]
            if not _is_var(g) or g not in cols:
                raise Unsupported("the group must be a body variable")
            gk = ops.project(k, n, cols[g], 2, 0, 0)
            sk, _ = ops.sort(gk, None, n)
            gr, cnt, m = ops.aggregate(sk, None, n, SH, 0)
            gh = ops.to_host(gr, m).astype(np.int64)
            cn = ops.to_host(cnt, m)
        else:
            gr, cnt, m = ops.aggregate(k, None, n, 64, 0)
            gh, cn = np.zeros(1, np.int64), ops.to_host(cnt, 1)
        rows = []
        for i in range(m):
            rows.append((tuple(("i", int(cn[i])) if j == apos else int(gh[i]) for j in range(len(head[1]))), None))
        return rows
