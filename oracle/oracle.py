"""ctypes front end of the CPU oracle (liboracle.so, built from sk_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline leg as the checker.  The engine never imports it.

Programs are handed to the interpreter as a flat int64 blob:

    npreds, {arity, trop, stratum}*, num_strata,
    nrules, {var_count, head_atom, agg_op, agg_slot, agg_pos, nbody, {neg, atom}*}*,
    nfacts, {pred, arity, {tag, val}*, wkind, wval}*

with ``atom = pred, arity, {kind, val}*`` (kind 0 var slot, 1 symbol id,
2 integer), ``tag`` 0 symbol / 1 integer and ``wkind`` 0 none (Bool),
1 finite, 2 +inf.  ``Prog`` below builds the blob from readable rules.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

OK, E_OVERFLOW, E_NEG_CYCLE = 0, 4, 5
E_ROUND_LIMIT = 18
ERR_NAMES = {0: "ok", 4: "overflow", 5: "negative_cycle", 10: "unknown_pred", 11: "unsafe_head",
             12: "unsafe_neg", 13: "neg_not_stratified", 14: "agg_in_recursion",
             15: "malformed", 16: "non_int_agg", 17: "ann_mismatch", 18: "round_limit"}
POS_INF = float("inf")

_lib = None


def build() -> Path:
    """Compile liboracle.so if stale (make in this directory)."""
    src = HERE / "sk_oracle.cpp"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        u32p, i64p, u8p, u64p = (C.POINTER(C.c_uint32), C.POINTER(C.c_int64),
                                 C.POINTER(C.c_uint8), C.POINTER(C.c_uint64))
        L.sko_interp.restype = C.c_int
        L.sko_interp.argtypes = [i64p, C.c_size_t, C.c_int, C.c_int, C.c_long,
                                 C.POINTER(i64p), C.POINTER(C.c_size_t), C.POINTER(C.c_long)]
        L.sko_free.argtypes = [C.c_void_p]
        L.sko_session_new.restype = C.c_void_p
        L.sko_session_new.argtypes = [i64p, C.c_size_t]
        L.sko_session_run.restype = C.c_int
        L.sko_session_run.argtypes = [C.c_void_p, C.c_int, C.c_long, i64p, C.POINTER(C.c_long),
                                      C.POINTER(C.c_double)]
        L.sko_session_free.argtypes = [C.c_void_p]
        L.sko_fast_tc.restype = C.c_int
        L.sko_fast_tc.argtypes = [u32p, u32p, C.c_size_t, C.POINTER(u32p), C.POINTER(u32p),
                                  C.POINTER(C.c_size_t), C.POINTER(C.c_long)]
        L.sko_fast_trop.restype = C.c_int
        L.sko_fast_trop.argtypes = [C.c_int, u32p, i64p, u8p, C.c_size_t, u32p, u32p, i64p, u8p,
                                    C.c_size_t, C.POINTER(u32p), C.POINTER(u32p), C.POINTER(i64p),
                                    C.POINTER(u8p), C.POINTER(C.c_size_t), C.POINTER(C.c_long)]
        L.sko_fingerprint.restype = C.c_uint64
        L.sko_fingerprint.argtypes = [u32p, u32p, i64p, u8p, C.c_size_t]
        L.sko_bfs_closure.restype = None
        L.sko_bfs_closure.argtypes = [u32p, u32p, C.c_size_t, C.c_int, u64p, u64p]
        L.sko_dijkstra_mssp.restype = C.c_int
        L.sko_dijkstra_mssp.argtypes = [u32p, i64p, C.c_size_t, u32p, u32p, i64p, C.c_size_t,
                                        C.c_int, u64p, u64p]
        L.sko_dijkstra_mssp_rows.restype = C.c_int
        L.sko_dijkstra_mssp_rows.argtypes = [u32p, i64p, C.c_size_t, u32p, u32p, i64p, C.c_size_t, C.c_int,
                                             C.POINTER(u32p), C.POINTER(u32p), C.POINTER(i64p),
                                             C.POINTER(C.c_size_t)]
        L.sko_count_pattern.restype = C.c_uint64
        L.sko_count_pattern.argtypes = [u32p, u32p, C.c_size_t, C.c_int]
        L.sko_brute_triangles.restype = C.c_uint64
        L.sko_brute_triangles.argtypes = [u32p, u32p, C.c_size_t, C.c_uint32]
        L.sko_brute_4cliques.restype = C.c_uint64
        L.sko_brute_4cliques.argtypes = [u32p, u32p, C.c_size_t, C.c_uint32]
        L.sko_prov_run.restype = C.c_void_p
        L.sko_prov_run.argtypes = [i64p, C.c_size_t, C.POINTER(C.c_double), C.c_size_t, i64p, C.c_size_t,
                                   C.POINTER(C.c_long), C.POINTER(C.c_int)]
        L.sko_prov_free.argtypes = [C.c_void_p]
        L.sko_prov_proofs.restype = C.c_long
        L.sko_prov_proofs.argtypes = [C.c_void_p, C.c_int, i64p, C.c_int, i64p, C.c_size_t]
        L.sko_prov_relation.restype = C.c_long
        L.sko_prov_relation.argtypes = [C.c_void_p, C.c_int, i64p, C.c_size_t]
        L.sko_compile_grad.restype = C.c_int
        L.sko_compile_grad.argtypes = [i64p, C.c_size_t, C.POINTER(C.c_double), C.c_size_t,
                                       C.POINTER(C.c_double), C.POINTER(C.c_double), i64p]
        L.sko_prov_tc.restype = C.c_long
        L.sko_prov_tc.argtypes = [C.c_uint32, u32p, u32p, C.c_size_t, C.POINTER(C.c_double), C.c_size_t,
                                  u32p, C.c_size_t, u32p, u32p, C.c_size_t, C.c_int, i64p, C.c_size_t,
                                  i64p, C.POINTER(C.c_long), C.POINTER(C.c_size_t)]
        L.sko_closure_count_fp.restype = C.c_int
        L.sko_closure_count_fp.argtypes = [C.c_uint32, u32p, u32p, C.c_uint64, u64p, u64p]
        L.sko_closure_batch.restype = C.c_int
        L.sko_closure_batch.argtypes = [C.c_uint32, u32p, u64p, u32p, u32p, C.c_int, u64p, u64p]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def _col(a, dt):
    return np.ascontiguousarray(np.asarray(a), dtype=dt)


PROB = object()  # weight marker of a probabilistic (leaf) fact: proof {+(i+1)}


class OracleError(Exception):
    def __init__(self, code: int):
        super().__init__(ERR_NAMES.get(code, str(code)))
        self.code = code
        self.kind = ERR_NAMES.get(code, str(code))


# ---------------------------------------------------------------------------
# A. the interpreter
# ---------------------------------------------------------------------------
@dataclass
class Prog:
    """A Core-IR program for the oracle interpreter.

    ``pred(name, arity, trop=False, stratum=0)`` declares; ``rule(head,
    *body)`` adds ``head :- body`` where atoms are ``(name, args)`` and args
    are variable names (str starting uppercase), symbol ids (``('s', id)``) or
    integers (``('i', v)``); a body atom prefixed ``'not'`` is negated:
    ``('not', name, args)``.  ``agg`` = ``(op, var, position)`` for an
    aggregate head.  ``fact(name, values, weight=None)`` seeds the EDB
    (values are symbol ids, or ``('i', v)`` for integers; weight an int,
    ``POS_INF`` or None for Bool).
    """

    preds: list = field(default_factory=list)
    rules: list = field(default_factory=list)
    facts: list = field(default_factory=list)

    def pred(self, name, arity, trop=False, stratum=0):
        self.preds.append((name, arity, trop, stratum))
        return self

    def _pi(self, name):
        for i, p in enumerate(self.preds):
            if p[0] == name:
                return i
        raise KeyError(name)

    def rule(self, head, *body, agg=None):
        self.rules.append((head, body, agg))
        return self

    def fact(self, name, values, weight=None):
        self.facts.append((name, values, weight))
        return self

    def facts_bulk(self, name, cols, weights=None, inf=None):
        """Append many binary/unary facts from numpy columns (symbol ids)."""
        self.facts.append(("__bulk__", name, cols, weights, inf))
        return self

    def blob(self) -> np.ndarray:
        out: list[int] = []
        out.append(len(self.preds))
        for _, ar, trop, st in self.preds:
            out += [ar, 1 if trop else 0, st]
        out.append(max((p[3] for p in self.preds), default=0) + 1)
        out.append(len(self.rules))
        for head, body, agg in self.rules:
            slots: dict[str, int] = {}

            def term(a):
                if isinstance(a, str):
                    return [0, slots.setdefault(a, len(slots))]
                if isinstance(a, tuple) and a[0] == "s":
                    return [1, int(a[1])]
                if isinstance(a, tuple) and a[0] == "i":
                    return [2, int(a[1])]
                if isinstance(a, (int, np.integer)):
                    return [1, int(a)]
                raise ValueError(a)

            # slots are numbered in body order first (the checker's order is
            # irrelevant to results), then head
            enc_body = []
            for lit in body:
                neg = lit[0] == "not"
                name, args = (lit[1], lit[2]) if neg else (lit[0], lit[1])
                enc = [1 if neg else 0, self._pi(name), len(args)]
                for a in args:
                    enc += term(a)
                enc_body.append(enc)
            hname, hargs = head
            enc_head = [self._pi(hname), len(hargs)]
            agg_op, agg_slot, agg_pos = -1, 0, 0
            for k, a in enumerate(hargs):
                if agg is not None and k == agg[2]:
                    enc_head += [0, slots.setdefault(agg[1], len(slots))]
                else:
                    enc_head += term(a)
            if agg is not None:
                agg_op = {"count": 0, "sum": 1, "min": 2, "max": 3}[agg[0]]
                agg_slot = slots[agg[1]]
                agg_pos = agg[2]
            out += [len(slots)] + enc_head + [agg_op, agg_slot, agg_pos, len(enc_body)]
            for e in enc_body:
                out += e
        nf_pos = len(out)
        out.append(0)
        nf = 0
        chunks = [np.asarray(out, dtype=np.int64)]
        for f in self.facts:
            if f[0] == "__bulk__":
                _, name, cols, weights, inf = f
                pi = self._pi(name)
                n = len(cols[0])
                ar = len(cols)
                width = 2 + 2 * ar + 2
                blk = np.zeros((n, width), dtype=np.int64)
                blk[:, 0] = pi
                blk[:, 1] = ar
                for c in range(ar):
                    blk[:, 2 + 2 * c] = 0
                    blk[:, 3 + 2 * c] = np.asarray(cols[c], dtype=np.int64)
                if weights is PROB:
                    blk[:, -2] = 3
                elif weights is None:
                    blk[:, -2] = 0
                else:
                    infm = np.zeros(n, bool) if inf is None else np.asarray(inf).astype(bool)
                    blk[:, -2] = np.where(infm, 2, 1)
                    blk[:, -1] = np.where(infm, 0, np.asarray(weights, dtype=np.int64))
                chunks.append(blk.ravel())
                nf += n
            else:
                name, values, weight = f
                rec = [self._pi(name), len(values)]
                for v in values:
                    if isinstance(v, tuple) and v[0] == "i":
                        rec += [1, int(v[1])]
                    else:
                        rec += [0, int(v)]
                if weight is None:
                    rec += [0, 0]
                elif weight is PROB:
                    rec += [3, 0]
                elif weight == POS_INF:
                    rec += [2, 0]
                else:
                    rec += [1, int(weight)]
                chunks.append(np.asarray(rec, dtype=np.int64))
                nf += 1
        chunks[0][nf_pos] = nf
        return np.concatenate(chunks)

    def run(self, semi_naive=True, threads=1, max_rounds=-1):
        """Returns ({pred name: [(tuple, weight-or-None)]}, rounds).  Raises OracleError."""
        L = lib()
        b = self.blob()
        out = C.POINTER(C.c_int64)()
        n = C.c_size_t()
        rounds = C.c_long(0)
        rc = L.sko_interp(_p(b, C.c_int64), len(b), 1 if semi_naive else 0, threads, max_rounds,
                          C.byref(out), C.byref(n), C.byref(rounds))
        if rc not in (OK, E_ROUND_LIMIT):
            raise OracleError(rc)
        arr = np.ctypeslib.as_array(out, shape=(n.value,)).copy() if n.value else np.zeros(0, np.int64)
        L.sko_free(C.cast(out, C.c_void_p))
        db = {}
        pos = 0
        for name, ar, trop, _ in self.preds:
            cnt = int(arr[pos])
            pos += 1
            rows = []
            width = 2 * ar + 2
            if cnt:
                blk = arr[pos:pos + cnt * width].reshape(cnt, width)
                for r in blk:
                    vals = tuple(int(r[2 * k + 1]) if r[2 * k] == 0 else ("i", int(r[2 * k + 1]))
                                 for k in range(ar))
                    wk = r[-2]
                    w = None if wk == 0 else (POS_INF if wk == 2 else int(r[-1]))
                    rows.append((vals, w))
            pos += cnt * width
            db[name] = rows
        return db, int(rounds.value)


class Session:
    """A program loaded once into the interpreter; ``run`` re-evaluates it
    from the EDB and returns ({pred: count}, rounds, seconds)."""

    def __init__(self, prog: "Prog"):
        self.prog = prog
        b = prog.blob()
        self.h = lib().sko_session_new(_p(b, C.c_int64), len(b))
        if not self.h:
            raise OracleError(15)

    def run(self, threads=1, max_rounds=-1):
        counts = np.zeros(len(self.prog.preds), np.int64)
        rounds = C.c_long(0)
        secs = C.c_double(0)
        rc = lib().sko_session_run(self.h, threads, max_rounds, _p(counts, C.c_int64), C.byref(rounds),
                                   C.byref(secs))
        if rc not in (OK, E_ROUND_LIMIT):
            raise OracleError(rc)
        return ({p[0]: int(c) for p, c in zip(self.prog.preds, counts)}, int(rounds.value),
                float(secs.value))

    def close(self):
        if self.h:
            lib().sko_session_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tc_program(src, dst) -> Prog:
    """path(X,Y) :- edge(X,Y).  path(X,Z) :- edge(X,Y), path(Y,Z)."""
    p = Prog().pred("edge", 2).pred("path", 2, stratum=1)
    p.rule(("path", ["X", "Y"]), ("edge", ["X", "Y"]))
    p.rule(("path", ["X", "Z"]), ("edge", ["X", "Y"]), ("path", ["Y", "Z"]))
    p.facts_bulk("edge", [src, dst])
    return p


def trop_paths_program(src, dst, w, inf=None) -> Prog:
    p = Prog().pred("edge", 2, trop=True).pred("reach", 2, trop=True, stratum=1)
    p.rule(("reach", ["X", "Y"]), ("edge", ["X", "Y"]))
    p.rule(("reach", ["X", "Z"]), ("edge", ["X", "Y"]), ("reach", ["Y", "Z"]))
    p.facts_bulk("edge", [src, dst], w, inf)
    return p


def mssp_program(sources, src, dst, w, source_w=None) -> Prog:
    """dist(S,Y) :- src(S), edge(S,Y).  dist(S,Z) :- dist(S,Y), edge(Y,Z)."""
    p = (Prog().pred("src", 1, trop=True).pred("edge", 2, trop=True)
         .pred("dist", 2, trop=True, stratum=1))
    p.rule(("dist", ["S", "Y"]), ("src", ["S"]), ("edge", ["S", "Y"]))
    p.rule(("dist", ["S", "Z"]), ("dist", ["S", "Y"]), ("edge", ["Y", "Z"]))
    sw = np.zeros(len(sources), np.int64) if source_w is None else source_w
    p.facts_bulk("src", [sources], sw)
    p.facts_bulk("edge", [src, dst], w)
    return p


def count_program(x, y) -> Prog:
    """ntri(count<X>) :- e(X,Y), e(Y,Z), e(X,Z)."""
    p = Prog().pred("e", 2).pred("ntri", 1, stratum=1)
    p.rule(("ntri", ["N"]), ("e", ["X", "Y"]), ("e", ["Y", "Z"]), ("e", ["X", "Z"]),
           agg=("count", "X", 0))
    p.facts_bulk("e", [x, y])
    return p


# ---------------------------------------------------------------------------
# B. fast restatements
# ---------------------------------------------------------------------------
def fast_tc(src, dst):
    L = lib()
    s, d = _col(src, np.uint32), _col(dst, np.uint32)
    os_, od = C.POINTER(C.c_uint32)(), C.POINTER(C.c_uint32)()
    n = C.c_size_t()
    r = C.c_long()
    L.sko_fast_tc(_p(s, C.c_uint32), _p(d, C.c_uint32), len(s), C.byref(os_), C.byref(od),
                  C.byref(n), C.byref(r))
    a = np.ctypeslib.as_array(os_, shape=(n.value,)).copy() if n.value else np.zeros(0, np.uint32)
    b = np.ctypeslib.as_array(od, shape=(n.value,)).copy() if n.value else np.zeros(0, np.uint32)
    L.sko_free(C.cast(os_, C.c_void_p))
    L.sko_free(C.cast(od, C.c_void_p))
    return a, b, int(r.value)


def fast_trop(shape, src, dst, w, inf=None, sources=None, source_w=None):
    """shape 0: all-pairs reach; shape 1: multi-source dist.  Raises OracleError."""
    L = lib()
    s, d = _col(src, np.uint32), _col(dst, np.uint32)
    ww = _col(w, np.int64)
    ii = _col(np.zeros(len(s)) if inf is None else inf, np.uint8)
    srcs = _col(np.zeros(0) if sources is None else sources, np.uint32)
    sw = _col(np.zeros(len(srcs)) if source_w is None else source_w, np.int64)
    si = np.zeros(len(srcs), np.uint8)
    os_, od, ow, oi = (C.POINTER(C.c_uint32)(), C.POINTER(C.c_uint32)(), C.POINTER(C.c_int64)(),
                       C.POINTER(C.c_uint8)())
    n = C.c_size_t()
    r = C.c_long()
    rc = L.sko_fast_trop(shape, _p(srcs, C.c_uint32), _p(sw, C.c_int64), _p(si, C.c_uint8), len(srcs),
                         _p(s, C.c_uint32), _p(d, C.c_uint32), _p(ww, C.c_int64), _p(ii, C.c_uint8),
                         len(s), C.byref(os_), C.byref(od), C.byref(ow), C.byref(oi), C.byref(n),
                         C.byref(r))
    if rc != OK:
        raise OracleError(rc)
    m = n.value
    cols = []
    for ptr, dt in ((os_, np.uint32), (od, np.uint32), (ow, np.int64), (oi, np.uint8)):
        cols.append(np.ctypeslib.as_array(ptr, shape=(m,)).copy() if m else np.zeros(0, dt))
        L.sko_free(C.cast(ptr, C.c_void_p))
    return cols[0], cols[1], cols[2], cols[3], int(r.value)


# ---------------------------------------------------------------------------
# C. independent oracles
# ---------------------------------------------------------------------------
def fingerprint(src, dst, w=None, inf=None) -> int:
    L = lib()
    s, d = _col(src, np.uint32), _col(dst, np.uint32)
    wp = None if w is None else _p(_col(w, np.int64), C.c_int64)
    ia = None if inf is None else _col(inf, np.uint8)
    keep = [s, d]
    if w is not None:
        keep.append(_col(w, np.int64))
        wp = _p(keep[-1], C.c_int64)
    return int(L.sko_fingerprint(_p(s, C.c_uint32), _p(d, C.c_uint32), wp,
                                 None if ia is None else _p(ia, C.c_uint8), len(s)))


POLY_C = 0x9E3779B97F4A7C15


def mix64_np(x) -> np.ndarray:
    """splitmix64 finalizer on uint64 arrays (wrapping arithmetic)."""
    z = np.asarray(x, np.uint64) + np.uint64(0x9E3779B97F4A7C15)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def poly_fingerprint(x, z, n: int) -> int:
    """Σ mix64(X) · c^Z mod 2^64 over tuples (X, Z) with Z < n — the batched
    reachability summary, computed directly from tuples."""
    x = np.asarray(x, np.uint64)
    z = np.asarray(z, np.int64)
    pw = np.ones(max(n, 1), np.uint64)
    with np.errstate(over="ignore"):
        for k in range(1, n):
            pw[k] = pw[k - 1] * np.uint64(POLY_C)
        return int((mix64_np(x) * pw[z]).sum(dtype=np.uint64)) if len(x) else 0


def closure_count_fp(n, src, dst) -> tuple[int, int]:
    """|path| and the row-polynomial fingerprint of path = closure(edge) on
    nodes [0, n) (SCC + DAG oracle)."""
    s, d = _col(src, np.uint32), _col(dst, np.uint32)
    c, f = C.c_uint64(), C.c_uint64()
    rc = lib().sko_closure_count_fp(n, _p(s, C.c_uint32), _p(d, C.c_uint32), len(s), C.byref(c), C.byref(f))
    if rc:
        raise ValueError("edge endpoint outside [0, n)")
    return int(c.value), int(f.value)


def closure_batch(nodes, edge_off, src, dst, threads=8) -> tuple[np.ndarray, np.ndarray]:
    """Per-instance (count, fingerprint) of a batch (see closure_count_fp)."""
    nd = _col(nodes, np.uint32)
    eo = _col(edge_off, np.uint64)
    s, d = _col(src, np.uint32), _col(dst, np.uint32)
    counts = np.zeros(len(nd), np.uint64)
    fps = np.zeros(len(nd), np.uint64)
    rc = lib().sko_closure_batch(len(nd), _p(nd, C.c_uint32), _p(eo, C.c_uint64), _p(s, C.c_uint32),
                                 _p(d, C.c_uint32), threads, _p(counts, C.c_uint64), _p(fps, C.c_uint64))
    if rc:
        raise ValueError("edge endpoint outside its instance's node range")
    return counts, fps


# ---------------------------------------------------------------------------
# A'. provenance capture, exact compilation, WMC and gradients (FP64)
# ---------------------------------------------------------------------------
PROV_ERRS = {20: "NotBool", 21: "BadProbability", 22: "ProofBudget", 23: "SoftAggregate",
             24: "CircuitBudget"}


class ProvError(Exception):
    def __init__(self, code: int):
        super().__init__(PROV_ERRS.get(code, ERR_NAMES.get(code, str(code))))
        self.code = code


def _deser(buf, i=0):
    """[n, (len, lits...)*] -> (list of proofs, next index)."""
    n = int(buf[i]); i += 1
    out = []
    for _ in range(n):
        ln = int(buf[i]); i += 1
        out.append([int(x) for x in buf[i:i + ln]]); i += ln
    return out, i


def _ser(proofs) -> np.ndarray:
    out = [len(proofs)]
    for p in proofs:
        out.append(len(p))
        out += [int(x) for x in p]
    return np.asarray(out, np.int64)


class ProvDb:
    """The saturated provenance database of a program (run_prov)."""

    def __init__(self, prog: "Prog", probs, modes: dict | None = None, max_proofs: int = 10_000):
        L = lib()
        self.prog = prog
        self.probs = np.ascontiguousarray(probs, np.float64)
        m = np.zeros(len(prog.preds), np.int64)
        for name, k in (modes or {}).items():
            m[prog._pi(name)] = int(k)
        b = prog.blob()
        err, rounds = C.c_int(), C.c_long()
        self.h = L.sko_prov_run(_p(b, C.c_int64), len(b), _p(self.probs, C.c_double), len(self.probs),
                                _p(m, C.c_int64), max_proofs, C.byref(rounds), C.byref(err))
        if not self.h:
            raise ProvError(err.value)
        self.rounds = rounds.value

    def proofs(self, pred: str, values) -> list | None:
        vals = []
        for v in values:
            vals += [1, int(v[1])] if isinstance(v, tuple) and v[0] == "i" else [0, int(v)]
        va = np.asarray(vals, np.int64)
        cap = 1 << 16
        while True:
            buf = np.zeros(cap, np.int64)
            n = lib().sko_prov_proofs(self.h, self.prog._pi(pred), _p(va, C.c_int64), len(values),
                                      _p(buf, C.c_int64), cap)
            if n < 0:
                return None
            if n <= cap:
                return _deser(buf)[0]
            cap = n

    def relation(self, pred: str) -> dict:
        cap = 1 << 20
        while True:
            buf = np.zeros(cap, np.int64)
            n = lib().sko_prov_relation(self.h, self.prog._pi(pred), _p(buf, C.c_int64), cap)
            if n <= cap:
                break
            cap = n
        ar = self.prog.preds[self.prog._pi(pred)][1]
        cnt, i = int(buf[0]), 1
        out = {}
        for _ in range(cnt):
            t = tuple(int(buf[i + 2 * c + 1]) for c in range(ar))
            i += 2 * ar
            ps, i = _deser(buf, i)
            out[t] = ps
        return out

    def close(self):
        if self.h:
            lib().sko_prov_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def compile_grad(proofs, probs, max_nodes: int = 1 << 20):
    """compile_exact + Circuit::grad (FP64): (P, dP/dp over every leaf, nodes)."""
    pr = np.ascontiguousarray(probs, np.float64)
    ser = _ser(proofs)
    pv, g, nn = C.c_double(), np.zeros(len(pr), np.float64), C.c_int64()
    rc = lib().sko_compile_grad(_p(ser, C.c_int64), len(pr), _p(pr, C.c_double), max_nodes, C.byref(pv),
                                _p(g, C.c_double), C.byref(nn))
    if rc:
        raise ProvError(rc)
    return pv.value, g, int(nn.value)


def prov_tc(n, src, dst, probs, k, qs, qt, threads=8):
    """Prov_k capture of path(X,Y) :- edge(X,Y). path(X,Z) :- edge(X,Y), path(Y,Z).
    restricted to the queried targets; returns ([proofs per query], {target: rounds})."""
    s, d = _col(src, np.uint32), _col(dst, np.uint32)
    pr = np.ascontiguousarray(probs, np.float64)
    qs_, qt_ = _col(qs, np.uint32), _col(qt, np.uint32)
    targets = np.unique(qt_).astype(np.uint32)
    rounds = (C.c_long * max(1, len(targets)))()
    q_off = np.zeros(len(qs_) + 1, np.int64)
    need = C.c_size_t()
    cap = max(1024, 64 * len(qs_))
    while True:
        buf = np.zeros(cap, np.int64)
        rc = lib().sko_prov_tc(n, _p(s, C.c_uint32), _p(d, C.c_uint32), len(s), _p(pr, C.c_double), k,
                               _p(targets, C.c_uint32), len(targets), _p(qs_, C.c_uint32), _p(qt_, C.c_uint32),
                               len(qs_), threads, _p(buf, C.c_int64), cap, _p(q_off, C.c_int64), rounds,
                               C.byref(need))
        if rc == 0:
            break
        cap = int(need.value)
    out = [_deser(buf, int(q_off[q]))[0] for q in range(len(qs_))]
    return out, {int(t): int(rounds[i]) for i, t in enumerate(targets)}


def bfs_closure(src, dst, threads=8):
    L = lib()
    s, d = _col(src, np.uint32), _col(dst, np.uint32)
    c, f = C.c_uint64(), C.c_uint64()
    L.sko_bfs_closure(_p(s, C.c_uint32), _p(d, C.c_uint32), len(s), threads, C.byref(c), C.byref(f))
    return int(c.value), int(f.value)


def dijkstra_mssp(sources, src, dst, w, source_w=None, threads=8):
    L = lib()
    srcs = _col(sources, np.uint32)
    sw = _col(np.zeros(len(srcs)) if source_w is None else source_w, np.int64)
    s, d, ww = _col(src, np.uint32), _col(dst, np.uint32), _col(w, np.int64)
    c, f = C.c_uint64(), C.c_uint64()
    rc = L.sko_dijkstra_mssp(_p(srcs, C.c_uint32), _p(sw, C.c_int64), len(srcs), _p(s, C.c_uint32),
                             _p(d, C.c_uint32), _p(ww, C.c_int64), len(s), threads, C.byref(c), C.byref(f))
    if rc:
        raise ValueError("Dijkstra oracle needs non-negative weights")
    return int(c.value), int(f.value)


def dijkstra_mssp_rows(sources, src, dst, w, source_w=None, threads=8):
    """(S, Z, dist) for every finite distance, sorted by (S, Z): numpy
    columns uint32, uint32, int64 (Dijkstra per source, `threads` threads)."""
    L = lib()
    srcs = _col(sources, np.uint32)
    sw = _col(np.zeros(len(srcs)) if source_w is None else source_w, np.int64)
    s, d, ww = _col(src, np.uint32), _col(dst, np.uint32), _col(w, np.int64)
    ps, pd, pw, n = C.POINTER(C.c_uint32)(), C.POINTER(C.c_uint32)(), C.POINTER(C.c_int64)(), C.c_size_t()
    rc = L.sko_dijkstra_mssp_rows(_p(srcs, C.c_uint32), _p(sw, C.c_int64), len(srcs), _p(s, C.c_uint32),
                                  _p(d, C.c_uint32), _p(ww, C.c_int64), len(s), threads, C.byref(ps), C.byref(pd),
                                  C.byref(pw), C.byref(n))
    if rc:
        raise ValueError("Dijkstra oracle needs non-negative weights")
    k = n.value
    cols = [np.ctypeslib.as_array(p, shape=(max(k, 1),))[:k].copy() for p in (ps, pd, pw)]
    for p in (ps, pd, pw):
        L.sko_free(C.cast(p, C.c_void_p))
    return cols[0], cols[1], cols[2]


def count_pattern(x, y, threads=8) -> int:
    L = lib()
    a, b = _col(x, np.uint32), _col(y, np.uint32)
    return int(L.sko_count_pattern(_p(a, C.c_uint32), _p(b, C.c_uint32), len(a), threads))


def brute_triangles(a, b, nodes) -> int:
    L = lib()
    x, y = _col(a, np.uint32), _col(b, np.uint32)
    return int(L.sko_brute_triangles(_p(x, C.c_uint32), _p(y, C.c_uint32), len(x), nodes))


def brute_4cliques(a, b, nodes) -> int:
    L = lib()
    x, y = _col(a, np.uint32), _col(b, np.uint32)
    return int(L.sko_brute_4cliques(_p(x, C.c_uint32), _p(y, C.c_uint32), len(x), nodes))


def asp_simplify_filter(head, body_start, body_lit, poss, cert):
    """The grounding-simplify filter as the reference's CPU path computes it
    (crates/strata-gpu/src/asp.rs:53-100, keep_literal + simplify_filter_cpu):
    returns (head, body_start, body_lit) of the surviving rules."""
    oh, os_, ol = [], [0], []
    for i in range(len(head)):
        kept, alive = [], True
        for lit in body_lit[body_start[i]:body_start[i + 1]]:
            a, pos = abs(int(lit)) - 1, lit > 0
            if pos:
                if poss[a] == 0:
                    alive = False
                    break
                if cert[a] == 0:
                    kept.append(int(lit))
            else:
                if cert[a] != 0:
                    alive = False
                    break
                if poss[a] != 0:
                    kept.append(int(lit))
        if not alive:
            continue
        oh.append(int(head[i]))
        ol.extend(kept)
        os_.append(len(ol))
    return oh, os_, ol
