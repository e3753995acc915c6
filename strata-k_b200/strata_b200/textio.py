"""The input and output contracts around the fixpoint (host side).

* ``SymbolDict`` — first-seen interning (strata-ir/src/dict.rs:24-43): ids are
  assigned in order of first sight, so the same input yields the same ids.
* ``load_tsv`` — Soufflé TSV rows split on tab, empty lines skipped, a Trop
  predicate's trailing column parsed as an i64 weight, a neural predicate's
  as a probability in [0, 1] (strata-k/src/input.rs:53-197, 204-234).
* ``load_tsv_device`` / ``render_relation_device`` — the same two contracts
  on the GPU (strata_tsv_load, strata_rel_render).
* ``render_db`` — canonical text: relations in name order, tuples in id order,
  ``pred(a, b)`` with `` = w`` / `` = inf`` for Trop (strata-cli/src/render.rs:29-92,
  strata-ir/src/output.rs:11).  A non-empty ``queries`` list filters the
  output like plain ``?q(...)`` queries (render.rs:21-64).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

POS_INF_TOKEN = "inf"


class SymbolDict:
    def __init__(self):
        self.by_str: dict[str, int] = {}
        self.by_id: list[str] = []

    def intern(self, s: str) -> int:
        i = self.by_str.get(s)
        if i is None:
            i = len(self.by_id)
            self.by_id.append(s)
            self.by_str[s] = i
        return i

    def get(self, s: str) -> int | None:
        return self.by_str.get(s)

    def resolve(self, i: int) -> str:
        return self.by_id[i] if 0 <= i < len(self.by_id) else "?"

    def __len__(self) -> int:
        return len(self.by_id)


class InputError(ValueError):
    pass


def _rows(source) -> list[tuple[int, list[str]]]:
    if isinstance(source, (str, Path)):
        text = Path(source).read_text()
        out = []
        for i, line in enumerate(text.splitlines()):
            line = line.rstrip("\r")
            if not line:
                continue
            out.append((i + 1, line.split("\t")))
        return out
    return [(i + 1, list(r)) for i, r in enumerate(source)]


def load_tsv(source, arity: int, dictionary: SymbolDict, trop: bool = False,
             neural: bool = False):
    """Parse rows of ``arity`` symbol columns (+ a trailing weight / probability).

    Returns (list of id columns as uint32 arrays, weights or None).  Errors
    follow input.rs: wrong column count, empty cell, unparsable trailing value,
    probability outside [0, 1].
    """
    rows = _rows(source)
    ncols = arity + (1 if (trop or neural) else 0)
    cols = [np.zeros(len(rows), np.uint32) for _ in range(arity)]
    weights = np.zeros(len(rows), np.int64) if trop else (np.zeros(len(rows)) if neural else None)
    for k, (lineno, cells) in enumerate(rows):
        if len(cells) != ncols:
            raise InputError(f"{lineno}: expects {ncols} column(s), found {len(cells)}")
        for c in range(arity):
            if cells[c] == "":
                raise InputError(f"{lineno}: empty value in column {c + 1}")
            cols[c][k] = dictionary.intern(cells[c])
        if trop:
            try:
                weights[k] = int(cells[arity].strip())
            except ValueError:
                raise InputError(f"{lineno}: needs a trailing integer weight") from None
        elif neural:
            try:
                p = float(cells[arity].strip())
            except ValueError:
                raise InputError(f"{lineno}: needs a trailing probability") from None
            if not 0.0 <= p <= 1.0:
                raise InputError(f"{lineno}: probability {p} is outside [0, 1]")
            weights[k] = p
    return cols, weights


def _dict_buffers(dictionary: SymbolDict):
    enc = [x.encode() for x in dictionary.by_id]
    off = np.zeros(len(enc) + 1, np.uint64)
    if enc:
        off[1:] = np.cumsum([len(e) for e in enc])
    return b"".join(enc), off


def load_tsv_device(eng, text, arity: int, dictionary: SymbolDict, trop: bool = False):
    """``load_tsv`` on the device (strata_tsv_load): the same rows, ids and
    errors; new symbols are appended to ``dictionary`` in first-seen order."""
    import ctypes as C

    from . import _lib as L
    data = text.encode() if isinstance(text, str) else bytes(text)
    dbytes, doff = _dict_buffers(dictionary)
    cols_p, w_p = C.POINTER(C.c_uint32)(), C.POINTER(C.c_int64)()
    rows, n_new, eline, ecol = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint32()
    nb, no = C.c_void_p(), C.POINTER(C.c_uint64)()
    rc = eng.lib.strata_tsv_load(eng.ctx, data, len(data), arity, 1 if trop else 0, dbytes or None,
                                 doff.ctypes.data_as(C.c_void_p), len(dictionary), C.byref(cols_p),
                                 C.byref(w_p) if trop else None, C.byref(rows), C.byref(nb), C.byref(no),
                                 C.byref(n_new), C.byref(eline), C.byref(ecol))
    if rc == L.E_INVALID and eline.value:
        raise InputError(eng.lib.strata_last_error(eng.ctx).decode())
    eng._check(rc)
    n = rows.value
    flat = np.ctypeslib.as_array(cols_p, shape=(max(1, n * arity),))[:n * arity].copy()
    eng.lib.strata_free(C.cast(cols_p, C.c_void_p))
    weights = None
    if trop:
        weights = np.ctypeslib.as_array(w_p, shape=(max(1, n),))[:n].copy()
        eng.lib.strata_free(C.cast(w_p, C.c_void_p))
    k = n_new.value
    offs = np.ctypeslib.as_array(no, shape=(k + 1,)).copy()
    raw = C.string_at(nb, int(offs[-1])) if k else b""
    for j in range(k):
        dictionary.intern(raw[int(offs[j]):int(offs[j + 1])].decode())
    eng.lib.strata_free(nb)
    eng.lib.strata_free(C.cast(no, C.c_void_p))
    return [flat[c * n:(c + 1) * n].astype(np.uint32) for c in range(arity)], weights


def render_relation_device(eng, rel, name: str, dictionary: SymbolDict) -> str:
    """The canonical text of a device relation (strata_rel_render): the same
    lines ``render_relation`` prints, built on the GPU."""
    import ctypes as C
    dbytes, doff = _dict_buffers(dictionary)
    out, n = C.c_void_p(), C.c_uint64()
    eng._check(eng.lib.strata_rel_render(eng.ctx, rel.rel, name.encode(), dbytes or None,
                                         doff.ctypes.data_as(C.c_void_p), len(dictionary), C.byref(out), C.byref(n)))
    text = C.string_at(out, n.value).decode()
    eng.lib.strata_free(out)
    return text


def render_weight(w: int, inf: bool) -> str:
    return POS_INF_TOKEN if inf else str(int(w))


def render_relation(name: str, cols, dictionary: SymbolDict, w=None, inf=None,
                    queries=None) -> list[str]:
    """Lines for one relation; ``cols`` are id columns already in id order."""
    n = len(cols[0]) if cols else 0
    names = [[dictionary.resolve(int(v)) for v in c] for c in cols]
    out = []
    for i in range(n):
        vals = [names[c][i] for c in range(len(cols))]
        if queries and not any(_match(q, name, vals) for q in queries):
            continue
        line = f"{name}({', '.join(vals)})"
        if w is not None:
            line += " = " + render_weight(w[i], bool(inf[i]) if inf is not None else False)
        out.append(line)
    return out


def _match(q, name, vals) -> bool:
    qname, pattern = q
    if qname != name or len(pattern) != len(vals):
        return False
    return all(p is None or p == v for p, v in zip(pattern, vals))


def render_db(relations: dict, dictionary: SymbolDict, queries=None) -> str:
    """``relations``: name -> (cols, w, inf) with rows sorted by id tuple."""
    lines = []
    for name in sorted(relations):
        if queries and not any(q[0] == name for q in queries):
            continue
        cols, w, inf = relations[name]
        lines += render_relation(name, cols, dictionary, w, inf, queries)
    return "".join(l + "\n" for l in lines)


def render_f64(x: float) -> str:
    """A float as the reference prints one (Rust's `{}` for f64): the shortest
    decimal that reads back to the same double, positional (no exponent),
    integral values without a fraction (`1`, `0`, `-0`)."""
    import math
    from decimal import Decimal
    x = float(x)
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "inf" if x > 0 else "-inf"
    if x == 0.0:
        return "-0" if math.copysign(1.0, x) < 0 else "0"
    r = repr(x)
    if "e" in r or "E" in r:
        r = format(Decimal(r), "f")
    if r.endswith(".0"):
        r = r[:-2]
    return r


def prob_line(p: float, pred: str, args: list[str], top_k: int | None = None) -> str:
    """`p :: pred(a, b)` — and for a Prov_k predicate the declared lower bound
    marker (strata-cli/src/prov.rs:64-82, render.rs:10)."""
    s = f"{render_f64(p)} :: {pred}({', '.join(args)})"
    if top_k is not None:
        s += f"  (lower bound, top-{top_k})"
    return s + "\n"


def grad_line(fact_p: float, pred: str, args: list[str], g: float, model: str | None = None) -> str:
    """One `?grad` line per probabilistic fact (strata-cli/src/prob.rs:174-189)."""
    s = f"  ∂/∂[{render_f64(fact_p)} :: {pred}({', '.join(args)})] = {render_f64(g)}"
    if model is not None:
        s += f'  (→ model "{model}")'
    return s + "\n"
