"""The input and output contracts on the device: strata_tsv_load (TSV rows,
first-seen interning, trailing i64 weights and their errors,
strata-k/src/input.rs:53-232) against the host restatement, and
strata_rel_render (strata-cli/src/render.rs:29-92) of GPU relations against
the host renderer and the routing workload's pinned lines
(strata-cli/tests/workloads.rs:26-32).  Exact text and ids."""
import json
from pathlib import Path

import numpy as np
import pytest

import strata_b200 as S
from strata_b200 import textio as T

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def _tsv(rows):
    return "".join("\t".join(r) + "\n" for r in rows)


def _both(engine, text, arity, trop, seed_syms=()):
    hd, dd = T.SymbolDict(), T.SymbolDict()
    for x in seed_syms:
        hd.intern(x), dd.intern(x)
    h = T.load_tsv([ln.split("\t") for ln in text.splitlines() if ln.rstrip("\r")], arity, hd, trop=trop) \
        if text else ([np.zeros(0, np.uint32)] * arity, np.zeros(0, np.int64) if trop else None)
    d = T.load_tsv_device(engine, text, arity, dd, trop=trop)
    return h, d, hd, dd


def test_routing_tsv_on_device_matches_host_ids(engine):
    g = json.loads((GOLDEN / "routing.json").read_text())
    seeds = [x for q in g["queries"] for x in q]
    (hc, hw), (dc, dw), hd, dd = _both(engine, _tsv(g["rows"]), 2, True, seeds)
    assert all(np.array_equal(a, b) for a, b in zip(hc, dc))
    assert np.array_equal(hw, dw)
    assert hd.by_id == dd.by_id


def test_tsv_line_endings_whitespace_and_weights(engine):
    text = "a\tb\t 5 \r\n\r\n\nb\tc\t+3\nc\ta\t-0\r\r\na\ta\t9223372036854775807\nb\tb\t-9223372036854775808"
    dd = T.SymbolDict()
    cols, w = T.load_tsv_device(engine, text, 2, dd, trop=True)
    assert dd.by_id == ["a", "b", "c"]
    assert cols[0].tolist() == [0, 1, 2, 0, 1] and cols[1].tolist() == [1, 2, 0, 0, 1]
    assert w.tolist() == [5, 3, 0, 2**63 - 1, -2**63]
    # unicode whitespace around the weight is trimmed (str::trim), symbols are verbatim
    cols, w = T.load_tsv_device(engine, "x y\t z\t　 7 \n", 2, dd, trop=True)
    assert w.tolist() == [7] and dd.by_id[-2:] == ["x y", " z"]


@pytest.mark.parametrize("text,line,col", [
    ("a\tb\n\nc\n", 3, 0),                  # too few cells
    ("a\tb\nc\t\td\n", 2, 0),              # too many cells
    ("a\tb\n\tb\n", 2, 1),                 # empty symbol cell
    ("a\tb\nb\t\n", 2, 2),
])
def test_tsv_row_errors_report_the_first_bad_line(engine, text, line, col):
    dd = T.SymbolDict()
    with pytest.raises(T.InputError, match=f"line {line}:"):
        T.load_tsv_device(engine, text, 2, dd)
    assert len(dd) == 0  # nothing is committed


@pytest.mark.parametrize("cell", ["5x", "", " ", "1_000", "9223372036854775808", "-9223372036854775809", "+", "--1"])
def test_tsv_bad_weights(engine, cell):
    with pytest.raises(T.InputError, match="line 2:"):
        T.load_tsv_device(engine, f"a\tb\t1\nb\tc\t{cell}\n", 2, T.SymbolDict(), trop=True)


def test_large_random_tsv_matches_host_interning(engine):
    rng = np.random.default_rng(9)
    names = np.array([f"n{int(x)}" for x in rng.integers(0, 200_000, 50_000)])
    a = names[rng.integers(0, len(names), 400_000)]
    b = names[rng.integers(0, len(names), 400_000)]
    text = "".join(f"{x}\t{y}\n" for x, y in zip(a, b))
    (hc, _), (dc, _), hd, dd = _both(engine, text, 2, False, ["n17", "zz"])
    assert all(np.array_equal(x, y) for x, y in zip(hc, dc))
    assert hd.by_id == dd.by_id
    # unary rows, appended to the same dictionary
    cols, _ = T.load_tsv_device(engine, "n5\nfresh\nn5\n", 1, dd)
    assert cols[0].tolist() == [dd.get("n5"), dd.get("fresh"), dd.get("n5")]


def test_render_gpu_relations_like_the_host_and_the_pinned_routing_lines(engine):
    import torch
    g = json.loads((GOLDEN / "routing.json").read_text())
    dd = T.SymbolDict()
    for a, b in g["queries"]:
        dd.intern(a), dd.intern(b)
    (s, d), w = T.load_tsv_device(engine, _tsv(g["rows"]), 2, dd, trop=True)
    t = lambda x, dt: torch.from_numpy(np.ascontiguousarray(x).astype(dt)).cuda()
    rel = engine.trop_paths_dev(t(s, np.int32), t(d, np.int32), t(w, np.int64))
    try:
        text = T.render_relation_device(engine, rel, "route", dd)
        host = rel.to_host()
        want = T.render_db({"route": ([host.src, host.dst], host.w, host.inf)}, dd)
        assert text == want
        lines = set(text.splitlines())
        assert all(p in lines for p in g["pinned"])
    finally:
        rel.free()
    # a Bool closure, symbols named from a longer dictionary
    bd = T.SymbolDict()
    for i in range(400):
        bd.intern(f"v{i}")
    rng = np.random.default_rng(4)
    src, dst = rng.integers(0, 400, 900), rng.integers(0, 400, 900)
    rel = engine.tc_bool_dev(t(src, np.int32), t(dst, np.int32))
    try:
        host = rel.to_host()
        assert T.render_relation_device(engine, rel, "path", bd) == T.render_db({"path": ([host.src, host.dst], None, None)}, bd)
    finally:
        rel.free()
