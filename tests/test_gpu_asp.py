"""The ASP grounding-simplify filter on the device (strata_asp_simplify_filter)
against the reference's CPU semantics restated in the oracle
(crates/strata-gpu/src/asp.rs:53-100) — exact arrays."""
import numpy as np
import pytest

import oracle as O
import strata_b200 as S

pytestmark = pytest.mark.gpu


def _prog(rng, n_rules, n_atoms, max_body=6):
    lens = rng.integers(0, max_body + 1, n_rules)
    start = np.zeros(n_rules + 1, np.uint32)
    start[1:] = np.cumsum(lens)
    atoms = rng.integers(0, n_atoms, int(start[-1]))
    sign = np.where(rng.random(int(start[-1])) < 0.7, 1, -1)
    lits = ((atoms + 1) * sign).astype(np.int32)
    head = rng.integers(-1, n_atoms, n_rules).astype(np.int32)
    return head, start, lits


def test_reference_case(engine):
    h, s, l = engine.asp_simplify_filter([3, 3], [0, 2, 4], [1, -3, 2, 3], [1, 1, 0, 1], [1, 1, 0, 0])
    assert h.tolist() == [3] and s.tolist() == [0, 0] and l.tolist() == []


@pytest.mark.parametrize("n_rules,n_atoms", [(1, 1), (1000, 50), (200_000, 5000), (3_000_000, 100_000)])
def test_random_programs_match_the_cpu_filter(engine, n_rules, n_atoms):
    rng = np.random.default_rng(n_rules)
    head, start, lits = _prog(rng, n_rules, n_atoms)
    poss = (rng.random(n_atoms) < 0.8).astype(np.uint8)
    cert = (rng.random(n_atoms) < 0.3).astype(np.uint8)  # some certain-but-not-possible: read as the CPU path does
    gh, gs, gl = engine.asp_simplify_filter(head, start, lits, poss, cert)
    if n_rules <= 200_000:
        wh, ws, wl = O.asp_simplify_filter(head, start, lits, poss, cert)
        assert gh.tolist() == wh and gs.tolist() == ws and gl.tolist() == wl
    else:  # vectorised restatement for the large case
        a = np.abs(lits) - 1
        pos = lits > 0
        dies = np.where(pos, poss[a] == 0, cert[a] != 0)
        keep = np.where(pos, cert[a] == 0, poss[a] != 0) & ~dies
        rule_of = np.repeat(np.arange(n_rules), np.diff(start.astype(np.int64)))
        dead = np.zeros(n_rules, bool)
        np.logical_or.at(dead, rule_of, dies)
        alive = ~dead
        assert np.array_equal(gh, head[alive])
        kept_lits = lits[keep & alive[rule_of]]
        assert np.array_equal(gl, kept_lits)
        per = np.bincount(rule_of[keep & alive[rule_of]], minlength=n_rules)[alive]
        assert np.array_equal(gs[1:].astype(np.int64), np.cumsum(per))


def test_literal_naming_no_atom_is_refused(engine):
    with pytest.raises(S.Cuda):
        engine.asp_simplify_filter([0], [0, 1], [5], [1, 1], [0, 0])
    with pytest.raises(S.Cuda):
        engine.asp_simplify_filter([0], [0, 1], [0], [1, 1], [0, 0])
