"""The planner (strata_b200.plan) on the reference planner's own cases
(crates/strata-gpu/src/plan.rs tests, contraction.rs:253-300): GYO
decomposition, the cost-based variable order with per-superstep
re-optimisation, contraction widths — and its use as the join order of
the operator-composed executor (results independent of the order)."""
import itertools

from strata_b200.plan import (Atom, Query, Stats, body_order, contraction_order, cost_based_order,
                              hypertree_decompose, order_cost, plan)


def e(a, b):
    return Atom("edge", [a, b])


def test_gyo_shapes():
    d = hypertree_decompose(Query([e(0, 1), e(1, 2), e(0, 2)]))
    assert not d.acyclic and d.width == 3 and len(d.cyclic_core) == 3
    d = hypertree_decompose(Query([e(0, 1), e(1, 2), e(2, 3)]))
    assert d.acyclic and d.width == 1 and not d.cyclic_core and len(d.join_tree) == 3
    assert hypertree_decompose(Query([e(0, 1), e(0, 2), e(0, 3)])).acyclic
    d = hypertree_decompose(Query([e(0, 1), e(1, 2), e(2, 3), e(3, 0)]))
    assert not d.acyclic and d.width == 4


def test_cbo_leads_with_the_small_relation():
    q = Query([Atom("R", [0, 1]), Atom("S", [1, 2])])
    st = Stats({"R": 10, "S": 1000}, {0: 10, 1: 100, 2: 1000})
    good, bad = order_cost([0, 1, 2], q, st), order_cost([2, 1, 0], q, st)
    assert good < bad
    order, cost = cost_based_order(q, st)
    assert cost == good and order.index(0) < order.index(2)


def test_per_superstep_reoptimisation():
    q = Query([Atom("R", [0, 1]), Atom("S", [1, 2])])
    s1 = Stats({"R": 10, "S": 1000}, {0: 10, 1: 100, 2: 1000})
    s2 = Stats({"R": 1000, "S": 10}, {0: 1000, 1: 100, 2: 10})
    o1, _ = cost_based_order(q, s1)
    o2, _ = cost_based_order(q, s2)
    assert o1[0] == 0 and o2[0] == 2 and o1 != o2


def test_plan_and_contraction_widths():
    p = plan(Query([e(0, 1), e(1, 2), e(0, 2)]), Stats({"edge": 1000}, {0: 100, 1: 100, 2: 100}))
    assert not p.decomposition.acyclic and len(p.order) == 3
    assert p.contraction_width == 3 == p.decomposition.width
    p = plan(Query([e(0, 1), e(1, 2), e(2, 3)]), Stats())
    assert p.decomposition.acyclic and p.contraction_width == 2
    c = contraction_order(Query([e(0, 1), e(1, 2), e(0, 2)]))
    assert c.width == 3 and len(c.order) == 3


def test_exhaustive_order_is_the_first_minimum():
    q = Query([Atom("A", [0, 1]), Atom("B", [1, 2]), Atom("C", [2, 3]), Atom("D", [3, 0])])
    st = Stats({"A": 5, "B": 500, "C": 50, "D": 5000}, {0: 7, 1: 70, 2: 700, 3: 7000})
    order, cost = cost_based_order(q, st)
    costs = [(order_cost(o, q, st), o) for o in itertools.permutations(q.vars())]
    m = min(c for c, _ in costs)
    assert cost == m and list(next(o for c, o in costs if c == m)) == order
    # greedy above eight variables still returns every variable once
    big = Query([Atom(f"r{i}", [i, i + 1]) for i in range(10)])
    o, _ = cost_based_order(big, Stats())
    assert sorted(o) == list(range(11))


def test_body_order_follows_the_variable_order():
    # a(X,Y) large, b(Y,Z) tiny: the tiny atom is bound first
    assert body_order([["X", "Y"], ["Y", "Z"]], [1_000_000, 3], 1000) == [1, 0]
    assert body_order([["X", "Y"], ["Y", "Z"]], [3, 1_000_000], 1000) == [0, 1]
