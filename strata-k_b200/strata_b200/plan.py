"""Query planning for multi-atom rule bodies: the hypertree decomposition
(GYO ear removal), the cost-based variable order and the min-degree
contraction width of the reference's planner
(crates/strata-gpu/src/plan.rs:83-262, crates/strata-gpu/src/contraction.rs:49-86).

The results must equal the reference's (same orders, same tie-breaks), so
the estimates follow its definitions: cardinalities default to 1000 and
domains to 1 when unknown, products saturate at 2^128 - 1 like u128, orders
are enumerated lexicographically over the sorted variables for at most 8
variables (the first minimum wins), greedily above that.

``strata_b200.ops.Program`` uses ``body_order`` to pick the join order of a
rule body from the variable order.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass, field

U128 = (1 << 128) - 1


def _sat(x: int) -> int:
    return x if x <= U128 else U128


@dataclass
class Atom:
    rel: str
    vars: list

    def varset(self) -> set:
        return set(self.vars)


@dataclass
class Query:
    atoms: list

    def vars(self) -> list:
        return sorted({v for a in self.atoms for v in a.vars})


@dataclass
class Decomposition:
    acyclic: bool
    width: int
    cyclic_core: list
    join_tree: list  # (atom, parent atom or None) in ear-removal order


def hypertree_decompose(q: Query) -> Decomposition:
    """GYO: repeatedly remove an ear — an atom whose variables shared with the
    other remaining atoms all lie in one of them (its parent), or that shares
    none — taking the first ear in atom order; what remains is the cyclic core."""
    vs = [a.varset() for a in q.atoms]
    alive = list(range(len(q.atoms)))
    tree = []
    while True:
        ear = None
        for e in alive:
            shared = {v for v in vs[e] if any(o != e and v in vs[o] for o in alive)}
            parent = next((o for o in alive if o != e and shared <= vs[o]), None)
            if not shared or parent is not None:
                ear = (e, parent)
                break
        if ear is None:
            break
        tree.append(ear)
        alive.remove(ear[0])
    acyclic = not alive
    return Decomposition(acyclic, 1 if acyclic else len(alive), alive, tree)


@dataclass
class Stats:
    card: dict = field(default_factory=dict)
    domain: dict = field(default_factory=dict)

    def card_of(self, rel) -> int:
        return int(self.card.get(rel, 1000))

    def domain_of(self, v) -> int:
        return max(int(self.domain.get(v, 1)), 1)


def est_join_size(atoms, stats: Stats) -> int:
    """Independence estimate Π|R| / Π_v D(v)^(k_v - 1), at least 1."""
    num, count = 1, {}
    for a in atoms:
        num = _sat(num * stats.card_of(a.rel))
        for v in a.vars:
            count[v] = count.get(v, 0) + 1
    den = 1
    for v, k in count.items():
        if k >= 2:
            den = _sat(den * _sat(stats.domain_of(v) ** (k - 1)))
    return max(num // max(den, 1), 1)


def est_prefix(prefix: set, q: Query, stats: Stats) -> int:
    """Bindings of the prefix variables: the join of the atoms it covers, times
    the domains of prefix variables no covered atom binds."""
    closed = [a for a in q.atoms if all(v in prefix for v in a.vars)]
    est = est_join_size(closed, stats)
    covered = {v for a in closed for v in a.vars}
    for v in sorted(prefix):
        if v not in covered:
            est = _sat(est * stats.domain_of(v))
    return est


def order_cost(order, q: Query, stats: Stats) -> int:
    """Sum of the estimated partial-result sizes after each variable."""
    prefix, cost = set(), 0
    for v in order:
        prefix.add(v)
        cost = _sat(cost + est_prefix(prefix, q, stats))
    return cost


def cost_based_order(q: Query, stats: Stats) -> tuple[list, int]:
    vs = q.vars()
    if len(vs) <= 8:
        best = None
        for o in itertools.permutations(vs):
            c = order_cost(o, q, stats)
            if best is None or c < best[1]:
                best = (list(o), c)
        return best if best is not None else ([], 0)
    order, remaining = [], sorted(vs)
    while remaining:
        nxt = min(remaining, key=lambda v: order_cost(order + [v], q, stats))
        order.append(nxt)
        remaining.remove(nxt)
    return order, order_cost(order, q, stats)


@dataclass
class Contraction:
    order: list
    width: int


def contraction_order(q: Query) -> Contraction:
    """Min-degree elimination on the interaction graph (ties to the smallest
    variable), with fill-in; width = the largest eliminated closed
    neighbourhood (treewidth + 1 of the heuristic)."""
    g = {v: set() for v in q.vars()}
    for a in q.atoms:
        for i, u in enumerate(a.vars):
            for w in a.vars[i + 1:]:
                if u != w:
                    g[u].add(w)
                    g[w].add(u)
    order, width = [], 0
    while g:
        v = min(g, key=lambda x: (len(g[x]), x))
        nb = sorted(g[v])
        width = max(width, len(nb) + 1)
        for i in range(len(nb)):
            for j in range(i + 1, len(nb)):
                g[nb[i]].add(nb[j])
                g[nb[j]].add(nb[i])
        for n in nb:
            g[n].discard(v)
        del g[v]
        order.append(v)
    return Contraction(order, width)


@dataclass
class Plan:
    decomposition: Decomposition
    order: list
    est_cost: int
    contraction_width: int


def plan(q: Query, stats: Stats) -> Plan:
    d = hypertree_decompose(q)
    order, cost = cost_based_order(q, stats)
    return Plan(d, order, cost, contraction_order(q).width)


def body_order(atoms: list, cards: list, domain: int) -> list:
    """Join order of a rule body's positive atoms from the cost-based variable
    order: atom i is placed when its last variable is bound (ties keep the
    written order).  `atoms` are lists of variable names, `cards` the atoms'
    relation sizes, `domain` the symbol universe."""
    names = sorted({v for a in atoms for v in a})
    idx = {v: i for i, v in enumerate(names)}
    q = Query([Atom(f"r{i}", [idx[v] for v in a]) for i, a in enumerate(atoms)])
    st = Stats({f"r{i}": int(c) for i, c in enumerate(cards)}, {i: int(domain) for i in range(len(names))})
    order, _ = cost_based_order(q, st)
    rank = {v: k for k, v in enumerate(order)}
    key = [max((rank[idx[v]] for v in a), default=-1) for a in atoms]
    return sorted(range(len(atoms)), key=lambda i: (key[i], i))
