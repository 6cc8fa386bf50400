"""Join ordering under estimated set cardinalities (CPU only: no device).

The join-order program weighs the executor's plans (one pipeline per input,
each probing the tables built from the branches hanging off it) with the
reference's cost model (engine/query/QueryGraph.cpp:62-66, 70-87): a join
costs its result's cardinality plus 10 x the hashed side's. The cardinality
of a connected input set comes either from the reference's row-count model
(the largest input's rows, QueryGraph.cpp:53-68) or from an estimator
(sampling or the learned MLP) as one number per set. Here the program under
arbitrary set cardinalities is checked against an exhaustive enumeration of
those plans, and the sub-plan enumeration against brute force.
"""
import itertools
import random

import pytest

from test_planner import _tree_plan


def _connected(mask, edges):
    nodes = [i for i in range(32) if mask >> i & 1]
    seen = {nodes[0]}
    stack = [nodes[0]]
    while stack:
        x = stack.pop()
        for a, b in edges:
            for u, v in ((a, b), (b, a)):
                if u == x and (mask >> v & 1) and v not in seen:
                    seen.add(v)
                    stack.append(v)
    return len(seen) == len(nodes)


def _exhaustive(n, edges, setcard):
    """Minimum cost and its driver over every plan the executor can run,
    a set's cardinality being setcard[mask]."""
    nbr = {i: set() for i in range(n)}
    for a, b in edges:
        nbr[a].add(b)
        nbr[b].add(a)

    def branch(v, away):
        seen, stack = {v}, [v]
        while stack:
            x = stack.pop()
            for y in nbr[x]:
                if y != away and y not in seen:
                    seen.add(y)
                    stack.append(y)
        return frozenset(seen)

    def m(S):
        return sum(1 << i for i in S)

    def cost(S, d):
        kids = [v for v in nbr[d] if v in S]
        best = None
        for perm in itertools.permutations(kids):
            c, cur = setcard[1 << d], {d}
            for v in perm:
                L = branch(v, d) & S
                c += cost(L, v)
                cur |= L
                c += setcard[m(cur)] + 10 * setcard[m(L)]
            best = c if best is None else min(best, c)
        return setcard[1 << d] if best is None else best

    full = frozenset(range(n))
    return [cost(full, d) for d in range(n)]


def _random_tree(rng, n):
    rows = [rng.choice([5, 20, 60, 200]) for _ in range(n)]
    edges = [(rng.randrange(c), c) for c in range(1, n)]
    return rows, edges


def _scan_edges(edges):
    # _tree_plan numbers scans in the order inputs join (the left-deep
    # tree's depth-first order): scan k is order[k].
    order = [edges[0][0]] + [c for _, c in edges]
    pos = {t: k for k, t in enumerate(order)}
    return order, [(pos[a], pos[b]) for a, b in edges]


@pytest.mark.parametrize("seed", range(6))
def test_subplans_are_the_connected_sets(pkg, seed):
    rng = random.Random(seed)
    n = rng.randint(2, 7)
    rows, edges = _random_tree(rng, n)
    plan = _tree_plan(pkg, rows, edges)
    _, sedges = _scan_edges(edges)
    for max_tables in (2, 3, n):
        got = list(pkg.subplans(pkg.CPlan(plan), max_tables))
        want = [m for m in range(1, 1 << n) if bin(m).count("1") <= max_tables and _connected(m, sedges)]
        assert got == want


@pytest.mark.parametrize("seed", range(10))
def test_join_order_under_set_cards_matches_exhaustive(pkg, seed):
    rng = random.Random(100 + seed)
    n = rng.randint(2, 6)
    rows, edges = _random_tree(rng, n)
    plan = pkg.CPlan(_tree_plan(pkg, rows, edges))
    order, sedges = _scan_edges(edges)
    # Arbitrary cardinalities per connected set (singletons: the input's rows).
    cards = [0.0] * (1 << n)
    for m in range(1, 1 << n):
        if bin(m).count("1") == 1:
            cards[m] = float(rows[order[m.bit_length() - 1]])
        elif _connected(m, sedges):
            cards[m] = float(rng.choice([1, 7, 50, 300, 5000]))
    costs = _exhaustive(n, sedges, cards)
    driver, cost = pkg.join_order(plan, cards)
    assert cost == pytest.approx(min(costs))
    assert costs[driver] == pytest.approx(min(costs))
    # Costing a given driver returns that driver's best plan.
    for d in range(n):
        dd, c = pkg.join_order(plan, cards, d)
        assert dd == d and c == pytest.approx(costs[d])


def test_join_order_without_cards_is_the_row_count_model(pkg):
    rows, edges = [300, 10, 300], [(0, 1), (1, 2)]
    plan = pkg.CPlan(_tree_plan(pkg, rows, edges))
    driver, cost = pkg.join_order(plan)
    assert driver == 0 and cost == pytest.approx(7210)
    # The same model written out as set cardinalities gives the same plan.
    cards = [0.0] * 8
    for m in range(1, 8):
        cards[m] = float(max(rows[i] for i in range(3) if m >> i & 1))
    assert pkg.join_order(plan, cards) == (driver, pytest.approx(cost))


def test_a_small_join_result_moves_the_driver(pkg):
    """A chain A(1000) - B(100) - C(900): with row counts A drives. If B joined
    with C is tiny, hashing B's branch (B+C) and driving from A stays best;
    if A joined with B is tiny and B with C huge, C drives instead."""
    rows, edges = [1000, 100, 900], [(0, 1), (1, 2)]
    plan = pkg.CPlan(_tree_plan(pkg, rows, edges))
    cards = [0.0] * 8
    cards[1], cards[2], cards[4] = 1000.0, 100.0, 900.0
    cards[3], cards[6], cards[7] = 5.0, 50000.0, 5.0  # AB tiny, BC huge
    driver, _ = pkg.join_order(plan, cards)
    assert driver == 2
    cards[3], cards[6] = 50000.0, 5.0  # AB huge, BC tiny
    driver, _ = pkg.join_order(plan, cards)
    assert driver == 0
