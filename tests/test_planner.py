"""Join ordering (CPU only: the planner needs no device).

The planner roots the join tree at the driver of the cheapest plan under the
reference's cost model (engine/query/QueryGraph.cpp:62-66, 70-87, 120-145):
a join costs the cardinality of its result plus 10 x the cardinality of the
side that is hashed, a result's cardinality is the largest of its inputs',
and a base input costs its cardinality. The plans it weighs are the ones the
executor runs: a pipeline scans one input (its driver), probes the tables
built from the branches hanging off that input, in some order, and each
branch is planned the same way with the input next to the driver as its own
driver. Here an exhaustive enumeration of those plans (every driver, every
order of every pipeline's branches) checks the planner's dynamic program."""
import itertools
import random
import re

import pytest


def _tree_plan(pkg, rows, edges):
    """A plan over inputs with the given row counts whose join nodes link
    exactly the input pairs in `edges` (a tree, each edge (parent, child)
    with the parent already joined). Every input has one INT32 column; each
    join node keeps every attribute, so later joins can use any input's."""
    plan = pkg.Plan()
    for r in rows:
        plan.new_input(pkg.table_from_rows([[i % 7] for i in range(r)], [pkg.INT32]))
    order = [edges[0][0]] + [c for _, c in edges]
    node = plan.new_scan_node(order[0], [(0, pkg.INT32)])
    pos = {order[0]: 0}  # input -> attribute index in the current node's output
    for parent, child in edges:
        scan = plan.new_scan_node(child, [(0, pkg.INT32)])
        width = len(pos)
        outs = [(i, pkg.INT32) for i in range(width + 1)]
        node = plan.new_join_node(True, node, scan, pos[parent], 0, outs)
        pos[child] = width
    plan.root = node
    return plan


def _exhaustive(card, edges):
    """Minimum cost and its driver over every plan the executor can run."""
    n = len(card)
    nbr = {i: set() for i in range(n)}
    for a, b in edges:
        nbr[a].add(b)
        nbr[b].add(a)

    def branch(v, away):  # inputs reachable from v without passing `away`
        seen, stack = {v}, [v]
        while stack:
            x = stack.pop()
            for y in nbr[x]:
                if y != away and y not in seen:
                    seen.add(y)
                    stack.append(y)
        return frozenset(seen)

    def cost(S, d):
        kids = [v for v in nbr[d] if v in S]
        best = None
        for perm in itertools.permutations(kids):
            c, cur = card[d], {d}
            for v in perm:
                L = branch(v, d) & S
                c += cost(L, v)
                cur |= L
                c += max(card[i] for i in cur) + 10 * max(card[i] for i in L)
            best = c if best is None else min(best, c)
        return card[d] if best is None else best

    full = frozenset(range(n))
    costs = [cost(full, d) for d in range(n)]
    best = min(costs)
    drivers = [d for d in range(n) if costs[d] == best]
    drivers.sort(key=lambda d: (-card[d], d))
    return best, drivers[0]


def _explained(pkg, plan):
    """(driver, cost) of the cheapest rooted plan, and the explain text (the
    plan run may be the reference space's when that is cheaper)."""
    text = pkg.explain(plan)
    m = re.search(r"rooted plan space, cheapest: driver input (\d+), cost ([0-9.e+]+)", text)
    assert m, text
    return int(m.group(1)), float(m.group(2)), text


def test_snowflake_is_driven_by_the_fact(pkg):
    w = pkg.Workload("snowflake", 2, 0.002)
    text = pkg.explain(w.plan_ptr())
    lines = text.strip().splitlines()
    assert re.match(r"driver: input \d+ \(table 0, ", lines[0]), text  # table 0 is the fact
    # four dimension builds, then the fact's pipeline probing all four
    pipes = [l for l in lines if l.startswith("pipeline")]
    assert len(pipes) == 5 and pipes[-1].endswith("-> result"), text
    assert pipes[-1].count("pipeline") == 5 and all("hash table" in l for l in pipes[:4]), text


def test_tie_goes_to_the_larger_input(pkg):
    """A 10-row hub joined with two 300-row inputs: driving from the hub
    hashes both large inputs (10 + 300 + 300 + (300 + 3,000) x 2 = 7,210),
    driving from a large input hashes the other one and the hub's branch
    (300 + (10 + 300 + 300 + 3,000) + 300 + 3,000 = 7,210). On equal cost the
    larger input drives (it is never hashed), then the lower index."""
    plan = _tree_plan(pkg, [300, 10, 300], [(0, 1), (1, 2)])
    driver, cost, text = _explained(pkg, plan)
    assert driver == 0, text
    assert cost == pytest.approx(7210), text
    # The reference's space has a cheaper plan (input 2 probes the hub and
    # its result is hashed on the hub's other key, carried as payload:
    # 10 + 300 + (300 + 100) + 300 + (300 + 3,000) = 4,310), and it runs.
    assert "runs: the reference space's plan" in text, text
    pipes = [l for l in text.strip().splitlines() if l.startswith("pipeline")]
    assert pipes[-1].startswith("pipeline 2: scan input 0") and pipes[-1].endswith("-> result"), text
    assert "hash table on attr 1 (payload of pipeline 0)" in pipes[1], text


@pytest.mark.parametrize("seed", range(12))
def test_driver_and_cost_match_exhaustive_enumeration(pkg, seed):
    rng = random.Random(seed)
    n = rng.randint(2, 6)
    rows = [rng.choice([1, 3, 10, 40, 100, 250]) for _ in range(n)]
    edges = []
    for c in range(1, n):
        edges.append((rng.randrange(c), c))
    # input order in the plan differs from the tree's numbering
    plan = _tree_plan(pkg, rows, edges)
    driver, cost, text = _explained(pkg, plan)
    best, want = _exhaustive(rows, edges)
    assert cost == pytest.approx(best), text
    assert driver == want, (text, rows, edges)


def _scan_guess(text):
    """(child pipeline, table it scans) of the explain's scan-guess line."""
    lines = text.strip().splitlines()
    m = re.search(r"scan guess: pipeline (\d+) on attr (\d+)", lines[-1])
    assert m, text
    k = int(m.group(1))
    t = re.match(rf"pipeline {k}: scan input \d+ \(table (\d+),", lines[1 + k])
    assert t, text
    return k, int(t.group(1))


def test_scan_guess_is_the_sparsest_build_key(pkg):
    """The drop-in path starts streaming the column of the probe whose build
    key column is sparsest over its key range: in the snowflake, the 1%
    dimension (table 1: 50 of every 5,000 keys)."""
    w = pkg.Workload("snowflake", 2, 0.01)
    assert _scan_guess(pkg.explain(w.plan_ptr()))[1] == 1


def test_scan_guess_follows_the_key_range_not_the_hit_rate(pkg):
    """A build side whose keys span a wide range is guessed, even when the
    other probe turns out more selective on the data (the device's sampling
    then decides otherwise and the guessed windows go unused; the GPU test
    test_pinned_scan_window_guess_mismatch runs this shape)."""
    plan = pkg.Plan()
    plan.new_input(pkg.table_from_rows([[i % 1000, i % 10000] for i in range(5000)], [pkg.INT32, pkg.INT32]))
    plan.new_input(pkg.table_from_rows([[k] for k in list(range(100)) + [100000]], [pkg.INT32]))
    plan.new_input(pkg.table_from_rows([[k] for k in range(10)], [pkg.INT32]))
    f = plan.new_scan_node(0, [(0, pkg.INT32), (1, pkg.INT32)])
    a = plan.new_scan_node(1, [(0, pkg.INT32)])
    b = plan.new_scan_node(2, [(0, pkg.INT32)])
    j1 = plan.new_join_node(False, f, a, 0, 0, [(0, pkg.INT32), (1, pkg.INT32)])
    plan.root = plan.new_join_node(False, j1, b, 1, 0, [(0, pkg.INT32), (1, pkg.INT32)])
    assert _scan_guess(pkg.explain(plan))[1] == 1


def _costs(pkg, plan):
    """(cheapest rooted plan's cost, cheapest reference-space plan's cost)."""
    text = pkg.explain(plan)
    first = text.splitlines()[0]
    m = re.search(r"plan space at best ([0-9.e+]+)", first)
    assert m, first
    return _explained(pkg, plan)[1], float(m.group(1))


def test_reference_space_equal_for_two_probes(pkg):
    """A fact with two dimensions: the reference's dynamic program (at most two
    probes per pipeline) finds the executor's plan: fact scanned, both hashed,
    100 + 10 + 10 + (100 + 100) x 2 = 520."""
    plan = _tree_plan(pkg, [100, 10, 10], [(0, 1), (0, 2)])
    est, ref = _costs(pkg, plan)
    assert est == pytest.approx(520) and ref == pytest.approx(520)


def test_reference_space_dearer_for_a_wide_star(pkg):
    """Three dimensions: the executor probes all three from the fact's pipeline
    (730); the reference's pipelines stop at two probes, so a partial join must
    be hashed (1,630)."""
    plan = _tree_plan(pkg, [100, 10, 10, 10], [(0, 1), (0, 2), (0, 3)])
    est, ref = _costs(pkg, plan)
    assert est == pytest.approx(730) and ref == pytest.approx(1630)


def test_reference_space_cheaper_with_payload_keys(pkg):
    """A chain fact(500) - D(10) - E(200): the reference's plans may key a hash
    table on an earlier probe's payload. Its best: E's pipeline probes D's table
    (10 + 200 + (200 + 100) = 510), the result is hashed on D's key to the fact,
    carried as D's payload, and probed by the fact (510 + 500 + (500 + 2,000) =
    3,510). The executor's rooted plans key every table on the scanned input's
    own column: D's pipeline probes E's table (2,410) and the fact probes that
    (5,410)."""
    plan = _tree_plan(pkg, [500, 10, 200], [(0, 1), (1, 2)])
    est, ref = _costs(pkg, plan)
    assert est == pytest.approx(5410) and ref == pytest.approx(3510)
    text = pkg.explain(plan)
    assert "reference plan space, cheapest: probe(input 0, hash(probe(input 2, hash(input 1))))" in text, text
    # ... and that plan is the one that runs: E's pipeline probes D's table and
    # hashes its result on D's key (D's payload); the fact probes it.
    assert "runs: the reference space's plan" in text, text
    pipes = [l for l in text.strip().splitlines() if l.startswith("pipeline")]
    assert len(pipes) == 3, text
    assert pipes[0].startswith("pipeline 0: scan input 1") and "hash table" in pipes[0], text
    assert pipes[1].startswith("pipeline 1: scan input 2") and "probe pipeline 0" in pipes[1], text
    assert "(payload of pipeline 0)" in pipes[1], text
    assert pipes[2].startswith("pipeline 2: scan input 0") and "probe pipeline 1" in pipes[2], text
    assert pipes[2].endswith("-> result"), text


def _reference_space_exhaustive(card, edges):
    """Cheapest plan of the reference's space by listing every plan: a plan of
    a set of inputs is one input (its pipeline probes nothing) or probe(R,
    hash(L)) for two connected halves L and R of the set split at one edge,
    R's top pipeline taking one probe more, at most two (QueryGraph.hpp:40);
    it costs its halves' costs + the set's cardinality + 10 x L's, a set's
    cardinality being its largest input's rows."""
    n = len(card)
    nbr = {i: set() for i in range(n)}
    for a, b in edges:
        nbr[a].add(b)
        nbr[b].add(a)

    def side(S, v, away):
        seen, stack = {v}, [v]
        while stack:
            x = stack.pop()
            for y in nbr[x]:
                if y in S and y != away and y not in seen:
                    seen.add(y)
                    stack.append(y)
        return frozenset(seen)

    memo = {}

    def plans(S):  # every (cost, probes of the top pipeline) of plans of S
        if S in memo:
            return memo[S]
        if len(S) == 1:
            out = [(card[next(iter(S))], 0)]
        else:
            out = []
            cs = max(card[i] for i in S)
            for a, b in edges:
                if a not in S or b not in S:
                    continue
                A, B = side(S, b, a), side(S, a, b)
                for L, R in ((A, B), (B, A)):
                    cl = max(card[i] for i in L)
                    for lc, _ in plans(L):
                        for rc, rp in plans(R):
                            if rp < 2:
                                out.append((lc + rc + cs + 10 * cl, rp + 1))
        memo[S] = out
        return out

    return min(c for c, _ in plans(frozenset(range(n))))


@pytest.mark.parametrize("seed", range(12))
def test_reference_space_cost_matches_exhaustive(pkg, seed):
    """The reference space's dynamic program (reference_dp_cost) against the
    listing of every plan of that space, on random join trees of 2-5 inputs
    under the row-count model."""
    rng = random.Random(700 + seed)
    n = rng.randint(2, 5)
    rows = [rng.choice([5, 20, 60, 200]) for _ in range(n)]
    edges = [(rng.randrange(c), c) for c in range(1, n)]
    plan = _tree_plan(pkg, rows, edges)
    order = [edges[0][0]] + [c for _, c in edges]  # scan k is input order[k]
    pos = {t: k for k, t in enumerate(order)}
    card = [rows[order[k]] for k in range(n)]
    sedges = [(pos[a], pos[b]) for a, b in edges]
    _, ref = _costs(pkg, plan)
    assert ref == pytest.approx(_reference_space_exhaustive(card, sedges))


def _star_plan(pkg, rows, key_type=None):
    """Input 0 joined with every other input on its column 0 = their column 0
    (one equivalence class over all of them); each input has one key column
    (INT32 unless `key_type`) and the root outputs every key."""
    key_type = pkg.INT32 if key_type is None else key_type
    plan = pkg.Plan()
    for r in rows:
        t = pkg.ColumnarTable(num_rows=r)
        t.columns.append(pkg.encode_column(key_type, [0] * r))
        plan.new_input(t)
    node = plan.new_scan_node(0, [(0, key_type)])
    for i in range(1, len(rows)):
        scan = plan.new_scan_node(i, [(0, key_type)])
        node = plan.new_join_node(True, node, scan, 0, 0, [(k, key_type) for k in range(i + 1)])
    plan.root = node
    return plan


def _restrictions(text):
    """{input: restricting pipeline's input} from the explain text."""
    scans = {}
    marks = {}
    for line in text.splitlines():
        m = re.match(r"pipeline (\d+): scan input (\d+)", line)
        if not m:
            continue
        scans[int(m.group(1))] = int(m.group(2))
        r = re.search(r"rows restricted by pipeline (\d+)'s filter", line)
        if r:
            marks[int(m.group(2))] = int(r.group(1))
    return {i: scans[p] for i, p in marks.items()}


def test_sideways_restriction_of_a_large_build(pkg):
    """A fact with two inputs joined on the same key: the build of the large
    one (300K rows) is restricted by the small one's filter (2K rows), the
    reference's Join restriction on a later scan of another input of the
    class (QueryPlan.cpp:620-624, :670-676)."""
    text = pkg.explain(_star_plan(pkg, [1_000_000, 2_000, 300_000]))
    assert _restrictions(text) == {2: 1}, text
    # three inputs of one class besides the fact: both large ones restricted
    # by the smallest
    text = pkg.explain(_star_plan(pkg, [1_000_000, 300_000, 5_000, 400_000]))
    assert _restrictions(text) == {1: 2, 3: 2}, text


@pytest.mark.parametrize("rows", [
    [1_000_000, 2_000, 200_000],     # restricted input below 2^18 rows
    [1_000_000, 140_000, 600_000],   # provider too large for a bloom filter
    [1_000_000, 80_000, 300_000],    # less than four times the provider's rows
    [1_000_000, 300_000, 300_000],   # equal inputs
])
def test_sideways_restriction_not_marked(pkg, rows):
    text = pkg.explain(_star_plan(pkg, rows))
    assert _restrictions(text) == {}, text


def test_sideways_restriction_not_on_int64_keys(pkg):
    """INT64-keyed tables carry no bloom filter to restrict with."""
    text = pkg.explain(_star_plan(pkg, [1_000_000, 2_000, 300_000], pkg.INT64))
    assert _restrictions(text) == {}, text


def _star_with_branch(pkg, rows, y_on_key=False):
    """Inputs F, A, X, Y (rows in that order), two INT32 columns each (k, y):
    F.k = A.k, F.k = X.k, and X.y = Y.y (or, with y_on_key, X.k = Y.k), so
    X's build probes Y and is keyed on the class of F.k and A.k."""
    plan = pkg.Plan()
    for r in rows:
        t = pkg.ColumnarTable(num_rows=r)
        t.columns.append(pkg.encode_column(pkg.INT32, [0] * r))
        t.columns.append(pkg.encode_column(pkg.INT32, [0] * r))
        plan.new_input(t)
    two = [(0, pkg.INT32), (1, pkg.INT32)]
    f = plan.new_scan_node(0, two)
    a = plan.new_scan_node(1, two)
    j = plan.new_join_node(True, f, a, 0, 0, [(i, pkg.INT32) for i in range(4)])
    x = plan.new_scan_node(2, two)
    j = plan.new_join_node(True, j, x, 0, 0, [(i, pkg.INT32) for i in range(6)])
    y = plan.new_scan_node(3, two)
    xa = 4 if y_on_key else 5  # X.k or X.y in the join's output
    j = plan.new_join_node(True, j, y, xa, 0 if y_on_key else 1, [(i, pkg.INT32) for i in range(8)])
    plan.root = j
    return plan


def test_sideways_restriction_of_a_build_that_probes(pkg):
    """X's build is fed by its probe of Y and keyed on the class of F.k and
    A.k: A's filter restricts it (A is not below X). No second batch is
    needed: every leaf is built before a pipeline that probes."""
    text = pkg.explain(_star_with_branch(pkg, [1_000_000, 2_000, 100_000, 5_000]))
    assert _restrictions(text) == {2: 1}, text


def test_sideways_restriction_never_by_a_table_below(pkg):
    """With X.k = Y.k, Y is both in X's key class and below X (X probes it):
    X's rows already match Y, so only A may restrict X."""
    text = pkg.explain(_star_with_branch(pkg, [1_000_000, 20_000, 100_000, 1_000], y_on_key=True))
    # Y (1,000 rows) is the smallest input of the class, A (20,000 rows)
    # restricts X's build.
    assert _restrictions(text) == {2: 1}, text


def _pipelines(text):
    """[(input, rows, [probed pipelines], restricting pipeline or None)] from
    the explain text, in pipeline order."""
    out = []
    for line in text.splitlines():
        m = re.match(r"pipeline (\d+): scan input (\d+) \(table \d+, (\d+) rows\)(.*)", line)
        if not m:
            continue
        rest = m.group(4)
        probes = [int(x) for x in re.findall(r"pipeline (\d+) on attr", rest)]
        r = re.search(r"rows restricted by pipeline (\d+)'s filter", rest)
        out.append((int(m.group(2)), int(m.group(3)), probes, int(r.group(1)) if r else None))
    return out


@pytest.mark.parametrize("seed,scale", [(1, 0.3), (2, 0.05)])
def test_sideways_restrictions_of_schema20_plans_are_sound(pkg, seed, scale):
    """Every restriction the planner marks over a batch of schema20 queries:
    the provider is a build that probes nothing, is small enough for a bloom
    filter, has at most a quarter of the restricted input's rows, is not
    itself restricted, and is not below the restricted build (it feeds no
    probe of it, directly or through other pipelines)."""
    w = pkg.Workload("schema20", seed, scale, queries=256)
    marked = 0
    try:
        for q in range(w.num_queries()):
            pipes = _pipelines(pkg.explain(w.query_ptr(q)))
            for p, (inp, rows, probes, by) in enumerate(pipes):
                if by is None:
                    continue
                marked += 1
                assert by != p and by < len(pipes) - 1, (q, p)
                _, prows, pprobes, pby = pipes[by]
                assert not pprobes and pby is None, (q, p, by)
                assert prows <= 131072 and prows * 4 <= rows, (q, p, by)
                if not probes:
                    assert rows >= 2**18, (q, p)  # a restricted leaf costs a second batch
                below, stack = set(), list(probes)
                while stack:
                    c = stack.pop()
                    if c not in below:
                        below.add(c)
                        stack.extend(pipes[c][2])
                assert by not in below, (q, p, by)
    finally:
        w.close()
    assert marked > 0
