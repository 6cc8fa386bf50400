"""The batched workload "schema20" (20 tables in a PK-FK tree, 256 random
acyclic join queries of 2-12 tables over them): generation, plans the host
planner accepts, results that match the reference engine. CPU only."""
import collections
import ctypes
import tempfile

import pytest

import oracle_lib
from test_oracle import needs_ref, run_reference, table_struct

SCALE = 0.01


@pytest.fixture(scope="module")
def schema20(pkg):
    return pkg.Workload("schema20", 3, SCALE)


def _tables(q):
    return (q.contents.num_nodes + 1) // 2


def _rows(oracle, q):
    result = oracle.execute(q)  # held while its rows are read
    return oracle.rows(result.view())


def test_schema20_shape(pkg, schema20):
    assert schema20.num_queries() == 256
    plan = schema20.plan_ptr().contents
    assert plan.num_inputs == 20
    # Query 0 is the workload's own plan.
    q0 = schema20.query_ptr(0).contents
    assert (q0.num_nodes, q0.root) == (plan.num_nodes, plan.root)
    sizes = collections.Counter(_tables(schema20.query_ptr(k)) for k in range(256))
    assert min(sizes) == 2 and max(sizes) >= 10
    assert sum(v for k, v in sizes.items() if k >= 5) >= 50
    with pytest.raises(pkg.EngineError):
        schema20.query_ptr(256)


def test_schema20_is_deterministic(pkg, oracle, schema20):
    again = pkg.Workload("schema20", 3, SCALE)
    other = pkg.Workload("schema20", 4, SCALE)
    for k in (0, 5, 33, 255):
        a = _rows(oracle, schema20.query_ptr(k))
        b = _rows(oracle, again.query_ptr(k))
        assert a.equals(b) and a.digest() == b.digest()
    rows = lambda w: [w.plan_ptr().contents.inputs[i].num_rows for i in range(20)]
    assert rows(schema20) == rows(again) and rows(schema20) != rows(other)


def test_schema20_results_are_bounded(pkg, oracle, schema20):
    # Every query's result stays within its largest table (the generator
    # drops a join that would blow up), and most results are non-empty.
    plan = schema20.plan_ptr().contents
    empty = 0
    for k in range(256):
        q = schema20.query_ptr(k).contents
        largest = max(plan.inputs[q.nodes[n].base_table_id].num_rows
                      for n in range(q.num_nodes) if q.nodes[n].kind == pkg.NODE_SCAN)
        n = len(_rows(oracle, schema20.query_ptr(k)))
        assert n <= largest, k
        empty += n == 0
    assert empty < 32


def test_schema20_plans_explain(pkg, schema20):
    # The host planner takes every query: one pipeline per scanned table.
    for k in range(0, 256, 7):
        q = schema20.query_ptr(k)
        text = pkg.explain(q)
        assert text.startswith("driver: input")
        assert sum(1 for line in text.splitlines() if line.startswith("pipeline ")) == _tables(q)


@needs_ref
@pytest.mark.parametrize("k", [0, 1, 2, 5, 10, 25, 27, 33, 52])
def test_schema20_oracle_matches_reference_engine(pkg, oracle, schema20, k):
    q = schema20.query_ptr(k)
    with tempfile.TemporaryDirectory() as tmp:
        ref = run_reference(pkg, q, tmp)
    ref_struct, keep = table_struct(pkg, ref)
    ora = oracle.execute(q)
    oracle_lib.assert_same_rows(oracle, ctypes.byref(ref_struct), ora.view(), f"schema20 query {k}")


@needs_ref
@pytest.mark.parametrize("seed", [4, 5])
def test_schema20_widest_queries_match_reference_engine(pkg, oracle, seed):
    # Other schemas: the four queries with the most tables, compared with the
    # reference engine.
    w = pkg.Workload("schema20", seed, SCALE)
    widest = sorted(range(256), key=lambda k: (-_tables(w.query_ptr(k)), k))[:4]
    assert _tables(w.query_ptr(widest[-1])) >= 6
    for k in widest:
        q = w.query_ptr(k)
        with tempfile.TemporaryDirectory() as tmp:
            ref = run_reference(pkg, q, tmp)
        ref_struct, keep = table_struct(pkg, ref)
        ora = oracle.execute(q)
        oracle_lib.assert_same_rows(oracle, ctypes.byref(ref_struct), ora.view(), f"schema20 seed {seed} query {k}")


def test_schema20w_has_int64_keys_and_the_same_results(pkg, oracle, schema20):
    """schema20w: the same tables with INT64 keys on every other table (low
    halves kept, high halves varying). Each query joins the same rows, so the
    oracle's row count matches schema20's; the reference reads join keys as
    32 bits, so these are checked against the oracle alone."""
    w = pkg.Workload("schema20w", 3, SCALE)
    plan = w.plan_ptr().contents
    types = [plan.inputs[t].columns[0].type for t in range(plan.num_inputs)]
    assert types.count(pkg.INT64) == 10 and types.count(pkg.INT32) == 10
    for k in range(0, 256, 16):
        a = len(_rows(oracle, w.query_ptr(k)))
        b = len(_rows(oracle, schema20.query_ptr(k)))
        assert a == b, f"query {k}: {a} != {b}"


def test_schema20_more_queries_extends_the_batch(pkg):
    """Query k depends only on (seed, scale, k): a workload of 300 queries
    starts with the default 256."""
    a = pkg.Workload("schema20", 3, SCALE)
    b = pkg.Workload("schema20", 3, SCALE, queries=300)
    assert b.num_queries() == 300
    for k in (0, 17, 255):
        qa, qb = a.query_ptr(k).contents, b.query_ptr(k).contents
        assert (qa.num_nodes, qa.root) == (qb.num_nodes, qb.root)
        assert [qa.nodes[i].base_table_id for i in range(qa.num_nodes)] == \
               [qb.nodes[i].base_table_id for i in range(qb.num_nodes)]
    assert a.base_rows(0) >= a.plan_ptr().contents.inputs[0].num_rows
