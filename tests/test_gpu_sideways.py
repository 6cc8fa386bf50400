"""Sideways restrictions between leaf builds, on the GPU, against the oracle.

A fact joined with two inputs on one key: the large input's build drops the
rows whose key the small input's bloom filter cannot hold (the reference's
Join restriction on a later scan of another input of the key class,
engine/query/QueryPlan.cpp:620-624, :670-676). Results must equal the
oracle's with the restriction on and off, on the host path and on resident
tables (first run and CUDA-graph replay)."""
import contextlib
import ctypes
import os

import numpy as np
import pytest

import oracle_lib

pytestmark = pytest.mark.gpu

INT32_EDGES = [-1, -2**31, 2**31 - 1, 0, 1]


def _keys(rng, n, lo, hi, null_p, edges=False):
    k = rng.integers(lo, hi, size=n, dtype=np.int64)
    out = [int(x) for x in k]
    if edges:
        for i in rng.choice(n, size=min(n, 16), replace=False):
            out[int(i)] = INT32_EDGES[int(i) % len(INT32_EDGES)]
    if null_p:
        for i in np.nonzero(rng.random(n) < null_p)[0]:
            out[int(i)] = None
    return out


def _star(pkg, seed, fact_rows, small_rows, large_rows, small_dom, edges=False):
    """Fact (key, INT64 payload) joined on its key with a small input (key,
    INT32 payload) and a large input (key, VARCHAR payload); the root outputs
    the fact's payload, the small input's payload, the large input's key and
    payload. Keys of the fact and the large input are drawn from [0, 200000),
    the small input's from [0, small_dom)."""
    rng = np.random.default_rng(seed)
    dom = 200_000
    fact = pkg.ColumnarTable(num_rows=fact_rows)
    fact.columns.append(pkg.encode_column(pkg.INT32, _keys(rng, fact_rows, 0, dom, 0.05, edges)))
    fact.columns.append(pkg.encode_column(pkg.INT64, [int(x) for x in rng.integers(-2**40, 2**40, size=fact_rows)]))
    small = pkg.ColumnarTable(num_rows=small_rows)
    small.columns.append(pkg.encode_column(pkg.INT32, _keys(rng, small_rows, 0, small_dom, 0.0, edges)))
    small.columns.append(pkg.encode_column(pkg.INT32, [int(x) for x in rng.integers(0, 1000, size=small_rows)]))
    large = pkg.ColumnarTable(num_rows=large_rows)
    large.columns.append(pkg.encode_column(pkg.INT32, _keys(rng, large_rows, 0, dom, 0.03, edges)))
    large.columns.append(pkg.encode_column(pkg.VARCHAR, [f"v{int(x)}" for x in rng.integers(0, 10**6, size=large_rows)]))
    plan = pkg.Plan()
    for t in (fact, small, large):
        plan.new_input(t)
    f = plan.new_scan_node(0, [(0, pkg.INT32), (1, pkg.INT64)])
    s = plan.new_scan_node(1, [(0, pkg.INT32), (1, pkg.INT32)])
    j1 = plan.new_join_node(True, f, s, 0, 0, [(0, pkg.INT32), (1, pkg.INT64), (2, pkg.INT32), (3, pkg.INT32)])
    l = plan.new_scan_node(2, [(0, pkg.INT32), (1, pkg.VARCHAR)])
    j2 = plan.new_join_node(True, j1, l, 0, 0, [(1, pkg.INT64), (3, pkg.INT32), (4, pkg.INT32), (5, pkg.VARCHAR)])
    plan.root = j2
    return pkg.CPlan(plan)


@contextlib.contextmanager
def _context(pkg, sideways):
    old = os.environ.get("B200JOIN_SIDEWAYS")
    os.environ["B200JOIN_SIDEWAYS"] = "1" if sideways else "0"
    try:
        c = pkg.Context(0)
    finally:
        if old is None:
            del os.environ["B200JOIN_SIDEWAYS"]
        else:
            os.environ["B200JOIN_SIDEWAYS"] = old
    try:
        yield c
    finally:
        c.close()


CASES = [
    # (seed, fact, small, large, small key domain, edge keys)
    (1, 1_000_000, 2_000, 300_000, 200_000, False),   # the small input holds ~1% of the keys
    (2, 600_000, 20_000, 400_000, 200_000, True),     # ~10%, keys at the INT32 edges
    (3, 500_000, 60_000, 300_000, 2_000, False),      # the small input holds few keys, many repeated
    (4, 400_000, 50_000, 300_000, 200_000, False),    # restriction that removes ~78%
]


@pytest.mark.parametrize("case", CASES, ids=[f"seed{c[0]}" for c in CASES])
def test_restricted_build_equals_oracle(pkg, oracle, case):
    seed, fact_rows, small_rows, large_rows, small_dom, edges = case
    cp = _star(pkg, seed, fact_rows, small_rows, large_rows, small_dom, edges)
    text = pkg.explain(cp)
    assert "rows restricted by pipeline" in text, text
    want = oracle.execute(cp.ref())
    launches = {}
    for sideways in (True, False):
        with _context(pkg, sideways) as c:
            with c.execute_raw(cp) as r:
                launches[sideways] = r.stats().kernel_launches
                got, keep = r.table_struct()
                oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(), f"seed {seed} sideways={sideways}")
    # The restricted build runs as a second batch of leaf builds.
    assert launches[True] > launches[False], launches


def test_restricted_build_resident_and_replayed(pkg, oracle):
    """Resident tables: the first run records the query, the second replays
    it as a CUDA graph; both equal the oracle."""
    cp = _star(pkg, 11, 800_000, 5_000, 350_000, 200_000, True)
    plan = cp.struct
    want = oracle.execute(cp.ref())
    with _context(pkg, True) as c:
        res = [c.upload(plan.inputs[i]) for i in range(plan.num_inputs)]
        try:
            for run in range(3):
                with c.execute_resident(cp, res) as r:
                    got, keep = r.table_struct()
                    oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(), f"resident run {run}")
        finally:
            for x in res:
                x.free()
