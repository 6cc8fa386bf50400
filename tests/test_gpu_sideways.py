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
from plangen import star_plan

pytestmark = pytest.mark.gpu


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
    cp = star_plan(pkg, seed, fact_rows, small_rows, large_rows, small_dom, edges)
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
    cp = star_plan(pkg, 11, 800_000, 5_000, 350_000, 200_000, True)
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


def _branch_plan(pkg, seed):
    """F (600K rows) joined with A (2K) and X (100K) on one key k, X also
    joined with Y (5K) on y: X's build probes Y and is restricted by A's
    filter (A is not below X)."""
    rng = np.random.default_rng(seed)
    dom, ydom = 200_000, 5_000

    def table(rows, kdom, ydom_):
        t = pkg.ColumnarTable(num_rows=rows)
        k = [int(v) for v in rng.integers(0, kdom, size=rows)]
        for i in rng.choice(rows, size=max(1, rows // 50), replace=False):
            k[int(i)] = None
        t.columns.append(pkg.encode_column(pkg.INT32, k))
        t.columns.append(pkg.encode_column(pkg.INT32, [int(v) for v in rng.integers(0, ydom_, size=rows)]))
        return t

    plan = pkg.Plan()
    for rows in (600_000, 2_000, 100_000, 5_000):
        plan.new_input(table(rows, dom, ydom))
    two = [(0, pkg.INT32), (1, pkg.INT32)]
    j = plan.new_join_node(True, plan.new_scan_node(0, two), plan.new_scan_node(1, two), 0, 0,
                           [(i, pkg.INT32) for i in range(4)])
    j = plan.new_join_node(True, j, plan.new_scan_node(2, two), 0, 0, [(i, pkg.INT32) for i in range(6)])
    j = plan.new_join_node(True, j, plan.new_scan_node(3, two), 5, 1, [(1, pkg.INT32), (3, pkg.INT32), (5, pkg.INT32), (6, pkg.INT32)])
    plan.root = j
    return pkg.CPlan(plan)


@pytest.mark.parametrize("seed", [31, 32])
def test_restricted_build_that_probes_equals_oracle(pkg, oracle, seed):
    """A build fed by a probe, restricted by a leaf's filter in its key
    class: the same rows with the restriction on and off."""
    cp = _branch_plan(pkg, seed)
    text = pkg.explain(cp)
    assert "probe pipeline" in text and "rows restricted by pipeline" in text, text
    want = oracle.execute(cp.ref())
    for sideways in (True, False):
        with _context(pkg, sideways) as c:
            with c.execute_raw(cp) as r:
                got, keep = r.table_struct()
                oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(),
                                            f"branch seed {seed} sideways={sideways}")


def test_schema20_batch_with_restricted_payload_keyed_builds(pkg, oracle):
    """schema20 seed 2 at x0.05: 120 of its 256 queries run builds keyed on a
    probed table's payload and restricted by a leaf's filter (the reference's
    plan space). Only the restricted queries, over resident tables: recorded,
    captured and replayed, each equal to the oracle."""
    w = pkg.Workload("schema20", 2, 0.05)
    ks = [k for k in range(256) if "rows restricted by pipeline" in pkg.explain(w.query_ptr(k))]
    assert len(ks) >= 100
    plan = w.plan_ptr().contents
    wants = {k: oracle.execute(w.query_ptr(k)) for k in ks}
    with _context(pkg, True) as c:
        res = [c.upload(plan.inputs[i]) for i in range(plan.num_inputs)]
        try:
            for run in ("record", "capture", "replay"):
                for k in ks:
                    with c.execute_resident(w.query_ptr(k), res) as r:
                        got, keep = r.table_struct()
                        oracle_lib.assert_same_rows(oracle, ctypes.byref(got), wants[k].view(),
                                                    f"schema20 seed 2 query {k} ({run})")
        finally:
            for x in res:
                x.free()
