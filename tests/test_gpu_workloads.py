"""The batched workload "schema20" on the engine: every query of the batch
(2-12 tables over 20 shared tables) from host pages, and again over the tables
made resident in HBM once, compared exactly with the oracle."""
import ctypes

import pytest

import oracle_lib

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def schema20(pkg):
    return pkg.Workload("schema20", 3, 0.01)


def test_schema20_queries_from_host_pages(pkg, ctx, oracle, schema20):
    for k in range(0, 256, 4):
        q = schema20.query_ptr(k)
        with ctx.execute_raw(q) as r:
            got, keep = r.table_struct()
            want = oracle.execute(q)
            oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(), f"schema20 query {k}")


def test_schema20_batch_resident(pkg, ctx, oracle, schema20):
    """The batch three times over resident tables: each query's first run
    records, its second is captured into a CUDA graph, its third replays it
    (the engine keeps the graphs of all 256 queries)."""
    plan = schema20.plan_ptr().contents
    res = [ctx.upload(plan.inputs[i]) for i in range(plan.num_inputs)]
    wants = [oracle.execute(schema20.query_ptr(k)) for k in range(256)]
    try:
        for run in ("record", "capture", "replay"):
            nonempty = 0
            for k in range(256):
                q = schema20.query_ptr(k)
                with ctx.execute_resident(q, res, flags=pkg.RESULT_HOST | pkg.RESULT_ASYNC) as r:
                    r.wait()
                    got, keep = r.table_struct()
                    nonempty += oracle_lib.assert_same_rows(oracle, ctypes.byref(got), wants[k].view(),
                                                            f"schema20 resident query {k} ({run})") > 0
            assert nonempty > 200
    finally:
        for x in res:
            x.free()


def test_schema20w_int64_keys(pkg, ctx, oracle):
    """schema20w (INT64 join keys on every other table, low halves shared
    across high halves): every fourth query from host pages and all 256 over
    resident tables (recorded, then captured), each equal to the oracle."""
    w = pkg.Workload("schema20w", 3, 0.01)
    for k in range(0, 256, 4):
        q = w.query_ptr(k)
        with ctx.execute_raw(q) as r:
            got, keep = r.table_struct()
            want = oracle.execute(q)
            oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(), f"schema20w query {k}")
    plan = w.plan_ptr().contents
    res = [ctx.upload(plan.inputs[i]) for i in range(plan.num_inputs)]
    try:
        for run in ("record", "capture"):
            for k in range(256):
                q = w.query_ptr(k)
                want = oracle.execute(q)
                with ctx.execute_resident(q, res) as r:
                    got, keep = r.table_struct()
                    oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(),
                                                f"schema20w resident query {k} ({run})")
    finally:
        for x in res:
            x.free()


def _digest(oracle, table_ptr):
    return oracle.rows(table_ptr).digest()


@pytest.mark.parametrize("name", ["schema20", "schema20w"])
def test_schema20_full_scale_every_query(pkg, ctx, oracle, name):
    """The batched workload at its stated size (scale 1.0: tables of 10K-40M
    rows before their filters, 7.5M rows after): all 256 queries over resident
    tables, each result's row multiset equal to the oracle's (compared by row
    count and order-independent digests of the rows; the oracle runs on host
    threads while the GPU works). schema20w has INT64 keys on half the
    tables."""
    from concurrent.futures import ThreadPoolExecutor
    import os

    w = pkg.Workload(name, 3, 1.0)
    plan = w.plan_ptr().contents
    res = [ctx.upload(plan.inputs[i]) for i in range(plan.num_inputs)]

    def oracle_digest(k):
        r = oracle.execute(w.query_ptr(k))  # ctypes releases the GIL: threads run in parallel
        return _digest(oracle, r.view())

    try:
        with ThreadPoolExecutor(max_workers=max(2, min(16, os.cpu_count() or 2))) as pool:
            wants = [pool.submit(oracle_digest, k) for k in range(256)]
            rows = 0
            for k in range(256):
                with ctx.execute_resident(w.query_ptr(k), res) as r:
                    got, keep = r.table_struct()
                    msg = oracle.validate(ctypes.byref(got))
                    assert msg is None, f"{name} query {k}: {msg}"
                    d = _digest(oracle, ctypes.byref(got))
                want = wants[k].result()
                assert d == want, f"{name} query {k}: rows/digest {d} != oracle {want}"
                rows += d[0]
        assert rows > 1_000_000
    finally:
        for x in res:
            x.free()
