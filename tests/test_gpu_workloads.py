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
