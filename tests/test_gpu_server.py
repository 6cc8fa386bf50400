"""Serving: queries of uneven sizes submitted together to a server with
several workers (contexts on one device) give, each, exactly the rows the
oracle gives for that query alone."""
import ctypes

import pytest

import oracle_lib

pytestmark = pytest.mark.gpu


def test_mixed_queries_same_alone_and_in_the_mix(pkg, oracle):
    small = pkg.Workload("snowflake", 11, 0.02)
    large = pkg.Workload("snowflake", 12, 0.1)
    plans = [(small, small.variant_ptr(1)), (small, small.variant_ptr(2)), (large, large.plan_ptr()),
             (small, small.variant_ptr(3)), (large, large.variant_ptr(1))]
    want = [oracle.execute(p) for _, p in plans]
    with pkg.Server(0, workers=4, scratch_cap_bytes=0) as srv:
        res = {}
        for w in (small, large):
            plan = w.plan_ptr().contents
            res[id(w)] = [srv.upload(plan.inputs[i]) for i in range(plan.num_inputs)]
        try:
            # Alone, one at a time.
            for k, (w, p) in enumerate(plans):
                r, _ = srv.wait(srv.submit(p, res[id(w)][:p.contents.num_inputs], pkg.RESULT_HOST))
                got, keep = r.table_struct()
                oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want[k].view(), f"alone {k}")
                r.free()
            # In the mix: 30 queries in flight at once, every plan several times.
            tickets = []
            for i in range(30):
                k = (i * 7) % len(plans)
                w, p = plans[k]
                tickets.append((k, srv.submit(p, res[id(w)][:p.contents.num_inputs], pkg.RESULT_HOST)))
            for k, t in tickets:
                r, ms = srv.wait(t)
                assert ms > 0
                got, keep = r.table_struct()
                oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want[k].view(), f"mix {k}")
                r.free()
        finally:
            for rs in res.values():
                for x in rs:
                    x.free()


def test_scratch_cap_serialises_without_blocking(pkg, oracle):
    """A cap below one query's scratch admits one query at a time."""
    w = pkg.Workload("snowflake", 13, 0.02)
    p = w.variant_ptr(2)
    want = oracle.execute(p)
    with pkg.Server(0, workers=3, scratch_cap_bytes=1) as srv:
        plan = w.plan_ptr().contents
        res = [srv.upload(plan.inputs[i]) for i in range(plan.num_inputs)]
        try:
            tickets = [srv.submit(p, res[:3], pkg.RESULT_HOST) for _ in range(6)]
            for t in tickets:
                r, _ = srv.wait(t)
                got, keep = r.table_struct()
                oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(), "capped")
                r.free()
        finally:
            for x in res:
                x.free()


def test_orderings_and_load_generator_give_the_oracle_rows(pkg, oracle):
    """The schema20 queries under every ordering mode (row counts, join
    samples, the learned estimator) return the oracle's rows, alone and
    through the C++ load generator (closed loop and Poisson arrivals, summed
    rows equal to the oracle's sum), with graph replay off and on."""
    import numpy as np

    w = pkg.Workload("schema20", 3, 0.01, queries=300)
    queries = list(range(0, 64, 2))
    def oracle_rows(k):
        result = oracle.execute(w.query_ptr(k))  # held while its rows are read
        return len(oracle.rows(result.view()))

    wants = {k: oracle_rows(k) for k in queries}
    est = pkg.Estimator(0, seed=1)
    # A quickly trained estimator: its estimates only steer the order.
    with pkg.Context(0) as ctx:
        plan = w.plan_ptr().contents
        res = [ctx.upload(plan.inputs[t]) for t in range(plan.num_inputs)]
        corpus = pkg.subplan_corpus(ctx, w, res, range(256, 300), max_per_query=32)
        est.train(corpus["features"], np.log2(corpus["card"] + 1.0), epochs=5, batch=128)
        for mode in (pkg.ORDER_ROWS, pkg.ORDER_SAMPLING, pkg.ORDER_LEARNED):
            ctx.set_ordering(mode, est if mode == pkg.ORDER_LEARNED else None)
            for k in queries[:12]:
                q = w.query_ptr(k)
                want = oracle.execute(q)
                with ctx.execute_resident(q, res) as r:
                    got, keep = r.table_struct()
                    oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(), f"query {k} ordering {mode}")
            assert ctx.scratch_estimate(w.query_ptr(queries[0]), res) > 0
        for x in res:
            x.free()
    plan_ptrs = [w.query_ptr(k) for k in queries]
    seq = np.array([i % len(queries) for i in range(3 * len(queries))], dtype=np.uint32)
    want_rows = sum(wants[queries[i]] for i in seq)
    for workers, graphs, mode in ((1, False, pkg.ORDER_SAMPLING), (4, True, pkg.ORDER_LEARNED)):
        with pkg.Server(0, workers=workers, scratch_cap_bytes=120 << 30) as srv:
            plan = w.plan_ptr().contents
            tabs = [srv.upload(plan.inputs[t]) for t in range(plan.num_inputs)]
            try:
                srv.set_ordering(mode, est if mode == pkg.ORDER_LEARNED else None)
                srv.set_graphs(graphs)
                lat, el, rows = srv.run_load(plan_ptrs, tabs, seq, 0.0, 2 * workers)
                assert rows == want_rows and el > 0 and (lat > 0).all()
                lat, el, rows = srv.run_load(plan_ptrs, tabs, seq, 500.0, 0, seed=3)
                assert rows == want_rows and el >= 0.9 * len(seq) / 500.0
            finally:
                for x in tabs:
                    x.free()
    est.close()
