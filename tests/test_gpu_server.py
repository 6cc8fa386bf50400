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
