"""The autotuner (bj_context_autotune): every combination of the tunable
build and scan parameters is run (the engine checks that all return the same
row count), the fastest is kept for the plan's shape class, and queries of
that class then return the oracle's rows -- graph replays included."""
import ctypes

import pytest

import oracle_lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,seed,scale", [("snowflake", 21, 0.05), ("join2", 22, 0.05)])
def test_autotune_then_oracle_rows(pkg, oracle, name, seed, scale):
    w = pkg.Workload(name, seed, scale)
    plan = w.plan_ptr()
    want = oracle.execute(plan)
    with pkg.Context(0) as ctx:
        inputs = plan.contents
        res = [ctx.upload(inputs.inputs[i]) for i in range(inputs.num_inputs)]
        try:
            report = ctx.autotune(plan, res, repeats=2)
            lines = report.strip().splitlines()
            assert lines[0].startswith("shape class") and lines[-1].startswith("chosen:"), report
            assert sum(1 for l in lines if " ms" in l and not l.startswith("chosen")) == 12, report
            for run in range(3):  # record, capture, replay
                with ctx.execute_resident(plan, res) as r:
                    got, keep = r.table_struct()
                    oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(), f"{name} tuned run {run}")
        finally:
            for x in res:
                x.free()
