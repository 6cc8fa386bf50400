"""bj_join_count_static: the join count that allocates no memory.

Some callers of this library cannot call cudaMalloc -- their device memory is
owned by another allocator (a framework's caching pool, or a budget fixed at
start-up), or they run where cudaMalloc's implicit device synchronisation is
not allowed. bj_join_count_static serves them: it counts the rows of a
two-table INT32 equi-join using only the caller's buffers and a fixed 4 MiB
scratch array compiled into the library.

The test calls it through the C ABI twice in a row on the same inputs (the
scratch keeps the previous call's contents, so the second call shows that
each call starts clean) and compares each count, exactly, with the row count
of bj_execute on the same join. The input buffers here come from torch; the
entry point itself allocates nothing.
"""
import random

import pytest

pytestmark = pytest.mark.gpu

CASES = [
    # build rows, probe rows, key domain, NULL probability
    (5000, 40000, 3000, 0.1),
    (200000, 300000, 150000, 0.0),
    (1, 10, 5, 0.5),
    (262144, 5000, 1 << 30, 0.0),  # the scratch's full capacity
]


def make_tables(pkg, seed, nb, npr, dom, null_p):
    rng = random.Random(seed)
    b = [[None if rng.random() < null_p else rng.randrange(dom)] for _ in range(nb)]
    p = [[None if rng.random() < null_p else rng.randrange(dom)] for _ in range(npr)]
    return pkg.table_from_rows(b, [pkg.INT32]), pkg.table_from_rows(p, [pkg.INT32])


def execute_count(pkg, ctx, tb, tp):
    plan = pkg.Plan()
    plan.new_input(tb)
    plan.new_input(tp)
    plan.new_scan_node(0, [(0, pkg.INT32)])
    plan.new_scan_node(1, [(0, pkg.INT32)])
    plan.new_join_node(True, 0, 1, 0, 0, [(0, pkg.INT32)])
    plan.root = 2
    with ctx.execute_raw(pkg.CPlan(plan)) as r:
        return r.num_rows


def test_join_count_static_matches_execute(pkg):
    import torch

    ctx = pkg.Context(0)
    try:
        for seed, (nb, npr, dom, null_p) in enumerate(CASES):
            tb, tp = make_tables(pkg, 77 + seed, nb, npr, dom, null_p)
            want = execute_count(pkg, ctx, tb, tp)
            db = torch.frombuffer(bytearray(tb.columns[0].data), dtype=torch.uint8).to("cuda")
            dp = torch.frombuffer(bytearray(tp.columns[0].data), dtype=torch.uint8).to("cuda")
            out = torch.full((1,), -1, dtype=torch.int64, device="cuda")
            torch.cuda.synchronize()
            for call in range(2):
                st = pkg.lib().bj_join_count_static(db.data_ptr(), tb.columns[0].num_pages, tb.num_rows,
                                                    dp.data_ptr(), tp.columns[0].num_pages, out.data_ptr(), None)
                assert st == 0, f"case {seed} call {call}: status {st}"
                torch.cuda.synchronize()
                assert int(out.item()) == want, f"case {seed} call {call}: {int(out.item())} != {want}"
    finally:
        ctx.close()


def test_join_count_static_rejects_oversized_build(pkg):
    import torch

    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    page = torch.zeros(8192, dtype=torch.uint8, device="cuda")
    st = pkg.lib().bj_join_count_static(page.data_ptr(), 1, 262145, page.data_ptr(), 1, out.data_ptr(), None)
    assert st == 1  # BJ_ERR_INVALID: beyond the fixed scratch
