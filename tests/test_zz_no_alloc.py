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
the CPU oracle gives for the same join and with bj_execute's. Bad input --
a malformed page, or build pages holding more values than the build_rows
passed -- must turn the count into ~0ull. The input buffers here come from
torch; the entry point itself allocates nothing.
"""
import random

import pytest

pytestmark = pytest.mark.gpu

ERR_COUNT = (1 << 64) - 1  # ~0ull: what the entry point writes for bad input

CASES = [
    # build rows, probe rows, key domain, NULL probability, share of keys set to -1
    (5000, 40000, 3000, 0.1, 0.0),
    (200000, 300000, 150000, 0.0, 0.0),
    (1, 10, 5, 0.5, 0.0),
    (262144, 5000, 1 << 30, 0.0, 0.0),  # the scratch's full capacity
    (3000, 20000, 2000, 0.05, 0.02),    # key -1 (0xFFFFFFFF) on both sides: not the empty-slot pattern
    (0, 1000, 100, 0.0, 0.0),           # empty build side
]


def draw(rng, dom, null_p, neg_p):
    if rng.random() < null_p:
        return None
    if rng.random() < neg_p:
        return -1
    return rng.randrange(dom)


def make_tables(pkg, seed, nb, npr, dom, null_p, neg_p):
    rng = random.Random(seed)
    b = [[draw(rng, dom, null_p, neg_p)] for _ in range(nb)]
    p = [[draw(rng, dom, null_p, neg_p)] for _ in range(npr)]
    return pkg.table_from_rows(b, [pkg.INT32]), pkg.table_from_rows(p, [pkg.INT32])


def join_plan(pkg, tb, tp):
    plan = pkg.Plan()
    plan.new_input(tb)
    plan.new_input(tp)
    plan.new_scan_node(0, [(0, pkg.INT32)])
    plan.new_scan_node(1, [(0, pkg.INT32)])
    plan.new_join_node(True, 0, 1, 0, 0, [(0, pkg.INT32)])
    plan.root = 2
    return pkg.CPlan(plan)


def device_pages(tbl):
    import torch

    data = tbl.columns[0].data if tbl.columns else b""
    buf = torch.frombuffer(bytearray(data or b"\0" * 8192), dtype=torch.uint8).to("cuda")
    return buf, (tbl.columns[0].num_pages if tbl.columns else 0)


def count_static(pkg, db, nbp, build_rows, dp, npp, out):
    import torch

    st = pkg.lib().bj_join_count_static(db.data_ptr(), nbp, build_rows, dp.data_ptr(), npp, out.data_ptr(), None)
    torch.cuda.synchronize()
    return st, int(out.item()) & ERR_COUNT


def test_join_count_static_matches_oracle(pkg, oracle):
    import torch

    ctx = pkg.Context(0)
    try:
        for seed, (nb, npr, dom, null_p, neg_p) in enumerate(CASES):
            tb, tp = make_tables(pkg, 77 + seed, nb, npr, dom, null_p, neg_p)
            cplan = join_plan(pkg, tb, tp)
            result = oracle.execute(cplan.ref())  # held while its rows are read
            want_n = len(oracle.rows(result.view()))
            with ctx.execute_raw(cplan.ref()) as r:
                assert r.num_rows == want_n, f"case {seed}: bj_execute {r.num_rows} != oracle {want_n}"
            db, nbp = device_pages(tb)
            dp, npp = device_pages(tp)
            out = torch.full((1,), -1, dtype=torch.int64, device="cuda")
            torch.cuda.synchronize()
            for call in range(2):
                st, got = count_static(pkg, db, nbp, tb.num_rows, dp, npp, out)
                assert st == 0, f"case {seed} call {call}: status {st}"
                assert got == want_n, f"case {seed} call {call}: {got} != oracle {want_n}"
    finally:
        ctx.close()


def test_join_count_static_rejects_oversized_build(pkg):
    import torch

    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    page = torch.zeros(8192, dtype=torch.uint8, device="cuda")
    st = pkg.lib().bj_join_count_static(page.data_ptr(), 1, 262145, page.data_ptr(), 1, out.data_ptr(), None)
    assert st == 1  # BJ_ERR_INVALID: beyond the fixed scratch


def test_join_count_static_flags_bad_input(pkg, oracle):
    import torch

    tb, tp = make_tables(pkg, 5, 4000, 9000, 3000, 0.0, 0.0)
    cplan = join_plan(pkg, tb, tp)  # its page buffers live as long as it does
    result = oracle.execute(cplan.ref())
    want_n = len(oracle.rows(result.view()))
    db, nbp = device_pages(tb)
    dp, npp = device_pages(tp)
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    # build_rows below the build pages' non-null values: flagged, not a short count
    st, got = count_static(pkg, db, nbp, tb.num_rows - 1, dp, npp, out)
    assert st == 0 and got == ERR_COUNT
    # a probe page whose header says more non-null values than rows
    bad = dp.clone()
    bad[npp * 8192 - 8192 + 2] = 0xff
    bad[npp * 8192 - 8192 + 3] = 0xff
    st, got = count_static(pkg, db, nbp, tb.num_rows, bad, npp, out)
    assert st == 0 and got == ERR_COUNT
    # the next good call counts again from a clean scratch
    st, got = count_static(pkg, db, nbp, tb.num_rows, dp, npp, out)
    assert st == 0 and got == want_n
