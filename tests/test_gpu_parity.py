"""Parity of the CUDA engine with the oracle, through the C ABI.

Bar: the result row multiset equals the oracle's exactly (integer, string and
index work is bit-exact), and every result page obeys the page format.
"""
import ctypes

import pytest

import oracle_lib
import plangen
from golden.make_golden import canon, to_plan

pytestmark = pytest.mark.gpu


def check_against_oracle(pkg, ctx, oracle, plan_ref, label):
    with ctx.execute_raw(plan_ref) as r:
        st = r.stats()
        assert st.kernel_launches > 0 or r.num_rows == 0
        got, keep = r.table_struct()
        want = oracle.execute(plan_ref.ref() if hasattr(plan_ref, "ref") else plan_ref)
        return oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(), label)


def test_golden_cases(pkg, ctx, golden):
    """The reference's API cases (tests/unit_tests.cpp:19-663) through bj_execute."""
    for case in golden:
        out = ctx.execute(to_plan(case, pkg))
        assert [c.type for c in out.columns] == case["expected_types"], case["name"]
        assert out.num_rows == len(case["expected"]), case["name"]
        assert canon(pkg.rows_of(out)) == canon(case["expected"]), case["name"]


@pytest.mark.parametrize("seed", range(60))
def test_random_plans(pkg, ctx, oracle, seed):
    tables, nodes, root = plangen.random_case(1000 + seed, max_rows=3000)
    cp = pkg.CPlan(plangen.to_plan(pkg, tables, nodes, root))
    check_against_oracle(pkg, ctx, oracle, cp, f"seed {1000 + seed}")


@pytest.mark.parametrize("seed", range(24))
def test_random_plans_int64_keys(pkg, ctx, oracle, seed):
    """INT64 join keys (no reference counterpart: the reference reads join
    keys as 32 bits) whose low halves collide across high halves, mixed with
    INT32 joins in one plan; checked against the oracle's 64-bit comparison."""
    tables, nodes, root = plangen.random_case(9000 + seed, max_rows=3000, int64_keys=True)
    cp = pkg.CPlan(plangen.to_plan(pkg, tables, nodes, root))
    check_against_oracle(pkg, ctx, oracle, cp, f"int64 seed {9000 + seed}")


@pytest.mark.parametrize("seed", range(16))
def test_random_plans_signed_int32_keys(pkg, ctx, oracle, seed):
    """INT32 join keys around zero and at the type's edges (-1 = 0xFFFFFFFF,
    INT32_MIN, INT32_MAX): hashing, bloom bits, bucket first keys and the
    key statistics take every bit pattern."""
    tables, nodes, root = plangen.random_case(7000 + seed, max_rows=3000 if seed % 4 else 30000,
                                              signed_keys=True)
    cp = pkg.CPlan(plangen.to_plan(pkg, tables, nodes, root))
    check_against_oracle(pkg, ctx, oracle, cp, f"signed seed {7000 + seed}")


@pytest.mark.parametrize("seed", range(6))
def test_signed_int32_keys_resident_with_join_samples(pkg, oracle, seed):
    """The same keys over resident tables with join orders from join samples:
    the key statistics' key -> count maps (empty slots marked by the all-ones
    64-bit pattern) take the keys -1, INT32_MIN and INT32_MAX."""
    tables, nodes, root = plangen.random_case(7100 + seed, min_tables=2, max_rows=3000, signed_keys=True)
    cp = pkg.CPlan(plangen.to_plan(pkg, tables, nodes, root))
    plan = cp.struct
    with pkg.Context(0) as c:
        c.set_ordering(pkg.ORDER_SAMPLING)
        res = [c.upload(plan.inputs[i]) for i in range(plan.num_inputs)]
        try:
            with c.execute_resident(cp, res) as r:
                got, keep = r.table_struct()
                want = oracle.execute(cp.ref())
                oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(), f"resident signed {7100 + seed}")
        finally:
            for x in res:
                x.free()


@pytest.mark.parametrize("seed", range(4))
def test_random_plans_int64_keys_wide_tables(pkg, ctx, oracle, seed):
    tables, nodes, root = plangen.random_case(9500 + seed, max_tables=3, max_rows=40000, int64_keys=True)
    cp = pkg.CPlan(plangen.to_plan(pkg, tables, nodes, root))
    check_against_oracle(pkg, ctx, oracle, cp, f"int64 seed {9500 + seed}")


@pytest.mark.parametrize("seed", range(10))
def test_random_plans_wide_tables(pkg, ctx, oracle, seed):
    """Larger inputs: columns of many pages, long chains of duplicates."""
    tables, nodes, root = plangen.random_case(5000 + seed, max_tables=3, max_rows=40000)
    cp = pkg.CPlan(plangen.to_plan(pkg, tables, nodes, root))
    check_against_oracle(pkg, ctx, oracle, cp, f"seed {5000 + seed}")


@pytest.mark.parametrize("name,seed,scale", [("join2", 1, 0.02), ("snowflake", 2, 0.02), ("snowflake", 7, 0.1)])
def test_workloads_small(pkg, ctx, oracle, name, seed, scale):
    w = pkg.Workload(name, seed, scale)
    n = check_against_oracle(pkg, ctx, oracle, w.plan_ptr(), f"{name} x{scale}")
    assert n > 0


def test_join2_full_size(pkg, ctx, oracle):
    """The two-table join at its benchmark size (R 1M, S 8M), compared exactly."""
    w = pkg.Workload("join2", 1, 1.0)
    n = check_against_oracle(pkg, ctx, oracle, w.plan_ptr(), "join2 full")
    assert 7_000_000 < n < 7_400_000


def test_snowflake_full_size(pkg, ctx, oracle):
    """The five-way snowflake at its benchmark size (50M-row fact), compared exactly."""
    w = pkg.Workload("snowflake", 2, 1.0)
    check_against_oracle(pkg, ctx, oracle, w.plan_ptr(), "snowflake full")


def test_resident_equals_host_path(pkg, ctx, oracle):
    w = pkg.Workload("snowflake", 3, 0.05)
    plan = w.plan_ptr().contents
    res = [ctx.upload(plan.inputs[i]) for i in range(plan.num_inputs)]
    try:
        with ctx.execute_resident(w.plan_ptr(), res) as r:
            got, keep = r.table_struct()
            want = oracle.execute(w.plan_ptr())
            oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(), "resident")
        # Device-only result: same page counts, pages readable by copy.
        with ctx.execute_resident(w.plan_ptr(), res, flags=pkg.RESULT_DEVICE) as r:
            t = r.to_table()
            assert t.num_rows == r.num_rows
    finally:
        for x in res:
            x.free()


def test_repeated_calls_reuse_context(pkg, ctx, oracle):
    w = pkg.Workload("join2", 4, 0.01)
    for _ in range(3):
        check_against_oracle(pkg, ctx, oracle, w.plan_ptr(), "repeat")


@pytest.mark.parametrize("lt,rt", [(1, 0), (2, 2)])  # INT64 = INT32, FP64 = FP64
def test_unsupported_join_key_is_rejected(pkg, ctx, lt, rt):
    plan = pkg.Plan()
    plan.new_input(pkg.table_from_rows([[1], [2]], [lt]))
    plan.new_input(pkg.table_from_rows([[1], [2]], [rt]))
    plan.new_scan_node(0, [(0, lt)])
    plan.new_scan_node(1, [(0, rt)])
    plan.new_join_node(True, 0, 1, 0, 0, [(0, lt)])
    plan.root = 2
    with pytest.raises(pkg.EngineError) as e:
        ctx.execute(plan)
    assert e.value.status == 4
    # The context stays usable after an error.
    plan2 = pkg.Plan()
    t2 = pkg.table_from_rows([[1], [2]], [pkg.INT32])
    plan2.new_input(t2)
    plan2.new_input(t2)
    plan2.new_scan_node(0, [(0, pkg.INT32)])
    plan2.new_scan_node(1, [(0, pkg.INT32)])
    plan2.new_join_node(True, 0, 1, 0, 0, [(0, pkg.INT32), (1, pkg.INT32)])
    plan2.root = 2
    assert sorted(pkg.rows_of(ctx.execute(plan2))) == [(1, 1), (2, 2)]


def test_row_count_mismatch_is_rejected(pkg, ctx):
    """Pages holding fewer rows than the table claims: caught by the page index."""
    plan = pkg.Plan()
    t = pkg.table_from_rows([[1], [2], [3]], [pkg.INT32])
    t.num_rows = 5
    plan.new_input(t)
    plan.new_input(pkg.table_from_rows([[1]], [pkg.INT32]))
    plan.new_scan_node(0, [(0, pkg.INT32)])
    plan.new_scan_node(1, [(0, pkg.INT32)])
    plan.new_join_node(True, 0, 1, 0, 0, [(0, pkg.INT32)])
    plan.root = 2
    with pytest.raises(pkg.EngineError) as e:
        ctx.execute(plan)
    assert e.value.status == 1


def test_inconsistent_bitmap_is_rejected(pkg, ctx):
    """A page whose non-null count contradicts its bitmap (checked on device
    before any value is read)."""
    plan = pkg.Plan()
    t = pkg.table_from_rows([[1], [None], [3]], [pkg.INT32])
    bad = bytearray(t.columns[0].data)
    bad[2] = 1  # header says 1 non-null, bitmap has 2
    t.columns[0] = pkg.Column(pkg.INT32, bytes(bad))
    plan.new_input(t)
    plan.new_input(pkg.table_from_rows([[1]], [pkg.INT32]))
    plan.new_scan_node(0, [(0, pkg.INT32)])
    plan.new_scan_node(1, [(0, pkg.INT32)])
    plan.new_join_node(True, 0, 1, 0, 0, [(0, pkg.INT32)])
    plan.root = 2
    with pytest.raises(pkg.EngineError) as e:
        ctx.execute(plan)
    assert e.value.status == 1


def test_empty_and_single_table_plans(pkg, ctx, oracle):
    # A table with no rows and no columns (engine/query/PlanImport.cpp:43-49).
    plan = pkg.Plan()
    plan.new_input(pkg.ColumnarTable(0, []))
    plan.new_input(pkg.table_from_rows([[1, "a"]], [pkg.INT32, pkg.VARCHAR]))
    plan.new_scan_node(0, [(0, pkg.INT32)])
    plan.new_scan_node(1, [(0, pkg.INT32), (1, pkg.VARCHAR)])
    plan.new_join_node(True, 0, 1, 0, 0, [(0, pkg.INT32), (2, pkg.VARCHAR)])
    plan.root = 2
    out = ctx.execute(plan)
    assert out.num_rows == 0 and [c.type for c in out.columns] == [pkg.INT32, pkg.VARCHAR]
    # A lone scan returns its rows, NULLs included.
    plan = pkg.Plan()
    rows = [[i if i % 3 else None, "s" * (i % 5), float(i)] for i in range(5000)]
    plan.new_input(pkg.table_from_rows(rows, [pkg.INT32, pkg.VARCHAR, pkg.FP64]))
    plan.new_scan_node(0, [(2, pkg.FP64), (0, pkg.INT32), (1, pkg.VARCHAR)])
    plan.root = 0
    check_against_oracle(pkg, ctx, oracle, pkg.CPlan(plan), "lone scan")


@pytest.mark.parametrize("name,seed,scale", [("join2", 5, 0.6), ("snowflake", 6, 0.1)])
def test_pinned_inputs_read_in_place(pkg, ctx, oracle, name, seed, scale):
    """Large columns in pinned host memory are read in place (no staging copy;
    columns under 16 MiB are still copied) and give the same rows."""
    import torch

    w = pkg.Workload(name, seed, scale)
    plan = w.plan_ptr().contents
    regs = []
    for i in range(plan.num_inputs):
        t = plan.inputs[i]
        for c in range(t.num_columns):
            col = t.columns[c]
            if col.num_pages:
                assert torch._C._cudart.cudaHostRegister(col.pages[0], col.num_pages * pkg.PAGE_SIZE, 3) == 0
                regs.append(col.pages[0])
    try:
        with ctx.execute_raw(w.plan_ptr()) as r:
            st = r.stats()
            assert st.mapped_input_bytes > 0
            got, keep = r.table_struct()
            want = oracle.execute(w.plan_ptr())
            oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(), f"{name} pinned")
    finally:
        for p in regs:
            torch._C._cudart.cudaHostUnregister(p)


@pytest.mark.parametrize("name,seed,scale", [("snowflake", 8, 0.05), ("join2", 9, 0.1)])
def test_repeated_resident_queries_replay_graphs(pkg, ctx, oracle, name, seed, scale):
    """A resident query run again and again: the first run records, the second
    is captured into a CUDA graph, later runs replay it. Every run's rows equal
    the oracle's; freeing a table drops the graph and the next run records anew."""
    w = pkg.Workload(name, seed, scale)
    plan = w.plan_ptr().contents
    res = [ctx.upload(plan.inputs[i]) for i in range(plan.num_inputs)]
    want = oracle.execute(w.plan_ptr())
    try:
        for _ in range(4):
            with ctx.execute_resident(w.plan_ptr(), res) as r:
                got, keep = r.table_struct()
                oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(), f"{name} resident replay")
                assert r.stats().kernel_launches > 0
        for _ in range(3):
            with ctx.execute_resident(w.plan_ptr(), res, flags=pkg.RESULT_DEVICE) as r:
                t = r.to_table()
                cols = (pkg.BjColumn * max(len(t.columns), 1))()
                bufs = []
                for c, col in enumerate(t.columns):
                    buf = ctypes.create_string_buffer(col.data, max(len(col.data), 1))
                    ptrs = (ctypes.c_void_p * max(col.num_pages, 1))(
                        *[ctypes.addressof(buf) + k * pkg.PAGE_SIZE for k in range(col.num_pages)])
                    bufs += [buf, ptrs]
                    cols[c].type, cols[c].num_pages = col.type, col.num_pages
                    cols[c].pages = ctypes.cast(ptrs, ctypes.POINTER(ctypes.c_void_p))
                tab = pkg.BjTable(t.num_rows, len(t.columns), ctypes.cast(cols, ctypes.POINTER(pkg.BjColumn)))
                oracle_lib.assert_same_rows(oracle, ctypes.byref(tab), want.view(), f"{name} device replay")
    finally:
        res[-1].free()
    # A new table in the freed slot: the old graph must not be used.
    res[-1] = ctx.upload(plan.inputs[plan.num_inputs - 1])
    try:
        for _ in range(3):
            with ctx.execute_resident(w.plan_ptr(), res) as r:
                got, keep = r.table_struct()
                oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(), f"{name} after free")
    finally:
        for x in res:
            x.free()


def _uniform_int32_pages(keys, rows_per_page=1984, ragged=False):
    """INT32 pages without NULLs, rows_per_page rows each (the last page the
    rest), built directly with numpy; ragged: every third page holds 1500
    rows instead."""
    import numpy as np

    keys = np.asarray(keys, dtype=np.int32)
    starts = [0]
    while starts[-1] < len(keys):
        starts.append(starts[-1] + (1500 if ragged and len(starts) % 3 == 0 else rows_per_page))
    starts[-1] = len(keys)
    npages = len(starts) - 1
    buf = np.zeros((npages, 8192), dtype=np.uint8)
    for p in range(npages):
        v = keys[starts[p]:starts[p + 1]]
        n = len(v)
        buf[p, 0:4] = np.frombuffer(np.array([n | (n << 16)], dtype=np.uint32).tobytes(), dtype=np.uint8)
        buf[p, 4:4 + 4 * n] = np.frombuffer(v.tobytes(), dtype=np.uint8)
        nbytes = (n + 7) // 8
        bm = np.zeros(nbytes, dtype=np.uint8)
        bits = np.ones(n, dtype=np.uint8)
        bm[:] = np.packbits(np.pad(bits, (0, nbytes * 8 - n)), bitorder="little")
        buf[p, 8192 - nbytes:] = bm
    return buf


@pytest.mark.parametrize("name,seed,scale", [("snowflake", 11, 0.05), ("join2", 12, 0.1)])
def test_async_resident_results(pkg, ctx, oracle, name, seed, scale):
    """RESULT_ASYNC: replays of a captured query are enqueued back to back
    (five in flight at once) and completed afterwards, in a different order
    than issued; each one's rows equal the oracle's, its stats are readable
    after the wait, and a synchronous call after them still works."""
    w = pkg.Workload(name, seed, scale)
    plan = w.plan_ptr().contents
    res = [ctx.upload(plan.inputs[i]) for i in range(plan.num_inputs)]
    want = oracle.execute(w.plan_ptr())
    try:
        for _ in range(2):  # record, then capture
            ctx.execute_resident(w.plan_ptr(), res).free()
        pending = [ctx.execute_resident(w.plan_ptr(), res, flags=pkg.RESULT_HOST | pkg.RESULT_ASYNC)
                   for _ in range(5)]
        for k in (3, 0, 4, 1, 2):
            r = pending[k]
            r.wait()
            got, keep = r.table_struct()
            oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(), f"{name} async #{k}")
            assert r.stats().kernel_launches > 0
            r.free()
        with ctx.execute_resident(w.plan_ptr(), res) as r:
            got, keep = r.table_struct()
            oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(), f"{name} sync after async")
    finally:
        for x in res:
            x.free()


@pytest.mark.parametrize("layout", ["uniform", "null_page", "ragged"])
def test_pinned_uniform_column_speculation(pkg, ctx, oracle, layout):
    """A large pinned INT32 column whose first and last pages look uniform
    runs without a device page index; every other header is checked on the
    host meanwhile. With one middle page changed to hold a NULL (same row
    count, different header) the check fails and the call reruns with the
    full index; ragged pages (row counts differ) take the page index from the
    start. The scanned column crosses the host link in 16 MiB windows (2101
    or more pages: two windows, the second partial), so window row offsets
    come from the uniform row count, the page index's row starts or its
    chunk bases: the rows are right in every case."""
    import numpy as np
    import torch

    rows = 2100 * 1984 + 1000
    keys = np.arange(rows, dtype=np.int64) % 5000
    pages = _uniform_int32_pages(keys, ragged=layout == "ragged")
    if layout == "null_page":
        p, n = 1000, 1984
        pages[p, 0:4] = np.frombuffer(np.array([n | ((n - 1) << 16)], dtype=np.uint32).tobytes(), dtype=np.uint8)
        nbytes = (n + 7) // 8
        pages[p, 8192 - nbytes + (n - 1) // 8] &= np.uint8(~(1 << ((n - 1) % 8)) & 0xFF)
    plan = pkg.Plan()
    plan.new_input(pkg.ColumnarTable(rows, [pkg.Column(pkg.INT32, pages.tobytes())]))
    plan.new_input(pkg.table_from_rows([[k, k * 10] for k in range(0, 5000, 37)], [pkg.INT32, pkg.INT64]))
    plan.new_scan_node(0, [(0, pkg.INT32)])
    plan.new_scan_node(1, [(0, pkg.INT32), (1, pkg.INT64)])
    plan.new_join_node(False, 0, 1, 0, 0, [(0, pkg.INT32), (2, pkg.INT64)])
    plan.root = 2
    cp = pkg.CPlan(plan)
    col = cp.struct.inputs[0].columns[0]
    base = col.pages[0]
    assert torch._C._cudart.cudaHostRegister(base, col.num_pages * pkg.PAGE_SIZE, 3) == 0
    try:
        with ctx.execute_raw(cp) as r:
            assert r.stats().mapped_input_bytes > 0
            got, keep = r.table_struct()
            want = oracle.execute(cp.ref())
            n = oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(), "speculated layout")
            assert n > 0
    finally:
        torch._C._cudart.cudaHostUnregister(base)


def test_pinned_scan_window_guess_mismatch(pkg, ctx, oracle):
    """Two pinned fact key columns; the host's guess of the probe to scan
    first (the build key column sparsest over its range) is wrong here, so the
    windows it began copying go unused and the scan streams the other column:
    the rows are still the oracle's."""
    import numpy as np
    import torch

    rows = 2100 * 1984
    rng = np.random.default_rng(5)
    fk_a = rng.integers(0, 1000, rows)    # hits A's keys 0..99: 10%
    fk_b = rng.integers(0, 10000, rows)   # hits B's keys 0..9: 0.1%, the most selective
    cols = [pkg.Column(pkg.INT32, _uniform_int32_pages(fk_a).tobytes()),
            pkg.Column(pkg.INT32, _uniform_int32_pages(fk_b).tobytes())]
    plan = pkg.Plan()
    plan.new_input(pkg.ColumnarTable(rows, cols))
    plan.new_input(pkg.table_from_rows([[k] for k in list(range(100)) + [100000]], [pkg.INT32]))  # sparse range
    plan.new_input(pkg.table_from_rows([[k] for k in range(10)], [pkg.INT32]))  # dense range
    f = plan.new_scan_node(0, [(0, pkg.INT32), (1, pkg.INT32)])
    a = plan.new_scan_node(1, [(0, pkg.INT32)])
    b = plan.new_scan_node(2, [(0, pkg.INT32)])
    j1 = plan.new_join_node(False, f, a, 0, 0, [(0, pkg.INT32), (1, pkg.INT32)])
    plan.root = plan.new_join_node(False, j1, b, 1, 0, [(0, pkg.INT32), (1, pkg.INT32)])
    cp = pkg.CPlan(plan)
    regs = []
    try:
        for c in range(2):
            col = cp.struct.inputs[0].columns[c]
            assert torch._C._cudart.cudaHostRegister(col.pages[0], col.num_pages * pkg.PAGE_SIZE, 3) == 0
            regs.append(col.pages[0])
        want = oracle.execute(cp.ref())
        for _ in range(2):
            with ctx.execute_raw(cp) as r:
                assert r.stats().mapped_input_bytes > 0
                got, keep = r.table_struct()
                assert oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(), "guess mismatch") > 0
    finally:
        for p_ in regs:
            torch._C._cudart.cudaHostUnregister(p_)


def test_resident_snapshot_round_trip(pkg, ctx, oracle, tmp_path):
    """Resident tables saved to snapshot files and loaded back (no page index
    pass) answer the query exactly; truncated or foreign files are rejected."""
    w = pkg.Workload("snowflake", 14, 0.05)
    plan = w.plan_ptr().contents
    res = [ctx.upload(plan.inputs[i]) for i in range(plan.num_inputs)]
    paths = [str(tmp_path / f"t{i}.bjres") for i in range(len(res))]
    for r, path in zip(res, paths):
        ctx.save_resident(r, path)
        r.free()
    loaded = [ctx.load_resident(path) for path in paths]
    try:
        with ctx.execute_resident(w.plan_ptr(), loaded) as r:
            got, keep = r.table_struct()
            want = oracle.execute(w.plan_ptr())
            assert oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(), "snapshot") > 0
    finally:
        for x in loaded:
            x.free()
    data = open(paths[0], "rb").read()
    bad = tmp_path / "truncated.bjres"
    bad.write_bytes(data[: len(data) // 2])
    with pytest.raises(pkg.EngineError):
        ctx.load_resident(str(bad))
    foreign = tmp_path / "foreign.bjres"
    foreign.write_bytes(b"not a snapshot" * 100)
    with pytest.raises(pkg.EngineError):
        ctx.load_resident(str(foreign))
    # The context is still usable.
    w2 = pkg.Workload("join2", 15, 0.01)
    check_against_oracle(pkg, ctx, oracle, w2.plan_ptr(), "after bad snapshots")


def test_intermediate_result_beyond_32_bit_items_is_refused(pkg, ctx, oracle):
    """A join step whose result would exceed 2^32 - 2 rows (here 300K x 100K
    matches of one key in the second probe stage) is refused with
    BJ_ERR_UNSUPPORTED instead of wrapping its 32-bit item count; the context
    stays usable."""
    plan = pkg.Plan()
    plan.new_input(pkg.table_from_rows([[1, 1]] * 300_000, [pkg.INT32, pkg.INT32]))  # C: the driver
    plan.new_input(pkg.table_from_rows([[1]] + [[k] for k in range(2, 100_001)], [pkg.INT32]))  # A: unique keys
    plan.new_input(pkg.table_from_rows([[1]] * 100_000, [pkg.INT32]))  # B: one key, 100K times
    plan.new_scan_node(0, [(0, pkg.INT32), (1, pkg.INT32)])
    plan.new_scan_node(1, [(0, pkg.INT32)])
    plan.new_scan_node(2, [(0, pkg.INT32)])
    plan.new_join_node(False, 0, 1, 0, 0, [(0, pkg.INT32), (1, pkg.INT32)])
    plan.new_join_node(False, 3, 2, 1, 0, [(0, pkg.INT32)])
    plan.root = 4
    with pytest.raises(pkg.EngineError) as e:
        ctx.execute(plan)
    assert e.value.status == 4 and "intermediate rows" in str(e.value)
    w = pkg.Workload("join2", 4, 0.01)
    check_against_oracle(pkg, ctx, oracle, w.plan_ptr(), "after an intermediate overflow")


@pytest.fixture(scope="module")
def ref_ctx(pkg):
    """A context that always runs the reference space's plans (probes and
    builds keyed on an earlier probe's payload, at most two probes per
    pipeline)."""
    c = pkg.Context(0)
    c.set_plan_space(pkg.PLAN_REFERENCE)
    yield c
    c.close()


@pytest.mark.parametrize("seed", range(40))
def test_random_plans_reference_space(pkg, ref_ctx, oracle, seed):
    tables, nodes, root = plangen.random_case(1000 + seed, max_rows=3000, int64_keys=seed % 2 == 1)
    cp = pkg.CPlan(plangen.to_plan(pkg, tables, nodes, root))
    check_against_oracle(pkg, ref_ctx, oracle, cp, f"reference space seed {1000 + seed}")


def test_workloads_reference_space(pkg, ref_ctx, oracle):
    """The snowflake and 64 schema20 queries (2-12 tables) as plans of the
    reference's space, from host pages, equal to the oracle."""
    w = pkg.Workload("snowflake", 7, 0.05)
    assert check_against_oracle(pkg, ref_ctx, oracle, w.plan_ptr(), "snowflake reference space") > 0
    s = pkg.Workload("schema20", 3, 0.01)
    for k in range(0, 256, 4):
        check_against_oracle(pkg, ref_ctx, oracle, s.query_ptr(k), f"schema20 query {k} reference space")
