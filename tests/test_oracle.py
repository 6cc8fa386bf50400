"""The oracle pinned against the reference: its golden API cases and the
reference engine itself (oracle/_ref/ref_runner, built from the reference's
sources by oracle/Makefile). CPU only."""
import ctypes
import os
import subprocess
import tempfile

import pytest

import oracle_lib
import plangen
from golden.make_golden import canon, to_plan


def oracle_rows_py(pkg, oracle, cplan):
    t = oracle.execute(cplan.ref())
    tab = ctypes.cast(t.view(), ctypes.POINTER(pkg.BjTable)).contents
    cols = []
    for c in range(tab.num_columns):
        col = tab.columns[c]
        data = b"".join(ctypes.string_at(col.pages[k], pkg.PAGE_SIZE) for k in range(col.num_pages))
        cols.append(pkg.Column(col.type, data))
    return pkg.rows_of(pkg.ColumnarTable(tab.num_rows, cols)), [c.type for c in cols]


def test_oracle_matches_reference_golden_cases(pkg, oracle, golden):
    """Every API case of tests/unit_tests.cpp:19-663 gives its ground truth."""
    for case in golden:
        rows, types = oracle_rows_py(pkg, oracle, pkg.CPlan(to_plan(case, pkg)))
        assert types == case["expected_types"], case["name"]
        assert canon(rows) == canon(case["expected"]), case["name"]


def test_oracle_validates_its_own_pages(pkg, oracle):
    for seed in range(5):
        tables, nodes, root = plangen.random_case(seed, max_rows=500)
        cp = pkg.CPlan(plangen.to_plan(pkg, tables, nodes, root))
        t = oracle.execute(cp.ref())
        assert oracle.validate(t.view()) is None


def test_oracle_rejects_broken_pages(pkg, oracle):
    """A page whose non-null count contradicts its bitmap is reported (the
    validator used on every engine result)."""
    col = pkg.encode_column(pkg.INT32, [1, None, 3])
    bad = bytearray(col.data)
    bad[2] = 3  # claims 3 non-null values, bitmap has 2
    buf = ctypes.create_string_buffer(bytes(bad), len(bad))
    ptrs = (ctypes.c_void_p * 1)(ctypes.addressof(buf))
    cols = (pkg.BjColumn * 1)()
    cols[0].type, cols[0].num_pages = pkg.INT32, 1
    cols[0].pages = ctypes.cast(ptrs, ctypes.POINTER(ctypes.c_void_p))
    tab = pkg.BjTable(3, 1, ctypes.cast(cols, ctypes.POINTER(pkg.BjColumn)))
    assert "non-null" in oracle.validate(ctypes.byref(tab))


needs_ref = pytest.mark.skipif(not os.path.exists(oracle_lib.REF_RUNNER),
                               reason="reference engine not built (oracle/Makefile ref)")


def run_reference(pkg, plan_obj, tmp):
    p = os.path.join(tmp, "p.bjplan")
    o = os.path.join(tmp, "o.bjt")
    pkg.save_plan(p, plan_obj)
    subprocess.run([oracle_lib.REF_RUNNER, "run", p, o], check=True, capture_output=True, timeout=600)
    return pkg.read_table_file(o)


def table_struct(pkg, table):
    keep = []
    cols = (pkg.BjColumn * max(len(table.columns), 1))()
    for c, col in enumerate(table.columns):
        buf = ctypes.create_string_buffer(col.data, max(len(col.data), 1))
        ptrs = (ctypes.c_void_p * max(col.num_pages, 1))(
            *[ctypes.addressof(buf) + k * pkg.PAGE_SIZE for k in range(col.num_pages)])
        keep += [buf, ptrs]
        cols[c].type, cols[c].num_pages = col.type, col.num_pages
        cols[c].pages = ctypes.cast(ptrs, ctypes.POINTER(ctypes.c_void_p))
    keep.append(cols)
    return pkg.BjTable(table.num_rows, len(table.columns), ctypes.cast(cols, ctypes.POINTER(pkg.BjColumn))), keep


@needs_ref
@pytest.mark.parametrize("seed", range(40))
def test_oracle_matches_reference_engine_random_plans(pkg, oracle, seed):
    # The reference engine needs at least one join (its scans of a lone table
    # assume a join column, engine/op/TableScan.cpp:480).
    tables, nodes, root = plangen.random_case(seed, max_tables=4, max_rows=2500, min_tables=2, max_width=3)
    plan = plangen.to_plan(pkg, tables, nodes, root)
    cp = pkg.CPlan(plan)
    # The reference turns an INT64 -1 / all-ones FP64 into NULL (its NULL is ~0ull,
    # engine/query/RuntimeValue.hpp:10); plangen never draws those values.
    with tempfile.TemporaryDirectory() as tmp:
        ref = run_reference(pkg, cp, tmp)
    ref_struct, keep = table_struct(pkg, ref)
    ora = oracle.execute(cp.ref())
    oracle_lib.assert_same_rows(oracle, ctypes.byref(ref_struct), ora.view(), f"seed {seed}")


@needs_ref
@pytest.mark.parametrize("name,seed,scale", [("join2", 1, 0.01), ("snowflake", 2, 0.02)])
def test_oracle_matches_reference_engine_workloads(pkg, oracle, name, seed, scale):
    w = pkg.Workload(name, seed, scale)
    with tempfile.TemporaryDirectory() as tmp:
        ref = run_reference(pkg, w.plan_ptr(), tmp)
    ref_struct, keep = table_struct(pkg, ref)
    ora = oracle.execute(w.plan_ptr())
    n = oracle_lib.assert_same_rows(oracle, ctypes.byref(ref_struct), ora.view(), name)
    assert n > 0


@needs_ref
@pytest.mark.parametrize("case", [
    (21, 60_000, 2_000, 40_000, 200_000),   # the small input holds ~1% of the keys
    (22, 50_000, 8_000, 30_000, 2_000),     # few keys, many repeated on every side
])
def test_oracle_matches_reference_engine_star_on_one_key(pkg, oracle, case):
    """Three inputs joined on one key class, the shape in which the reference
    restricts the large input's scan by the small input's finished table
    (engine/query/QueryPlan.cpp:620-624, :670-676): the oracle gives the
    reference engine's rows."""
    cp = plangen.star_plan(pkg, *case)
    with tempfile.TemporaryDirectory() as tmp:
        ref = run_reference(pkg, cp, tmp)
    ref_struct, keep = table_struct(pkg, ref)
    ora = oracle.execute(cp.ref())
    n = oracle_lib.assert_same_rows(oracle, ctypes.byref(ref_struct), ora.view(), f"star {case}")
    assert n > 0
