"""The C++ drop-in: a program built against include/contest/plan.h and linked
with libcontest_b200.so (no engine sources) runs plans through
Contest::build_context / execute / destroy_context, and its results equal the
oracle's. Its result pages are freed by Column's destructor with plain delete."""
import ctypes
import os
import subprocess

import pytest

import oracle_lib
from golden.make_golden import canon, to_plan
from test_oracle import table_struct

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
PKG = os.path.join(REPO, "contest-sigmod2025_b200")


@pytest.fixture(scope="module")
def dropin(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("dropin") / "contest_dropin")
    subprocess.run(["g++", "-std=c++20", "-O2", "-o", exe, os.path.join(HERE, "cpp", "contest_dropin.cpp"),
                    "-L" + PKG, "-lcontest_b200", "-lb200join", "-Wl,-rpath," + PKG], check=True)
    return exe


def run(dropin, pkg, plan, tmp_path, repeat=1):
    p, o = str(tmp_path / "p.bjplan"), str(tmp_path / "o.bjt")
    pkg.save_plan(p, plan)
    subprocess.run([dropin, p, o, str(repeat)], check=True, timeout=600)
    return pkg.read_table_file(o)


def test_golden_cases_through_contest_api(pkg, golden, dropin, tmp_path):
    for case in golden:
        out = run(dropin, pkg, to_plan(case, pkg), tmp_path)
        assert [c.type for c in out.columns] == case["expected_types"], case["name"]
        assert canon(pkg.rows_of(out)) == canon(case["expected"]), case["name"]


@pytest.mark.parametrize("name,seed,scale", [("join2", 3, 0.1), ("snowflake", 4, 0.1)])
def test_workloads_through_contest_api(pkg, oracle, dropin, tmp_path, name, seed, scale):
    w = pkg.Workload(name, seed, scale)
    out = run(dropin, pkg, w.plan_ptr(), tmp_path, repeat=2)
    got, keep = table_struct(pkg, out)
    want = oracle.execute(w.plan_ptr())
    assert oracle_lib.assert_same_rows(oracle, ctypes.byref(got), want.view(), name) > 0
