"""The C-ABI libraries load and export every symbol their headers declare.
CPU only: nothing here calls into CUDA."""
import ctypes
import os
import re
import subprocess

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "contest-sigmod2025_b200")


def declared(header):
    text = open(header).read()
    return sorted(set(re.findall(r"BJ_API\s+[\w\s\*]+?\b(bjw?_\w+)\s*\(", text)))


def test_engine_exports_every_declared_symbol(pkg):
    names = declared(os.path.join(REPO, "include", "b200join.h"))
    assert "bj_execute" in names and "bj_context_create" in names
    lib = ctypes.CDLL(os.path.join(PKG, "libb200join.so"))
    for n in names:
        assert hasattr(lib, n), n
    # the Python binding covers the same set
    assert sorted(pkg.ABI) == names


def test_workload_library_exports(pkg):
    names = declared(os.path.join(PKG, "csrc", "workloads.h"))
    lib = ctypes.CDLL(os.path.join(PKG, "libb200join_workloads.so"))
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(pkg.WORKLOAD_ABI) == names


def test_contest_dropin_exports_contest_api():
    out = subprocess.run(["nm", "-DC", os.path.join(PKG, "libcontest_b200.so")], capture_output=True, text=True,
                         check=True).stdout
    for sym in ["Contest::build_context()", "Contest::destroy_context(void*)", "Contest::execute(Plan const&, void*)"]:
        assert re.search(r" T " + re.escape(sym), out), sym


def test_python_page_codec_round_trip(pkg):
    rows = [[i if i % 7 else None, f"s{i}" * (i % 4) if i % 5 else None, i * 1.5, -i * (1 << 33)]
            for i in range(5000)]
    rows.append([1, "x" * 20000, 0.0, 0])  # long string page run
    t = pkg.table_from_rows(rows, [pkg.INT32, pkg.VARCHAR, pkg.FP64, pkg.INT64])
    back = pkg.rows_of(t)
    assert [list(r) for r in back] == rows
