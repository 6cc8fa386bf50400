"""Generates tests/golden/unit_cases.json: the reference's API test cases.

Each case restates one Catch2 test of the contest repository's
tests/unit_tests.cpp (line given per case) as data: input tables as rows,
the plan's nodes, and the expected result rows (the test's ground truth,
sorted). The tests in tests/ run every case through the oracle and through
the engine.

Run with --check to also execute every case with the reference engine built
by oracle/Makefile (oracle/_ref/ref_runner) and confirm that it returns the
expected rows.
"""
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))

I, V = 0, 3  # INT32, VARCHAR
N = None


def scan(t, attrs):
    return {"kind": "scan", "table": t, "attrs": attrs}


def join(build_left, left, right, la, ra, attrs):
    return {"kind": "join", "build_left": build_left, "left": left, "right": right, "left_attr": la,
            "right_attr": ra, "attrs": attrs}


def case(name, source, tables, nodes, root, types, expected):
    return {"name": name, "source": source, "tables": tables, "nodes": nodes, "root": root,
            "expected_types": types, "expected": sorted(expected, key=lambda r: json.dumps(r))}


def cases():
    out = []
    one = {"types": [I], "rows": [[1]]}
    out.append(case("empty_join", "tests/unit_tests.cpp:19", [{"types": [I], "rows": []}, {"types": [I], "rows": []}],
                    [scan(0, [[0, I]]), scan(1, [[0, I]]), join(True, 0, 1, 0, 0, [[0, I], [1, I]])], 2, [I, I], []))
    out.append(case("one_line_join", "tests/unit_tests.cpp:39", [one, one],
                    [scan(0, [[0, I]]), scan(1, [[0, I]]), join(True, 0, 1, 0, 0, [[0, I], [1, I]])], 2, [I, I],
                    [[1, 1]]))
    t123 = {"types": [I], "rows": [[1], [2], [3]]}
    out.append(case("simple_join", "tests/unit_tests.cpp:68", [t123, t123],
                    [scan(0, [[0, I]]), scan(1, [[0, I]]), join(True, 0, 1, 0, 0, [[0, I], [1, I]])], 2, [I, I],
                    [[1, 1], [2, 2], [3, 3]]))
    out.append(case("empty_result", "tests/unit_tests.cpp:102", [t123, {"types": [I], "rows": [[4], [5], [6]]}],
                    [scan(0, [[0, I]]), scan(1, [[0, I]]), join(True, 0, 1, 0, 0, [[0, I], [1, I]])], 2, [I, I], []))
    dup = {"types": [I], "rows": [[1], [1], [2], [3]]}
    out.append(case("multiple_same_keys", "tests/unit_tests.cpp:134", [dup, dup],
                    [scan(0, [[0, I]]), scan(1, [[0, I]]), join(True, 0, 1, 0, 0, [[0, I], [1, I]])], 2, [I, I],
                    [[1, 1]] * 4 + [[2, 2], [3, 3]]))
    nul = {"types": [I], "rows": [[1], [1], [N], [2], [3]]}
    out.append(case("null_keys", "tests/unit_tests.cpp:172", [nul, nul],
                    [scan(0, [[0, I]]), scan(1, [[0, I]]), join(True, 0, 1, 0, 0, [[0, I], [1, I]])], 2, [I, I],
                    [[1, 1]] * 4 + [[2, 2], [3, 3]]))
    mc = {"types": [I, V], "rows": [[1, "xxx"], [1, "yyy"], [N, "zzz"], [2, "uuu"], [3, "vvv"]]}
    out.append(case("multiple_columns", "tests/unit_tests.cpp:211", [mc, mc],
                    [scan(0, [[0, I]]), scan(1, [[1, V], [0, I]]),
                     join(True, 0, 1, 0, 1, [[0, I], [2, I], [1, V]])], 2, [I, I, V],
                    [[1, 1, "xxx"], [1, 1, "xxx"], [1, 1, "yyy"], [1, 1, "yyy"], [2, 2, "uuu"], [3, 3, "vvv"]]))
    br = {"types": [I, V], "rows": [[10, "xxx"], [10, "yyy"], [N, "zzz"], [20, "uuu"], [30, "vvv"]]}
    out.append(case("build_on_right", "tests/unit_tests.cpp:252", [br, br],
                    [scan(0, [[0, I]]), scan(1, [[1, V], [0, I]]),
                     join(False, 0, 1, 0, 1, [[0, I], [2, I], [1, V]])], 2, [I, I, V],
                    [[10, 10, "xxx"], [10, 10, "xxx"], [10, 10, "yyy"], [10, 10, "yyy"], [20, 20, "uuu"],
                     [30, 30, "vvv"]]))
    out.append(case("ternary", "tests/unit_tests.cpp:294", [br, br, br],
                    [scan(0, [[0, I]]), scan(1, [[1, V], [0, I]]), scan(2, [[0, I]]),
                     join(False, 0, 1, 0, 1, [[0, I], [2, I], [1, V]]),
                     join(False, 2, 3, 0, 0, [[0, I], [1, I], [3, V]])], 4, [I, I, V],
                    [[10, 10, "xxx"]] * 4 + [[10, 10, "yyy"]] * 4 + [[20, 20, "uuu"], [30, 30, "vvv"]]))
    cp1 = {"types": [I, V], "rows": [[10, "xxx"], [10, "xxx"], [10, "yyy"], [N, "zzz"], [20, "uuu"], [20, "uuu"],
                                     [30, "vvv"]]}
    cp2 = {"types": [I, I], "rows": [[10, 20]]}
    out.append(case("cross_product", "tests/unit_tests.cpp:343", [cp1, cp2, cp1],
                    [scan(0, [[0, I], [1, V]]), scan(1, [[0, I], [1, I]]), scan(2, [[0, I], [1, V]]),
                     join(False, 0, 1, 0, 0, [[0, I], [1, V], [2, I], [3, I]]),
                     join(False, 3, 2, 3, 0, [[0, I], [1, V], [2, I], [3, I], [4, I], [5, V]])], 4,
                    [I, V, I, I, I, V],
                    [[10, "xxx", 10, 20, 20, "uuu"]] * 4 + [[10, "yyy", 10, 20, 20, "uuu"]] * 2))
    # 5 tables: R, S (singleton), T, U (singleton), V.
    r = {"types": [I, V], "rows": [[10, "r1"], [20, "r2"], [30, "r3"]]}
    s = {"types": [I, I], "rows": [[10, 100]]}
    t = {"types": [I, V, I], "rows": [[100, "200", 300], [100, "210", 300], [101, "220", 300]]}
    u = {"types": [I, I], "rows": [[300, 400]]}
    v = {"types": [I, V], "rows": [[400, "v1"], [401, "v2"]]}
    a7 = [[0, I], [1, V], [2, I], [3, I], [4, I], [5, V], [6, I]]
    out.append(case("cross_product_5_tables", "tests/unit_tests.cpp:398", [r, s, t, u, v],
                    [scan(0, [[0, I], [1, V]]), scan(1, [[0, I], [1, I]]), scan(2, [[0, I], [1, V], [2, I]]),
                     scan(3, [[0, I], [1, I]]), scan(4, [[0, I], [1, V]]),
                     join(False, 0, 1, 0, 0, [[0, I], [1, V], [2, I], [3, I]]),
                     join(False, 5, 2, 3, 0, a7),
                     join(False, 6, 3, 6, 0, a7 + [[7, I], [8, I]]),
                     join(False, 7, 4, 8, 0, a7 + [[7, I], [8, I], [9, I], [10, V]])], 8,
                    [I, V, I, I, I, V, I, I, I, I, V],
                    [[10, "r1", 10, 100, 100, "200", 300, 300, 400, 400, "v1"],
                     [10, "r1", 10, 100, 100, "210", 300, 300, 400, 400, "v1"]]))
    # 7 tables chained, singletons at odd positions.
    d = [{"types": [I, I], "rows": rows} for rows in (
        [[10, 111], [20, 222]], [[10, 100]], [[100, 200], [100, 210]], [[200, 300]], [[300, 400], [300, 410]],
        [[400, 500]], [[500, 600], [500, 610]])]
    nodes = [scan(k, [[0, I], [1, I]]) for k in range(7)]
    nodes.append(join(False, 0, 1, 0, 0, [[k, I] for k in range(4)]))
    for step, (left, la) in enumerate([(7, 3), (8, 5), (9, 7), (10, 9), (11, 11)]):
        width = 4 + 2 * (step + 1)
        nodes.append(join(False, left, 2 + step, la, 0, [[k, I] for k in range(width)]))
    out.append(case("cross_product_7_tables", "tests/unit_tests.cpp:513", d, nodes, 12, [I] * 14,
                    [[10, 111, 10, 100, 100, 200, 200, 300, 300, 400, 400, 500, 500, 600],
                     [10, 111, 10, 100, 100, 200, 200, 300, 300, 400, 400, 500, 500, 610]]))
    return out


def to_plan(c, pkg):
    plan = pkg.Plan()
    for t in c["tables"]:
        plan.new_input(pkg.table_from_rows(t["rows"], t["types"]))
    for n in c["nodes"]:
        attrs = [tuple(a) for a in n["attrs"]]
        if n["kind"] == "scan":
            plan.new_scan_node(n["table"], attrs)
        else:
            plan.new_join_node(n["build_left"], n["left"], n["right"], n["left_attr"], n["right_attr"], attrs)
    plan.root = c["root"]
    return plan


def canon(rows):
    return sorted([list(r) for r in rows], key=lambda r: json.dumps(r))


def main():
    cs = cases()
    with open(os.path.join(HERE, "unit_cases.json"), "w") as f:
        json.dump(cs, f, indent=1)
    print(f"wrote {len(cs)} cases")
    if "--check" in sys.argv:
        import importlib
        sys.path.insert(0, REPO)
        pkg = importlib.import_module("contest-sigmod2025_b200")
        runner = os.path.join(REPO, "oracle", "_ref", "ref_runner")
        with tempfile.TemporaryDirectory() as tmp:
            for c in cs:
                p = os.path.join(tmp, "p.bjplan")
                o = os.path.join(tmp, "o.bjt")
                pkg.save_plan(p, to_plan(c, pkg))
                subprocess.run([runner, "run", p, o], check=True, capture_output=True)
                got = pkg.rows_of(pkg.read_table_file(o))
                ok = canon(got) == canon(c["expected"])
                print(f"{c['name']:28s} reference engine {'agrees' if ok else 'DIFFERS'} ({len(got)} rows)")
                if not ok:
                    sys.exit(1)


if __name__ == "__main__":
    main()
