"""Seeded random plans for parity tests.

Random join trees over 1-6 tables: INT32 join keys drawn from small domains
(so keys repeat and chains fan out), NULL keys, INT32/INT64/FP64/VARCHAR
payloads with NULLs, empty and long (>8185 byte) strings, intermediate
projections that drop attributes, and root outputs that repeat or reorder
attributes. Table sizes span empty, one row and multi-page columns.

With int64_keys, every table also has an INT64 key column whose values share
their low 32 bits across several high halves (negative ones included), and
joins pair INT64 keys where both sides carry one: keys that only a full
64-bit comparison tells apart. (The reference reads join keys as 32 bits,
engine/op/TableScan.cpp:328; these plans are checked against the oracle.)
"""
import random

import numpy as np

INT32, INT64, FP64, VARCHAR = 0, 1, 2, 3


def _value(rng, ty, dom, null_p, long_p):
    if rng.random() < null_p:
        return None
    if ty == INT32:
        return rng.randrange(dom)
    if ty == INT64:
        return rng.randrange(-(1 << 62), 1 << 62)
    if ty == FP64:
        return rng.choice([0.0, -0.0, 1.5, -2.25, 1e300, rng.random() * 1e6])
    if rng.random() < long_p:
        return "L" * rng.randrange(8186, 20000)
    return "".join(chr(32 + rng.randrange(95)) for _ in range(rng.randrange(0, 24)))


def _key64(rng, dom, null_p):
    if rng.random() < null_p:
        return None
    return (rng.choice([0, 1, 7, -1, -5]) << 32) | rng.randrange(dom)


# INT32 keys at the edges of the type and around zero (signed_keys).
_EDGE32 = [-1, -2, -(1 << 31), (1 << 31) - 1, (1 << 31) - 2, 0, 1]


def _key32_signed(rng, dom, null_p, edge_p):
    """An INT32 key from a small domain that straddles zero, or (with
    probability edge_p) one of the type's edge values (-1 is 0xFFFFFFFF, the
    all-ones pattern)."""
    if rng.random() < null_p:
        return None
    if rng.random() < edge_p:
        return rng.choice(_EDGE32)
    return rng.randrange(-(dom // 2), dom - dom // 2)  # dom values around zero


def random_case(seed, max_tables=5, max_rows=3000, min_tables=1, max_width=None, int64_keys=False,
                signed_keys=False):
    """max_width caps the attributes a join node outputs (the reference only
    instantiates pipelines carrying a few attributes, engine/genpipelines.py:15-49).
    signed_keys draws the INT32 join keys from a domain around zero plus the
    type's edge values."""
    """Returns (tables, nodes, root) in the form tests/golden/make_golden.py uses."""
    rng = random.Random(seed)
    ntables = rng.randint(min_tables, max_tables)
    tables = []
    for _ in range(ntables):
        r = rng.random()
        nrows = 0 if r < 0.04 else 1 if r < 0.1 else rng.randint(2, 40) if r < 0.5 else rng.randint(41, max_rows)
        nkeys = rng.randint(1, 2)
        npay = rng.randint(0, 3)
        types = [INT32] * nkeys + [rng.choice([INT32, INT64, FP64, VARCHAR]) for _ in range(npay)]
        dom = max(1, int(nrows * rng.choice([0.2, 0.5, 1.0, 3.0])))
        null_p = rng.choice([0.0, 0.0, 0.05, 0.3])
        long_p = 0.002 if rng.random() < 0.3 else 0.0
        rows = [[_value(rng, ty, dom, null_p, long_p) for ty in types] for _ in range(nrows)]
        if signed_keys:
            # About 20 edge values per table whatever its size: their
            # repeats multiply across a join chain.
            edge_p = min(0.2, 20.0 / max(nrows, 1))
            for r in rows:
                for k in range(nkeys):
                    r[k] = _key32_signed(rng, dom, null_p, edge_p)
        if int64_keys:
            types.insert(1, INT64)
            for r in rows:
                r.insert(1, _key64(rng, dom, null_p))
        tables.append({"types": types, "rows": rows, "keys64": {1} if int64_keys else set()})
    nodes = []
    subtrees = []  # (node id, [type per output attr])
    for t, tab in enumerate(tables):
        cols = list(range(len(tab["types"])))
        rng.shuffle(cols)
        keep = cols[:rng.randint(1, len(cols))]
        if not any(tab["types"][c] == INT32 for c in keep):
            keep.append(next(c for c in cols if tab["types"][c] == INT32))
        if int64_keys and 1 not in keep and rng.random() < 0.8:
            keep.append(1)
        attrs = [[c, tab["types"][c]] for c in keep]
        nodes.append({"kind": "scan", "table": t, "attrs": attrs})
        # per output attribute: (type, is a key column)
        subtrees.append((len(nodes) - 1, [a[1] for a in attrs],
                         [a[1] == INT32 or a[0] in tab["keys64"] for a in attrs]))
    while len(subtrees) > 1:
        a = subtrees.pop(rng.randrange(len(subtrees)))
        b = subtrees.pop(rng.randrange(len(subtrees)))
        key_ty = INT32
        if int64_keys and rng.random() < 0.6:
            if any(t == INT64 and k for t, k in zip(a[1], a[2])) and any(t == INT64 and k for t, k in zip(b[1], b[2])):
                key_ty = INT64
        la = rng.choice([i for i, ty in enumerate(a[1]) if ty == key_ty and a[2][i]])
        ra = rng.choice([i for i, ty in enumerate(b[1]) if ty == key_ty and b[2][i]])
        both = a[1] + b[1]
        idx = list(range(len(both)))
        if rng.random() < 0.5 or (max_width and len(idx) > max_width):
            rng.shuffle(idx)
            idx = idx[:rng.randint(1, min(len(idx), max_width or len(idx)))]
        if not any(both[i] == INT32 for i in idx):
            idx.append(next(i for i in range(len(both)) if both[i] == INT32))
        keyflags = a[2] + b[2]
        attrs = [[i, both[i]] for i in idx]
        nodes.append({"kind": "join", "build_left": rng.random() < 0.5, "left": a[0], "right": b[0], "left_attr": la,
                      "right_attr": ra, "attrs": attrs})
        subtrees.append((len(nodes) - 1, [x[1] for x in attrs], [keyflags[i] for i in idx]))
    root, rtypes, _ = subtrees[0]
    if rng.random() < 0.3 and nodes[root]["kind"] == "join":
        # Root output repeating / reordering attributes.
        n = nodes[root]
        base = n["attrs"]
        n["attrs"] = [rng.choice(base) for _ in range(rng.randint(1, min(len(base) + 2, max_width or 99)))]
    return tables, nodes, root


def to_plan(pkg, tables, nodes, root):
    plan = pkg.Plan()
    for t in tables:
        plan.new_input(pkg.table_from_rows(t["rows"], t["types"]))
    for n in nodes:
        attrs = [tuple(a) for a in n["attrs"]]
        if n["kind"] == "scan":
            plan.new_scan_node(n["table"], attrs)
        else:
            plan.new_join_node(n["build_left"], n["left"], n["right"], n["left_attr"], n["right_attr"], attrs)
    plan.root = root
    return plan



INT32_EDGES = [-1, -2**31, 2**31 - 1, 0, 1]


def _star_keys(rng, n, lo, hi, null_p, edges=False):
    k = rng.integers(lo, hi, size=n, dtype=np.int64)
    out = [int(x) for x in k]
    if edges:
        for i in rng.choice(n, size=min(n, 16), replace=False):
            out[int(i)] = INT32_EDGES[int(i) % len(INT32_EDGES)]
    if null_p:
        for i in np.nonzero(rng.random(n) < null_p)[0]:
            out[int(i)] = None
    return out


def star_plan(pkg, seed, fact_rows, small_rows, large_rows, small_dom, edges=False):
    """A fact (INT32 key, INT64 payload) joined on its key with a small input
    (key, INT32 payload) and a large input (key, VARCHAR payload): one key
    class over three inputs, the shape whose large build a sideways
    restriction filters by the small input's bloom filter. Keys of the fact
    and the large input lie in [0, 200000), the small input's in
    [0, small_dom); 5% of the fact's keys and 3% of the large input's are
    NULL; with `edges`, up to 16 keys per table are INT32 edge values (-1,
    INT32_MIN, INT32_MAX, 0, 1). The root outputs the fact's payload, the small
    input's payload, the large input's key and payload."""
    rng = np.random.default_rng(seed)
    dom = 200_000
    fact = pkg.ColumnarTable(num_rows=fact_rows)
    fact.columns.append(pkg.encode_column(pkg.INT32, _star_keys(rng, fact_rows, 0, dom, 0.05, edges)))
    fact.columns.append(pkg.encode_column(pkg.INT64, [int(x) for x in rng.integers(-2**40, 2**40, size=fact_rows)]))
    small = pkg.ColumnarTable(num_rows=small_rows)
    small.columns.append(pkg.encode_column(pkg.INT32, _star_keys(rng, small_rows, 0, small_dom, 0.0, edges)))
    small.columns.append(pkg.encode_column(pkg.INT32, [int(x) for x in rng.integers(0, 1000, size=small_rows)]))
    large = pkg.ColumnarTable(num_rows=large_rows)
    large.columns.append(pkg.encode_column(pkg.INT32, _star_keys(rng, large_rows, 0, dom, 0.03, edges)))
    large.columns.append(pkg.encode_column(pkg.VARCHAR, [f"v{int(x)}" for x in rng.integers(0, 10**6, size=large_rows)]))
    plan = pkg.Plan()
    for t in (fact, small, large):
        plan.new_input(t)
    f = plan.new_scan_node(0, [(0, pkg.INT32), (1, pkg.INT64)])
    s = plan.new_scan_node(1, [(0, pkg.INT32), (1, pkg.INT32)])
    j1 = plan.new_join_node(True, f, s, 0, 0, [(0, pkg.INT32), (1, pkg.INT64), (2, pkg.INT32), (3, pkg.INT32)])
    lg = plan.new_scan_node(2, [(0, pkg.INT32), (1, pkg.VARCHAR)])
    j2 = plan.new_join_node(True, j1, lg, 0, 0, [(1, pkg.INT64), (3, pkg.INT32), (4, pkg.INT32), (5, pkg.VARCHAR)])
    plan.root = j2
    return pkg.CPlan(plan)
