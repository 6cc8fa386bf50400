"""Python host-side mirror of the contest API over the B200 join engine.

The engine itself is C++/CUDA (libb200join.so, C ABI in include/b200join.h).
This module mirrors the contest's plan-building interface (include/plan.h of
the contest repository: ``Plan.new_scan_node / new_join_node / new_input``,
``ColumnarTable``, ``Contest::build_context / execute / destroy_context``) so
tests and tools read like the reference's own tests
(tests/unit_tests.cpp:19-663), and binds the C ABI with ctypes.

The package directory name contains a hyphen; import it with
``importlib.import_module("contest-sigmod2025_b200")``.

There is no CPU fallback: if the CUDA library is missing or no GPU is
visible, ``build_context`` raises.
"""
from __future__ import annotations

import ctypes
import os
import struct
from dataclasses import dataclass, field
from typing import Iterable, List, Optional, Sequence, Tuple

_HERE = os.path.dirname(os.path.abspath(__file__))
PAGE_SIZE = 8192

INT32, INT64, FP64, VARCHAR = 0, 1, 2, 3
TYPE_NAMES = {INT32: "INT32", INT64: "INT64", FP64: "FP64", VARCHAR: "VARCHAR"}
NODE_JOIN, NODE_SCAN = 0, 1
RESULT_HOST, RESULT_DEVICE, RESULT_ASYNC = 0, 1, 2

STATUS = {0: "OK", 1: "INVALID", 2: "CUDA", 3: "OOM", 4: "UNSUPPORTED", 5: "INTERNAL", 6: "NO_DEVICE"}


class EngineError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"b200join {STATUS.get(status, status)}: {msg}")
        self.status = status


# ---------------------------------------------------------------------------
# C structures (include/b200join.h)

class BjColumn(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("reserved", ctypes.c_uint32), ("num_pages", ctypes.c_uint64),
                ("pages", ctypes.POINTER(ctypes.c_void_p))]


class BjTable(ctypes.Structure):
    _fields_ = [("num_rows", ctypes.c_uint64), ("num_columns", ctypes.c_uint64), ("columns", ctypes.POINTER(BjColumn))]


class BjAttr(ctypes.Structure):
    _fields_ = [("index", ctypes.c_uint64), ("type", ctypes.c_int32), ("reserved", ctypes.c_uint32)]


class BjNode(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("build_left", ctypes.c_int32), ("base_table_id", ctypes.c_uint64),
                ("left", ctypes.c_uint64), ("right", ctypes.c_uint64), ("left_attr", ctypes.c_uint64),
                ("right_attr", ctypes.c_uint64), ("num_output_attrs", ctypes.c_uint64),
                ("output_attrs", ctypes.POINTER(BjAttr))]


class BjPlan(ctypes.Structure):
    _fields_ = [("num_nodes", ctypes.c_uint64), ("nodes", ctypes.POINTER(BjNode)), ("num_inputs", ctypes.c_uint64),
                ("inputs", ctypes.POINTER(BjTable)), ("root", ctypes.c_uint64)]


class BjStats(ctypes.Structure):
    _fields_ = [("kernel_launches", ctypes.c_uint64), ("pipelines", ctypes.c_uint64), ("h2d_bytes", ctypes.c_uint64),
                ("d2h_bytes", ctypes.c_uint64), ("input_pages", ctypes.c_uint64), ("output_pages", ctypes.c_uint64),
                ("device_ms", ctypes.c_double), ("total_ms", ctypes.c_double),
                ("scan_kernel_ms", ctypes.c_double), ("scan_kernel_launches", ctypes.c_uint64),
                ("scan_kernel_bytes", ctypes.c_uint64), ("mapped_input_bytes", ctypes.c_uint64),
                ("phase_ms", ctypes.c_double * 4), ("arena_bytes", ctypes.c_uint64)]


# Every symbol include/b200join.h declares, with its ctypes signature.
_VP, _U64, _I32, _INT = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int32, ctypes.c_int
ABI = {
    "bj_version": (ctypes.c_char_p, []),
    "bj_context_create": (_INT, [_INT, ctypes.POINTER(_VP)]),
    "bj_context_destroy": (None, [_VP]),
    "bj_last_error": (ctypes.c_char_p, [_VP]),
    "bj_execute": (_INT, [_VP, ctypes.POINTER(BjPlan), ctypes.POINTER(_VP)]),
    "bj_resident_upload": (_INT, [_VP, ctypes.POINTER(BjTable), ctypes.POINTER(_VP)]),
    "bj_resident_free": (None, [_VP, _VP]),
    "bj_resident_save": (_INT, [_VP, _VP, ctypes.c_char_p]),
    "bj_resident_load": (_INT, [_VP, ctypes.c_char_p, ctypes.POINTER(_VP)]),
    "bj_execute_resident": (_INT, [_VP, ctypes.POINTER(BjPlan), ctypes.POINTER(_VP), _INT, ctypes.POINTER(_VP)]),
    "bj_result_num_rows": (_U64, [_VP]),
    "bj_result_num_columns": (_U64, [_VP]),
    "bj_result_column_type": (_I32, [_VP, _U64]),
    "bj_result_column_num_pages": (_U64, [_VP, _U64]),
    "bj_result_page": (_VP, [_VP, _U64, _U64]),
    "bj_result_device_page": (_VP, [_VP, _U64, _U64]),
    "bj_result_copy_pages": (_INT, [_VP, _U64, ctypes.POINTER(_VP)]),
    "bj_result_stats": (_INT, [_VP, ctypes.POINTER(BjStats)]),
    "bj_result_free": (None, [_VP]),
    "bj_context_stream": (_VP, [_VP]),
    "bj_context_profile": (None, [_VP, _INT]),
    "bj_join_count_static": (_INT, [_VP, _U64, _U64, _VP, _U64, _VP, _VP]),
    "bj_server_create": (_INT, [_INT, _INT, _U64, ctypes.POINTER(_VP)]),
    "bj_server_destroy": (None, [_VP]),
    "bj_server_context": (_VP, [_VP, _INT]),
    "bj_server_submit": (_INT, [_VP, ctypes.POINTER(BjPlan), ctypes.POINTER(_VP), _INT, ctypes.POINTER(_U64)]),
    "bj_server_wait": (_INT, [_VP, _U64, ctypes.POINTER(_VP), ctypes.POINTER(ctypes.c_double)]),
    "bj_server_resident_free": (None, [_VP, _VP]),
    "bj_plan_explain": (_INT, [ctypes.POINTER(BjPlan), ctypes.c_char_p, _U64, ctypes.POINTER(_U64)]),
    "bj_result_wait": (_INT, [_VP]),
    "bj_context_set_ordering": (_INT, [_VP, _INT, _VP]),
    "bj_server_set_ordering": (_INT, [_VP, _INT, _VP]),
    "bj_server_set_graphs": (None, [_VP, _INT]),
    "bj_context_set_graphs": (None, [_VP, _INT]),
    "bj_context_set_plan_space": (_INT, [_VP, _INT]),
    "bj_context_autotune": (_INT, [_VP, ctypes.POINTER(BjPlan), ctypes.POINTER(_VP), _INT, ctypes.c_char_p, _U64,
                                   ctypes.POINTER(_U64)]),
    "bj_plan_scratch_estimate": (_INT, [_VP, ctypes.POINTER(BjPlan), ctypes.POINTER(_VP), ctypes.POINTER(_U64)]),
    "bj_server_run_load": (_INT, [_VP, _VP, _U64, _VP, _VP, _U64, ctypes.c_double, ctypes.c_uint32, _U64, _VP,
                                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_U64)]),
    "bj_resident_set_base_rows": (_INT, [_VP, _U64]),
    "bj_subplans": (_INT, [ctypes.POINTER(BjPlan), ctypes.c_uint32, _U64, _VP, ctypes.POINTER(_U64)]),
    "bj_subplan_cards": (_INT, [_VP, ctypes.POINTER(BjPlan), ctypes.POINTER(_VP), _VP, _U64, _VP]),
    "bj_subplan_sample_cards": (_INT, [_VP, ctypes.POINTER(BjPlan), ctypes.POINTER(_VP), _VP, _U64, _VP]),
    "bj_subplan_features": (_INT, [_VP, ctypes.POINTER(BjPlan), ctypes.POINTER(_VP), _VP, _U64, _VP]),
    "bj_join_order": (_INT, [ctypes.POINTER(BjPlan), _VP, _INT, ctypes.POINTER(ctypes.c_uint32),
                             ctypes.POINTER(ctypes.c_double)]),
    "bj_estimator_create": (_INT, [_INT, _U64, ctypes.POINTER(_VP)]),
    "bj_estimator_destroy": (None, [_VP]),
    "bj_estimator_num_params": (_U64, []),
    "bj_estimator_get_params": (_INT, [_VP, _VP]),
    "bj_estimator_set_params": (_INT, [_VP, _VP]),
    "bj_estimator_train": (_INT, [_VP, _VP, _VP, _U64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, _U64, _VP]),
    "bj_estimator_predict": (_INT, [_VP, _VP, _U64, _VP]),
    "bj_estimator_gradients": (_INT, [_VP, _VP, _VP, _U64, _VP, _VP]),
    "bj_estimator_save": (_INT, [_VP, ctypes.c_char_p]),
    "bj_estimator_load": (_INT, [_INT, ctypes.c_char_p, ctypes.POINTER(_VP)]),
}

ORDER_ROWS, ORDER_SAMPLING, ORDER_LEARNED = 0, 1, 2
PLAN_AUTO, PLAN_ROOTED, PLAN_REFERENCE = 0, 1, 2
EST_FEATURES, EST_HIDDEN, EST_MAX_TABLES = 1792, 256, 12

WORKLOAD_ABI = {
    "bjw_workload_create": (_INT, [ctypes.c_char_p, _U64, ctypes.c_double, ctypes.POINTER(_VP)]),
    "bjw_workload_create_queries": (_INT, [ctypes.c_char_p, _U64, ctypes.c_double, _U64, ctypes.POINTER(_VP)]),
    "bjw_workload_base_rows": (_U64, [_VP, _U64]),
    "bjw_workload_load": (_INT, [ctypes.c_char_p, ctypes.POINTER(_VP)]),
    "bjw_workload_plan": (ctypes.POINTER(BjPlan), [_VP]),
    "bjw_workload_scan_bytes": (_U64, [_VP]),
    "bjw_workload_variant": (ctypes.POINTER(BjPlan), [_VP, _INT]),
    "bjw_workload_num_queries": (_U64, [_VP]),
    "bjw_workload_query": (ctypes.POINTER(BjPlan), [_VP, _U64]),
    "bjw_workload_free": (None, [_VP]),
    "bjw_save_plan": (_INT, [ctypes.c_char_p, ctypes.POINTER(BjPlan)]),
    "bjw_save_table": (_INT, [ctypes.c_char_p, ctypes.POINTER(BjTable)]),
    "bjw_encode_column": (_INT, [_I32, _U64, _VP, _VP, _VP, _VP, ctypes.POINTER(_VP)]),
    "bjw_pages_count": (_U64, [_VP]),
    "bjw_pages_ptrs": (ctypes.POINTER(_VP), [_VP]),
    "bjw_pages_free": (None, [_VP]),
}

_lib = None
_wlib = None


def _bind(lib, table):
    for name, (res, args) in table.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def library_path() -> str:
    return os.path.join(_HERE, "libb200join.so")


def lib():
    """The engine library (libb200join.so); raises if it has not been built."""
    global _lib
    if _lib is None:
        path = library_path()
        if not os.path.exists(path):
            raise EngineError(6, f"{path} is missing: run `make -C {_HERE}` (or __graft_entry__.build())")
        _lib = _bind(ctypes.CDLL(path), ABI)
    return _lib


def wlib():
    """The workload/encoder library (libb200join_workloads.so)."""
    global _wlib
    if _wlib is None:
        path = os.path.join(_HERE, "libb200join_workloads.so")
        if not os.path.exists(path):
            raise EngineError(6, f"{path} is missing: run `make -C {_HERE}`")
        _wlib = _bind(ctypes.CDLL(path), WORKLOAD_ABI)
    return _wlib


# ---------------------------------------------------------------------------
# Tables and pages

@dataclass
class Column:
    """A column of 8 KiB pages (mirrors the contest's Column)."""
    type: int
    data: bytes = b""  # num_pages * PAGE_SIZE bytes

    @property
    def num_pages(self) -> int:
        return len(self.data) // PAGE_SIZE

    def page(self, i: int) -> bytes:
        return self.data[i * PAGE_SIZE:(i + 1) * PAGE_SIZE]


@dataclass
class ColumnarTable:
    num_rows: int = 0
    columns: List[Column] = field(default_factory=list)


def encode_column(dtype: int, values: Sequence) -> Column:
    """Encodes Python values (None = NULL) into pages with the contest's
    packing rules (C++ encoder in libb200join_workloads.so)."""
    n = len(values)
    valid = (ctypes.c_uint8 * max(n, 1))(*[0 if v is None else 1 for v in values]) if n else None
    out = ctypes.c_void_p()
    if dtype == VARCHAR:
        blobs = [b"" if v is None else (v.encode() if isinstance(v, str) else bytes(v)) for v in values]
        offs = [0]
        for b in blobs:
            offs.append(offs[-1] + len(b))
        joined = b"".join(blobs)
        off_arr = (ctypes.c_uint64 * (n + 1))(*offs)
        byte_buf = ctypes.create_string_buffer(joined, max(len(joined), 1))
        st = wlib().bjw_encode_column(dtype, n, None, valid, off_arr, byte_buf, ctypes.byref(out))
    else:
        ctype = {INT32: ctypes.c_int32, INT64: ctypes.c_int64, FP64: ctypes.c_double}[dtype]
        arr = (ctype * max(n, 1))(*[0 if v is None else v for v in values])
        st = wlib().bjw_encode_column(dtype, n, arr, valid, None, None, ctypes.byref(out))
    if st != 0:
        raise EngineError(st, "encode_column failed")
    try:
        cnt = wlib().bjw_pages_count(out)
        ptrs = wlib().bjw_pages_ptrs(out)
        data = b"".join(ctypes.string_at(ptrs[i], PAGE_SIZE) for i in range(cnt))
    finally:
        wlib().bjw_pages_free(out)
    return Column(dtype, data)


def table_from_rows(rows: Sequence[Sequence], types: Sequence[int]) -> ColumnarTable:
    """Row table -> ColumnarTable (the contest's Table::to_columnar)."""
    t = ColumnarTable(num_rows=len(rows))
    for c, ty in enumerate(types):
        t.columns.append(encode_column(ty, [r[c] for r in rows]))
    return t


def decode_column(col: Column) -> List:
    """Pages -> Python values (None = NULL); the contest's from_columnar."""
    out: List = []
    i = 0
    n = col.num_pages
    while i < n:
        pg = col.page(i)
        nrows, nv = struct.unpack_from("<HH", pg, 0)
        if col.type == VARCHAR and nrows == 0xFFFF:
            s = pg[4:4 + nv]
            while i + 1 < n and struct.unpack_from("<H", col.page(i + 1), 0)[0] == 0xFFFE:
                i += 1
                q = col.page(i)
                s += q[4:4 + struct.unpack_from("<H", q, 2)[0]]
            out.append(s.decode("latin-1"))
            i += 1
            continue
        bm = pg[PAGE_SIZE - (nrows + 7) // 8:]
        dense = 0
        if col.type == VARCHAR:
            offs = struct.unpack_from(f"<{nv}H", pg, 4) if nv else ()
            base = 4 + 2 * nv
        for r in range(nrows):
            if not (bm[r >> 3] >> (r & 7)) & 1:
                out.append(None)
                continue
            if col.type == INT32:
                out.append(struct.unpack_from("<i", pg, 4 + 4 * dense)[0])
            elif col.type == INT64:
                out.append(struct.unpack_from("<q", pg, 8 + 8 * dense)[0])
            elif col.type == FP64:
                out.append(struct.unpack_from("<d", pg, 8 + 8 * dense)[0])
            else:
                b = offs[dense - 1] if dense else 0
                out.append(pg[base + b:base + offs[dense]].decode("latin-1"))
            dense += 1
        i += 1
    return out


def rows_of(table: ColumnarTable) -> List[Tuple]:
    """ColumnarTable -> list of row tuples (the contest's Table::from_columnar)."""
    cols = [decode_column(c) for c in table.columns]
    for c in cols:
        if len(c) != table.num_rows:
            raise ValueError(f"column holds {len(c)} rows, table says {table.num_rows}")
    return list(zip(*cols)) if cols else [()] * table.num_rows


# ---------------------------------------------------------------------------
# Plans

@dataclass
class PlanNode:
    kind: int
    output_attrs: List[Tuple[int, int]]
    base_table_id: int = 0
    build_left: bool = True
    left: int = 0
    right: int = 0
    left_attr: int = 0
    right_attr: int = 0


class Plan:
    """Mirrors the contest's Plan (plan.h:112-149)."""

    def __init__(self):
        self.nodes: List[PlanNode] = []
        self.inputs: List[ColumnarTable] = []
        self.root = 0

    def new_scan_node(self, base_table_id: int, output_attrs: Iterable[Tuple[int, int]]) -> int:
        self.nodes.append(PlanNode(NODE_SCAN, list(output_attrs), base_table_id=base_table_id))
        return len(self.nodes) - 1

    def new_join_node(self, build_left: bool, left: int, right: int, left_attr: int, right_attr: int,
                      output_attrs: Iterable[Tuple[int, int]]) -> int:
        self.nodes.append(PlanNode(NODE_JOIN, list(output_attrs), build_left=build_left, left=left, right=right,
                                   left_attr=left_attr, right_attr=right_attr))
        return len(self.nodes) - 1

    def new_input(self, table: ColumnarTable) -> int:
        self.inputs.append(table)
        return len(self.inputs) - 1


class CPlan:
    """A bj_plan built from a Python Plan; keeps every buffer alive."""

    def __init__(self, plan: Plan):
        self._keep = []
        tables = (BjTable * max(len(plan.inputs), 1))()
        for i, t in enumerate(plan.inputs):
            cols = (BjColumn * max(len(t.columns), 1))()
            for c, col in enumerate(t.columns):
                buf = ctypes.create_string_buffer(col.data, max(len(col.data), 1))
                ptrs = (ctypes.c_void_p * max(col.num_pages, 1))(
                    *[ctypes.addressof(buf) + k * PAGE_SIZE for k in range(col.num_pages)])
                self._keep += [buf, ptrs]
                cols[c].type = col.type
                cols[c].num_pages = col.num_pages
                cols[c].pages = ctypes.cast(ptrs, ctypes.POINTER(ctypes.c_void_p))
            self._keep.append(cols)
            tables[i].num_rows = t.num_rows
            tables[i].num_columns = len(t.columns)
            tables[i].columns = ctypes.cast(cols, ctypes.POINTER(BjColumn))
        nodes = (BjNode * max(len(plan.nodes), 1))()
        for n, pn in enumerate(plan.nodes):
            attrs = (BjAttr * max(len(pn.output_attrs), 1))()
            for a, (idx, ty) in enumerate(pn.output_attrs):
                attrs[a].index = idx
                attrs[a].type = ty
            self._keep.append(attrs)
            nodes[n].kind = pn.kind
            nodes[n].build_left = int(pn.build_left)
            nodes[n].base_table_id = pn.base_table_id
            nodes[n].left, nodes[n].right = pn.left, pn.right
            nodes[n].left_attr, nodes[n].right_attr = pn.left_attr, pn.right_attr
            nodes[n].num_output_attrs = len(pn.output_attrs)
            nodes[n].output_attrs = ctypes.cast(attrs, ctypes.POINTER(BjAttr))
        self._keep += [tables, nodes]
        self.struct = BjPlan(len(plan.nodes), ctypes.cast(nodes, ctypes.POINTER(BjNode)), len(plan.inputs),
                             ctypes.cast(tables, ctypes.POINTER(BjTable)), plan.root)

    def ref(self):
        return ctypes.byref(self.struct)


def save_plan(path: str, plan) -> None:
    """Writes a plan (Plan, CPlan or POINTER(BjPlan)) in the engine's plan file format."""
    if isinstance(plan, Plan):
        plan = CPlan(plan)
    p = plan.ref() if isinstance(plan, CPlan) else plan
    st = wlib().bjw_save_plan(path.encode(), p)
    if st != 0:
        raise EngineError(st, f"cannot write {path}")


def read_table_file(path: str) -> ColumnarTable:
    """Reads a result table file ("BJTABL01", include/contest/plan_io.h)."""
    with open(path, "rb") as f:
        data = f.read()
    if data[:8] != b"BJTABL01":
        raise ValueError(f"{path}: not a table file")
    nrows, ncols = struct.unpack_from("<QQ", data, 8)
    off = 24
    t = ColumnarTable(num_rows=nrows)
    for _ in range(ncols):
        ty, _pad, npg = struct.unpack_from("<iIQ", data, off)
        off += 16
        t.columns.append(Column(ty, data[off:off + npg * PAGE_SIZE]))
        off += npg * PAGE_SIZE
    return t


class Workload:
    """A seeded synthetic workload built by libb200join_workloads.so."""

    def __init__(self, name: str, seed: int, scale: float = 1.0, path: Optional[str] = None,
                 queries: Optional[int] = None):
        h = ctypes.c_void_p()
        if path:
            st = wlib().bjw_workload_load(path.encode(), ctypes.byref(h))
        elif queries is not None:
            st = wlib().bjw_workload_create_queries(name.encode(), seed, scale, queries, ctypes.byref(h))
        else:
            st = wlib().bjw_workload_create(name.encode(), seed, scale, ctypes.byref(h))
        if st != 0:
            raise EngineError(st, f"cannot build workload {name}")
        self.handle = h
        self.name, self.seed, self.scale = name, seed, scale

    def plan_ptr(self):
        return wlib().bjw_workload_plan(self.handle)

    def scan_bytes(self) -> int:
        return wlib().bjw_workload_scan_bytes(self.handle)

    def base_rows(self, table: int) -> int:
        """Rows of input `table` before its load-time filter (schema20)."""
        return wlib().bjw_workload_base_rows(self.handle, table)

    def num_queries(self) -> int:
        return wlib().bjw_workload_num_queries(self.handle)

    def query_ptr(self, k: int):
        """Query k of a batched workload ("schema20": 256 queries over shared
        tables; query 0 is plan_ptr())."""
        p = wlib().bjw_workload_query(self.handle, k)
        if not p:
            raise EngineError(1, f"{self.name} has no query {k}")
        return p

    def variant_ptr(self, dims: int):
        """Snowflake: the fact joined with its first `dims` dimensions (its
        inputs are the workload's first dims + 1 tables)."""
        p = wlib().bjw_workload_variant(self.handle, dims)
        if not p:
            raise EngineError(1, f"no {dims}-dimension variant of {self.name}")
        return p

    def close(self):
        if self.handle:
            wlib().bjw_workload_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Engine


class Result:
    """A bj_result: rows, per-column pages (host or device), stats."""

    def __init__(self, ctx: "Context", handle):
        self._ctx = ctx
        self.handle = handle

    def _check(self, st: int, what: str):
        if st != 0:
            msg = lib().bj_last_error(self._ctx.handle).decode() if self._ctx else "see the server's worker context"
            raise EngineError(st, f"{what}: {msg}")

    @property
    def num_rows(self) -> int:
        return lib().bj_result_num_rows(self.handle)

    @property
    def num_columns(self) -> int:
        return lib().bj_result_num_columns(self.handle)

    def column_type(self, c: int) -> int:
        return lib().bj_result_column_type(self.handle, c)

    def column_pages(self, c: int) -> int:
        return lib().bj_result_column_num_pages(self.handle, c)

    def wait(self) -> None:
        """Completes a RESULT_ASYNC result; raises if its device checks failed."""
        self._check(lib().bj_result_wait(self.handle), "bj_result_wait")

    def stats(self) -> BjStats:
        s = BjStats()
        self._check(lib().bj_result_stats(self.handle, ctypes.byref(s)), "bj_result_stats")
        return s

    def to_table(self) -> ColumnarTable:
        t = ColumnarTable(num_rows=self.num_rows)
        for c in range(self.num_columns):
            n = self.column_pages(c)
            bufs = (ctypes.c_char * (max(n, 1) * PAGE_SIZE))()
            ptrs = (ctypes.c_void_p * max(n, 1))(*[ctypes.addressof(bufs) + k * PAGE_SIZE for k in range(n)])
            st = lib().bj_result_copy_pages(self.handle, c, ptrs)
            if st != 0:
                raise EngineError(st, "bj_result_copy_pages failed")
            t.columns.append(Column(self.column_type(c), bytes(bufs)[:n * PAGE_SIZE]))
        return t

    def table_struct(self):
        """A BjTable view of the host pages (valid while this result lives)."""
        cols = (BjColumn * max(self.num_columns, 1))()
        keep = [cols]
        for c in range(self.num_columns):
            n = self.column_pages(c)
            ptrs = (ctypes.c_void_p * max(n, 1))(*[lib().bj_result_page(self.handle, c, k) for k in range(n)])
            keep.append(ptrs)
            cols[c].type = self.column_type(c)
            cols[c].num_pages = n
            cols[c].pages = ctypes.cast(ptrs, ctypes.POINTER(ctypes.c_void_p))
        t = BjTable(self.num_rows, self.num_columns, ctypes.cast(cols, ctypes.POINTER(BjColumn)))
        return t, keep

    def free(self):
        if self.handle:
            lib().bj_result_free(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.free()


class Resident:
    def __init__(self, ctx: "Context", handle):
        self._ctx, self.handle = ctx, handle

    def set_base_rows(self, base_rows: int) -> None:
        """Rows before the load-time filter (the estimator's selectivity feature)."""
        lib().bj_resident_set_base_rows(self.handle, base_rows)

    def free(self):
        if self.handle:
            lib().bj_resident_free(self._ctx.handle, self.handle)
            self.handle = None


class Context:
    """Contest::build_context / execute / destroy_context over the C ABI."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        st = lib().bj_context_create(device, ctypes.byref(h))
        if st != 0:
            raise EngineError(st, "bj_context_create failed (is a CUDA device visible?)")
        self.handle = h

    def _check(self, st: int, what: str):
        if st != 0:
            raise EngineError(st, f"{what}: {lib().bj_last_error(self.handle).decode()}")

    def execute_raw(self, plan) -> Result:
        """Runs a CPlan / POINTER(BjPlan); returns the Result handle."""
        p = plan.ref() if isinstance(plan, CPlan) else plan
        r = ctypes.c_void_p()
        self._check(lib().bj_execute(self.handle, p, ctypes.byref(r)), "bj_execute")
        return Result(self, r)

    def execute(self, plan: Plan) -> ColumnarTable:
        """Contest::execute: returns the result as a ColumnarTable."""
        with self.execute_raw(CPlan(plan)) as r:
            return r.to_table()

    def upload(self, table_struct) -> Resident:
        r = ctypes.c_void_p()
        self._check(lib().bj_resident_upload(self.handle, ctypes.byref(table_struct), ctypes.byref(r)),
                    "bj_resident_upload")
        return Resident(self, r)

    def save_resident(self, resident: Resident, path: str) -> None:
        self._check(lib().bj_resident_save(self.handle, resident.handle, path.encode()), "bj_resident_save")

    def load_resident(self, path: str) -> Resident:
        r = ctypes.c_void_p()
        self._check(lib().bj_resident_load(self.handle, path.encode(), ctypes.byref(r)), "bj_resident_load")
        return Resident(self, r)

    def execute_resident(self, plan, residents: Sequence[Resident], flags: int = RESULT_HOST) -> Result:
        p = plan.ref() if isinstance(plan, CPlan) else plan
        arr = (ctypes.c_void_p * max(len(residents), 1))(*[x.handle for x in residents])
        r = ctypes.c_void_p()
        self._check(lib().bj_execute_resident(self.handle, p, arr, flags, ctypes.byref(r)), "bj_execute_resident")
        return Result(self, r)

    def stream(self) -> int:
        return lib().bj_context_stream(self.handle) or 0

    def set_ordering(self, mode: int, estimator: Optional["Estimator"] = None) -> None:
        """Join ordering of resident queries: ORDER_ROWS, ORDER_SAMPLING or
        ORDER_LEARNED (with an estimator; sampling is its fallback)."""
        self._check(lib().bj_context_set_ordering(self.handle, mode, estimator.handle if estimator else None),
                    "bj_context_set_ordering")

    def _subplan_call(self, fn, plan, residents, masks, out, what):
        import numpy as np
        m = np.ascontiguousarray(masks, dtype=np.uint32)
        arr = (ctypes.c_void_p * max(len(residents), 1))(*[x.handle for x in residents])
        p = plan.ref() if isinstance(plan, CPlan) else plan
        self._check(fn(self.handle, p, arr, m.ctypes.data, len(m), out.ctypes.data), what)
        return out

    def scratch_estimate(self, plan, residents) -> int:
        """Estimated device scratch of a resident plan (bj_plan_scratch_estimate)."""
        arr = (ctypes.c_void_p * max(len(residents), 1))(*[x.handle for x in residents])
        p = plan.ref() if isinstance(plan, CPlan) else plan
        out = ctypes.c_uint64()
        self._check(lib().bj_plan_scratch_estimate(self.handle, p, arr, ctypes.byref(out)), "bj_plan_scratch_estimate")
        return out.value

    def set_graphs(self, on: bool) -> None:
        lib().bj_context_set_graphs(self.handle, 1 if on else 0)

    def set_plan_space(self, space: int) -> None:
        """PLAN_AUTO (the cheaper), PLAN_ROOTED or PLAN_REFERENCE."""
        self._check(lib().bj_context_set_plan_space(self.handle, space), "bj_context_set_plan_space")

    def autotune(self, plan, residents, repeats: int = 5) -> str:
        """Tunes build and scan parameters for the plan's shape class
        (bj_context_autotune); returns the report."""
        arr = (ctypes.c_void_p * max(len(residents), 1))(*[x.handle for x in residents])
        p = plan.ref() if isinstance(plan, CPlan) else plan
        buf = ctypes.create_string_buffer(8192)
        n = ctypes.c_uint64()
        self._check(lib().bj_context_autotune(self.handle, p, arr, repeats, buf, 8192, ctypes.byref(n)),
                    "bj_context_autotune")
        return buf.value.decode()

    def subplan_cards(self, plan, residents, masks):
        """Exact cardinality of each sub-plan (device counts)."""
        import numpy as np
        return self._subplan_call(lib().bj_subplan_cards, plan, residents, masks,
                                  np.zeros(len(masks), dtype=np.float64), "bj_subplan_cards")

    def subplan_sample_cards(self, plan, residents, masks):
        import numpy as np
        return self._subplan_call(lib().bj_subplan_sample_cards, plan, residents, masks,
                                  np.zeros(len(masks), dtype=np.float64), "bj_subplan_sample_cards")

    def subplan_features(self, plan, residents, masks):
        import numpy as np
        return self._subplan_call(lib().bj_subplan_features, plan, residents, masks,
                                  np.zeros((len(masks), EST_FEATURES), dtype=np.float32), "bj_subplan_features")

    def profile(self, on: bool) -> None:
        lib().bj_context_profile(self.handle, 1 if on else 0)

    def close(self):
        if self.handle:
            lib().bj_context_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def subplans(plan, max_tables: int = EST_MAX_TABLES):
    """Connected input sets of a plan (bit masks over its scans in depth-first
    order, left child first), ascending."""
    import numpy as np
    p = plan.ref() if isinstance(plan, CPlan) else plan
    n = ctypes.c_uint64()
    st = lib().bj_subplans(p, max_tables, 0, None, ctypes.byref(n))
    if st != 0:
        raise EngineError(st, "bj_subplans")
    out = np.zeros(max(n.value, 1), dtype=np.uint32)
    st = lib().bj_subplans(p, max_tables, n.value, out.ctypes.data, ctypes.byref(n))
    if st != 0:
        raise EngineError(st, "bj_subplans")
    return out[:n.value]


def join_order(plan, cards=None, driver: int = -1):
    """(driver, cost) of the executor's cheapest plan under set cardinalities
    cards[mask] (None: the row-count model); driver >= 0 costs that driver."""
    import numpy as np
    p = plan.ref() if isinstance(plan, CPlan) else plan
    c = None if cards is None else np.ascontiguousarray(cards, dtype=np.float64)
    d, cost = ctypes.c_uint32(), ctypes.c_double()
    st = lib().bj_join_order(p, None if c is None else c.ctypes.data, driver, ctypes.byref(d), ctypes.byref(cost))
    if st != 0:
        raise EngineError(st, "bj_join_order")
    return d.value, cost.value


class Estimator:
    """The learned cardinality estimator (bj_estimator_*): a BF16 MLP trained
    and run on the device by the library's own kernels."""

    def __init__(self, device: int = 0, seed: int = 0, path: Optional[str] = None):
        h = ctypes.c_void_p()
        if path:
            st = lib().bj_estimator_load(device, path.encode(), ctypes.byref(h))
        else:
            st = lib().bj_estimator_create(device, seed, ctypes.byref(h))
        if st != 0:
            raise EngineError(st, "cannot create the estimator")
        self.handle = h

    @staticmethod
    def num_params() -> int:
        return lib().bj_estimator_num_params()

    def params(self):
        import numpy as np
        out = np.zeros(self.num_params(), dtype=np.float32)
        st = lib().bj_estimator_get_params(self.handle, out.ctypes.data)
        if st != 0:
            raise EngineError(st, "bj_estimator_get_params")
        return out

    def set_params(self, p) -> None:
        import numpy as np
        a = np.ascontiguousarray(p, dtype=np.float32)
        assert a.size == self.num_params()
        st = lib().bj_estimator_set_params(self.handle, a.ctypes.data)
        if st != 0:
            raise EngineError(st, "bj_estimator_set_params")

    def train(self, features, targets, epochs: int = 30, batch: int = 256, lr: float = 1e-3, seed: int = 0):
        import numpy as np
        f = np.ascontiguousarray(features, dtype=np.float32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        losses = np.zeros(epochs, dtype=np.float32)
        st = lib().bj_estimator_train(self.handle, f.ctypes.data, t.ctypes.data, len(t), epochs, batch, lr, seed,
                                      losses.ctypes.data)
        if st != 0:
            raise EngineError(st, "bj_estimator_train")
        return losses

    def predict(self, features):
        import numpy as np
        f = np.ascontiguousarray(features, dtype=np.float32)
        out = np.zeros(len(f), dtype=np.float32)
        st = lib().bj_estimator_predict(self.handle, f.ctypes.data, len(f), out.ctypes.data)
        if st != 0:
            raise EngineError(st, "bj_estimator_predict")
        return out

    def gradients(self, features, targets):
        import numpy as np
        f = np.ascontiguousarray(features, dtype=np.float32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        g = np.zeros(self.num_params(), dtype=np.float32)
        st = lib().bj_estimator_gradients(self.handle, f.ctypes.data, t.ctypes.data, len(t), loss.ctypes.data,
                                          g.ctypes.data)
        if st != 0:
            raise EngineError(st, "bj_estimator_gradients")
        return float(loss[0]), g

    def save(self, path: str) -> None:
        st = lib().bj_estimator_save(self.handle, path.encode())
        if st != 0:
            raise EngineError(st, "bj_estimator_save")

    def close(self):
        if self.handle:
            lib().bj_estimator_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def q_error(est, true):
    """max(est / true, true / est) with both floored at 1 (the usual q-error)."""
    import numpy as np
    e = np.maximum(np.asarray(est, dtype=np.float64), 1.0)
    t = np.maximum(np.asarray(true, dtype=np.float64), 1.0)
    return np.maximum(e / t, t / e)


def subplan_corpus(ctx: "Context", workload: "Workload", residents, queries, max_per_query: int = 256, seed: int = 0,
                   with_features: bool = True):
    """Sub-plans of the given queries of a batched workload over its resident
    tables, labelled with their exact cardinalities (device counts): returns a
    dict of arrays `features` (n x EST_FEATURES; absent without
    with_features), `card` (exact), `sample` (sampling estimates), `query`,
    `mask`. A query with more than max_per_query sub-plans of two or more
    inputs contributes a seeded random choice of them."""
    import numpy as np
    rng = np.random.default_rng(seed)
    feats, cards, samples, qids, masks = [], [], [], [], []
    for k in queries:
        plan = workload.query_ptr(k)
        m = subplans(plan, EST_MAX_TABLES)
        m = m[[bin(int(x)).count("1") >= 2 for x in m]]
        if len(m) > max_per_query:
            m = np.sort(rng.choice(m, max_per_query, replace=False))
        if len(m) == 0:
            continue
        cards.append(ctx.subplan_cards(plan, residents, m))
        samples.append(ctx.subplan_sample_cards(plan, residents, m))
        if with_features:
            feats.append(ctx.subplan_features(plan, residents, m))
        qids.append(np.full(len(m), k, dtype=np.int64))
        masks.append(m)
    card = np.concatenate(cards)
    # A count past 2^64 - 1 comes back infinite; as a label it is 2^64.
    card = np.where(np.isfinite(card), card, 2.0 ** 64)
    out = {"card": card, "sample": np.concatenate(samples), "query": np.concatenate(qids),
           "mask": np.concatenate(masks)}
    if with_features:
        out["features"] = np.concatenate(feats)
    return out


def set_cards_of(ctx: "Context", plan, residents, mode: int, estimator: Optional["Estimator"] = None):
    """Set cardinalities of every connected input set of a plan, as an array
    over input masks (2^scans entries): exact device counts (mode None), join
    samples (ORDER_SAMPLING) or the learned estimator (ORDER_LEARNED; sets of
    one input keep their row counts, as in the engine)."""
    import numpy as np
    masks = subplans(plan, 32)
    n = max(int(m).bit_length() for m in masks)
    cards = np.zeros(1 << n, dtype=np.float64)
    if mode is None:
        vals = ctx.subplan_cards(plan, residents, masks)
    else:
        vals = ctx.subplan_sample_cards(plan, residents, masks)
        if mode == ORDER_LEARNED:
            multi = np.array([bin(int(m)).count("1") > 1 for m in masks])
            if multi.any():
                f = ctx.subplan_features(plan, residents, masks[multi])
                vals = vals.copy()
                vals[multi] = np.maximum(np.exp2(estimator.predict(f).astype(np.float64)) - 1.0, 0.0)
    cards[masks] = vals
    return cards


class ServerResident:
    """A resident table shared by a server's workers."""

    def __init__(self, server: "Server", handle):
        self._server, self.handle = server, handle

    def set_base_rows(self, base_rows: int) -> None:
        lib().bj_resident_set_base_rows(self.handle, base_rows)

    def free(self):
        if self.handle:
            lib().bj_server_resident_free(self._server.handle, self.handle)
            self.handle = None


class Server:
    """Concurrent queries over resident tables (bj_server_*): `workers`
    contexts on one device, admission by estimated device scratch."""

    def __init__(self, device: int = 0, workers: int = 4, scratch_cap_bytes: int = 0):
        h = ctypes.c_void_p()
        st = lib().bj_server_create(device, workers, scratch_cap_bytes, ctypes.byref(h))
        if st != 0:
            raise EngineError(st, "bj_server_create failed")
        self.handle = h
        self._plans = {}

    def upload(self, table_struct) -> ServerResident:
        ctx0 = lib().bj_server_context(self.handle, 0)
        r = ctypes.c_void_p()
        st = lib().bj_resident_upload(ctx0, table_struct, ctypes.byref(r))
        if st != 0:
            raise EngineError(st, "bj_resident_upload failed")
        return ServerResident(self, r)

    def submit(self, plan_ptr, residents: Sequence[ServerResident], flags: int = RESULT_DEVICE) -> int:
        arr = (ctypes.c_void_p * len(residents))(*[x.handle for x in residents])
        t = ctypes.c_uint64()
        st = lib().bj_server_submit(self.handle, plan_ptr, arr, flags, ctypes.byref(t))
        if st != 0:
            raise EngineError(st, "bj_server_submit failed")
        self._plans[t.value] = arr  # the table array must outlive the query
        return t.value

    def set_ordering(self, mode: int, estimator: Optional["Estimator"] = None) -> None:
        st = lib().bj_server_set_ordering(self.handle, mode, estimator.handle if estimator else None)
        if st != 0:
            raise EngineError(st, "bj_server_set_ordering failed")

    def set_graphs(self, on: bool) -> None:
        lib().bj_server_set_graphs(self.handle, 1 if on else 0)

    def run_load(self, plan_ptrs, residents: Sequence[ServerResident], seq, rate_qps: float = 0.0,
                 window: int = 16, seed: int = 0):
        """The C++ load generator (bj_server_run_load): queries plan_ptrs[seq[i]]
        as a Poisson stream of rate_qps (closed loop of `window` outstanding
        queries when rate_qps <= 0). Returns (latencies in ms, elapsed seconds,
        summed result rows)."""
        import numpy as np
        plans = (ctypes.c_void_p * len(plan_ptrs))(*[ctypes.cast(p, ctypes.c_void_p).value for p in plan_ptrs])
        arr = (ctypes.c_void_p * len(residents))(*[x.handle for x in residents])
        sq = np.ascontiguousarray(seq, dtype=np.uint32)
        lat = np.zeros(max(len(sq), 1), dtype=np.float64)
        el = ctypes.c_double()
        rows = ctypes.c_uint64()
        st = lib().bj_server_run_load(self.handle, plans, len(plan_ptrs), arr, sq.ctypes.data, len(sq), rate_qps,
                                      window, seed, lat.ctypes.data, ctypes.byref(el), ctypes.byref(rows))
        if st != 0:
            raise EngineError(st, "bj_server_run_load: a query failed")
        return lat[:len(sq)], el.value, rows.value

    def wait(self, ticket: int):
        """(Result, latency in ms) of a submitted query."""
        r = ctypes.c_void_p()
        ms = ctypes.c_double()
        st = lib().bj_server_wait(self.handle, ticket, ctypes.byref(r), ctypes.byref(ms))
        self._plans.pop(ticket, None)
        if st != 0:
            raise EngineError(st, "query failed")
        return Result(None, r), ms.value

    def close(self):
        if self.handle:
            lib().bj_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def explain(plan) -> str:
    """The pipelines the engine runs for `plan` (Plan, CPlan or POINTER(BjPlan)):
    the driver and the plan's estimated cost, then one line per pipeline.
    Needs no GPU."""
    if isinstance(plan, Plan):
        plan = CPlan(plan)
    p = plan.ref() if isinstance(plan, CPlan) else plan
    n = ctypes.c_uint64(0)
    st = lib().bj_plan_explain(p, None, 0, ctypes.byref(n))
    if st != 0:
        raise EngineError(st, "bj_plan_explain failed")
    buf = ctypes.create_string_buffer(n.value + 1)
    st = lib().bj_plan_explain(p, buf, n.value + 1, ctypes.byref(n))
    if st != 0:
        raise EngineError(st, "bj_plan_explain failed")
    return buf.value.decode()


def build_context(device: int = 0) -> Context:
    return Context(device)


def destroy_context(ctx: Context) -> None:
    ctx.close()


def execute(plan: Plan, ctx: Context) -> ColumnarTable:
    return ctx.execute(plan)
