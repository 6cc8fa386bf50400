"""ctypes binding of the CPU oracle (oracle/liboracle.so) -- test infrastructure.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use the
oracle, and only as the checker.
"""
import ctypes
import os
import subprocess

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(REPO, "oracle", "liboracle.so")
REF_RUNNER = os.path.join(REPO, "oracle", "_ref", "ref_runner")

_VP = ctypes.c_void_p


class Oracle:
    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), "oracle"], check=True, capture_output=True)
        L = ctypes.CDLL(ORACLE_SO)
        L.oracle_execute.argtypes = [_VP, ctypes.POINTER(_VP), ctypes.c_char_p, ctypes.c_uint64]
        L.oracle_table_view.restype = _VP
        L.oracle_table_view.argtypes = [_VP]
        L.oracle_table_free.argtypes = [_VP]
        L.oracle_validate_table.argtypes = [_VP, ctypes.c_char_p, ctypes.c_uint64]
        L.oracle_rows_from_table.argtypes = [_VP, ctypes.POINTER(_VP), ctypes.c_char_p, ctypes.c_uint64]
        L.oracle_rows_count.restype = ctypes.c_uint64
        L.oracle_rows_count.argtypes = [_VP]
        L.oracle_rows_equal.argtypes = [_VP, _VP, ctypes.POINTER(ctypes.c_uint64)]
        L.oracle_rows_digest.argtypes = [_VP, ctypes.POINTER(ctypes.c_uint64)]
        L.oracle_rows_format.argtypes = [_VP, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_uint64]
        L.oracle_rows_free.argtypes = [_VP]
        self.L = L

    def execute(self, plan_ptr):
        """Runs a plan (ctypes pointer to BjPlan) on the CPU; returns an OracleTable."""
        h = _VP()
        err = ctypes.create_string_buffer(1024)
        st = self.L.oracle_execute(ctypes.cast(plan_ptr, _VP), ctypes.byref(h), err, 1024)
        if st != 0:
            raise RuntimeError("oracle: " + err.value.decode())
        return OracleTable(self, h)

    def validate(self, table_ptr):
        err = ctypes.create_string_buffer(1024)
        if self.L.oracle_validate_table(ctypes.cast(table_ptr, _VP), err, 1024) != 0:
            return err.value.decode()
        return None

    def rows(self, table_ptr):
        h = _VP()
        err = ctypes.create_string_buffer(1024)
        st = self.L.oracle_rows_from_table(ctypes.cast(table_ptr, _VP), ctypes.byref(h), err, 1024)
        if st != 0:
            raise RuntimeError("oracle rows: " + err.value.decode())
        return Rows(self, h)


class OracleTable:
    def __init__(self, o, h):
        self.o, self.h = o, h

    def view(self):
        return self.o.L.oracle_table_view(self.h)

    def __del__(self):
        if self.h:
            self.o.L.oracle_table_free(self.h)
            self.h = None


class Rows:
    def __init__(self, o, h):
        self.o, self.h = o, h

    def __len__(self):
        return self.o.L.oracle_rows_count(self.h)

    def equals(self, other):
        d = ctypes.c_uint64()
        ok = self.o.L.oracle_rows_equal(self.h, other.h, ctypes.byref(d))
        return bool(ok), d.value

    def digest(self):
        out = (ctypes.c_uint64 * 3)()
        self.o.L.oracle_rows_digest(self.h, out)
        return tuple(out)

    def row(self, i):
        buf = ctypes.create_string_buffer(4096)
        self.o.L.oracle_rows_format(self.h, i, buf, 4096)
        return buf.value.decode("latin-1")

    def __del__(self):
        if self.h:
            self.o.L.oracle_rows_free(self.h)
            self.h = None


def assert_same_rows(oracle, got_table_ptr, want_table_ptr, label=""):
    """Exact row-multiset equality of two BjTable views, with a readable diff."""
    msg = oracle.validate(got_table_ptr)
    assert msg is None, f"{label}: result pages violate the format: {msg}"
    got = oracle.rows(got_table_ptr)
    want = oracle.rows(want_table_ptr)
    ok, pos = got.equals(want)
    if not ok:
        lines = [f"{label}: row multisets differ (got {len(got)} rows, want {len(want)}); first sorted diff at {pos}"]
        for i in range(max(0, pos - 2), min(pos + 3, max(len(got), len(want)))):
            g = got.row(i) if i < len(got) else "-"
            w = want.row(i) if i < len(want) else "-"
            lines.append(f"  [{i}] got {g}   want {w}")
        raise AssertionError("\n".join(lines))
    return len(got)
