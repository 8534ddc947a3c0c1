"""ctypes binding of the C ABI in include/voila_cuda.h.

The Python side mirrors the reference's query lifecycle: a Database of typed columns with
declared min/max (runtime::Database, db-engine-paradigms/include/common/runtime/Database.hpp:28-75),
a plan (relalg tree, relalg.hpp) and a query that is created with a flavor, run, reset and
freed (voila_query_new/run/reset/free, codegen.cpp:371-392).  Results come back as
QueryResult text rows "a|b|c" (runtime_framework.cpp:77-111) or as int64 columns.

There is no CPU execution path: without the compiled library or a B200 the calls fail.
"""
import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvoila_cuda.so")

VC_OK = 0
ERRORS = {1: "invalid", 2: "cuda", 3: "capacity", 4: "timeout", 5: "compile", 6: "unsupported", 7: "no device"}

TYPES = {"u8": 1, "i16": 2, "i32": 3, "i64": 4, "str": 5}
STR = 5
# host arrays per column type (strings: Python str objects; on the device they are codes)
NP_TYPES = {1: np.uint8, 2: np.int16, 3: np.int32, 4: np.int64, 5: object}
STR_WIDTH = 32  # rows of a host-generated string column (NUL-padded)

GEN_KINDS = {"uniform": 0, "seq": 1, "perm": 2, "zipf": 3, "choice": 4, "div": 5, "mod": 6, "words": 7}

_lib_handle = None


class VoilaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{ERRORS.get(code, code)}] {msg}")
        self.code = code


def lib():
    """Loads libvoila_cuda.so (built in-tree by python -m vldb_voila_b200.build)."""
    global _lib_handle
    if _lib_handle is not None:
        return _lib_handle
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m vldb_voila_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    c = ctypes
    P = c.c_void_p
    sigs = {
        "vc_last_error": (c.c_char_p, []),
        "vc_version": (c.c_char_p, []),
        "vc_engine_create": (c.c_int, [c.c_int, c.POINTER(P)]),
        "vc_engine_create_offline": (c.c_int, [c.c_int, c.POINTER(P)]),
        "vc_engine_destroy": (c.c_int, [P]),
        "vc_table_create": (c.c_int, [P, c.c_char_p, c.c_int64]),
        "vc_table_drop": (c.c_int, [P, c.c_char_p]),
        "vc_column_add": (c.c_int, [P, c.c_char_p, c.c_char_p, c.c_int, c.c_int64, c.c_int64]),
        "vc_column_upload": (c.c_int, [P, c.c_char_p, c.c_char_p, P, c.c_int64, P]),
        "vc_column_download": (c.c_int, [P, c.c_char_p, c.c_char_p, P, c.c_int64, P]),
        "vc_column_attach": (c.c_int, [P, c.c_char_p, c.c_char_p, P]),
        "vc_column_device_ptr": (c.c_int, [P, c.c_char_p, c.c_char_p, c.POINTER(P)]),
        "vc_column_generate": (c.c_int, [P, c.c_char_p, c.c_char_p, c.c_int32, c.c_int64, c.c_int64, c.c_int64,
                                         c.c_double, c.c_uint64, P, P]),
        "vc_gen_host": (c.c_int, [c.c_int32, c.c_int32, c.c_int64, c.c_int64, c.c_int64, c.c_double, c.c_uint64,
                                  c.c_int64, P, c.c_int64, c.c_int64, P]),
        "vc_gen_zipf_cdf": (c.c_int, [c.c_double, c.c_int64, P]),
        "vc_workload_describe": (c.c_int, [c.c_char_p, P, c.c_size_t, c.POINTER(c.c_size_t)]),
        "vc_workload_batch": (c.c_int, [c.c_int, c.c_uint64, c.c_int64, c.c_int64, P, c.c_size_t,
                                        c.POINTER(c.c_size_t)]),
        "vc_query_new": (c.c_int, [P, c.c_char_p, c.c_char_p, c.POINTER(P)]),
        "vc_query_run": (c.c_int, [P, P]),
        "vc_query_reset": (c.c_int, [P]),
        "vc_query_free": (c.c_int, [P]),
        "vc_query_result_shape": (c.c_int, [P, c.POINTER(c.c_int64), c.POINTER(c.c_int32)]),
        "vc_query_result_copy": (c.c_int, [P, P, c.c_int64]),
        "vc_query_result_text": (c.c_int, [P, P, c.c_size_t, c.POINTER(c.c_size_t)]),
        "vc_query_info": (c.c_int, [P, P, c.c_size_t, c.POINTER(c.c_size_t)]),
        "vc_query_source": (c.c_int, [P, P, c.c_size_t, c.POINTER(c.c_size_t)]),
        "vc_query_profile": (c.c_int, [P, c.c_int]),
        "vc_query_time": (c.c_int, [P, c.c_int, c.c_int, P, c.POINTER(c.c_float), c.c_int]),
        "vc_mlp_create": (c.c_int, [c.c_int, c.c_int, c.c_int, c.c_int, c.c_uint64, c.POINTER(P)]),
        "vc_mlp_free": (c.c_int, [P]),
        "vc_mlp_num_params": (c.c_int, [P, c.POINTER(c.c_int64)]),
        "vc_mlp_get_params": (c.c_int, [P, P, c.c_int64]),
        "vc_mlp_set_params": (c.c_int, [P, P, c.c_int64]),
        "vc_mlp_loss_grad": (c.c_int, [P, P, P, P, c.c_int, c.POINTER(c.c_float), P]),
        "vc_mlp_train": (c.c_int, [P, P, P, P, c.c_int, c.c_int, c.c_int, c.c_float, c.c_uint64,
                                   c.POINTER(c.c_float)]),
        "vc_mlp_predict": (c.c_int, [P, P, c.c_int, P]),
        "vc_batch_new": (c.c_int, [c.POINTER(P), c.c_int, c.POINTER(c.c_char_p), c.c_int, c.c_int64, c.POINTER(P)]),
        "vc_batch_new_split": (c.c_int, [c.POINTER(P), c.c_int, c.POINTER(c.c_char_p), c.c_int, c.c_int64, c.c_int64,
                                         c.POINTER(P)]),
        "vc_batch_run": (c.c_int, [P, P]),
        "vc_batch_wait": (c.c_int, [P]),
        "vc_batch_latencies": (c.c_int, [P, c.POINTER(c.c_double), c.c_int]),
        "vc_batch_info": (c.c_int, [P, P, c.c_size_t, c.POINTER(c.c_size_t)]),
        "vc_batch_source": (c.c_int, [P, P, c.c_size_t, c.POINTER(c.c_size_t)]),
        "vc_batch_items": (c.c_int, [P, P, c.c_int64, c.POINTER(c.c_int64)]),
        "vc_batch_free": (c.c_int, [P]),
        "vc_batch_set_wait_limit": (c.c_int, [P, c.c_uint64]),
        "vc_batch_hold_item": (c.c_int, [P, c.c_int64, c.c_int]),
        "vc_query_timings": (c.c_int, [P, c.POINTER(c.c_float), c.c_int, c.POINTER(c.c_int), P, c.c_size_t]),
        "vc_stream_read": (c.c_int, [P, c.c_int64, P, P]),
        "vc_plan_columns": (c.c_int, [c.c_char_p, P, c.c_size_t, c.POINTER(c.c_size_t)]),
        "vc_column_upload_strings": (c.c_int, [P, c.c_char_p, c.c_char_p, P, P, c.c_int64]),
        "vc_column_attach_host": (c.c_int, [P, c.c_char_p, c.c_char_p, P]),
        "vc_dict_size": (c.c_int, [P, c.POINTER(c.c_int64)]),
        "vc_dict_string": (c.c_int, [P, c.c_int64, P, c.c_size_t, c.POINTER(c.c_size_t)]),
        "vc_table_import": (c.c_int, [P, c.c_char_p, c.c_char_p, c.c_char_p, c.c_int, c.POINTER(c.c_int64)]),
        "vc_column_info": (c.c_int, [P, c.c_char_p, c.c_char_p, c.POINTER(c.c_int32), c.POINTER(c.c_int64),
                                     c.POINTER(c.c_int64), c.POINTER(c.c_int64)]),
        "vc_plan_describe": (c.c_int, [P, c.c_char_p, c.c_char_p, P, c.c_size_t, c.POINTER(c.c_size_t)]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib_handle = L
    return L


def check(rc):
    if rc != VC_OK:
        raise VoilaError(rc, lib().vc_last_error().decode())


def _b(s):
    return s.encode() if isinstance(s, str) else s


def _text_call(fn, *args):
    n = ctypes.c_size_t(0)
    check(fn(*args, None, 0, ctypes.byref(n)))
    buf = ctypes.create_string_buffer(n.value + 1)
    check(fn(*args, buf, n.value + 1, ctypes.byref(n)))
    return buf.raw[:n.value].decode()


def _stream_ptr(stream):
    """Accepts None, an int handle, or a torch.cuda.Stream."""
    if stream is None:
        return None
    if isinstance(stream, int):
        return ctypes.c_void_p(stream)
    return ctypes.c_void_p(int(stream.cuda_stream))


# ---------------------------------------------------------------------------- workloads


@dataclass
class ColumnSpec:
    table: str
    name: str
    type: int
    kind: int
    a: int
    b: int
    c: int
    s: float
    seed: int
    n: int
    lo: int
    hi: int

    @property
    def dtype(self):
        return NP_TYPES[self.type]


@dataclass
class Workload:
    spec: str
    template: str
    fact_table: str
    fact_rows: int
    algo_bytes: int
    probe_bytes: int
    tables: dict = field(default_factory=dict)     # name -> rows
    columns: list = field(default_factory=list)    # ColumnSpec
    plan: str = ""

    def table_columns(self, table):
        return [c for c in self.columns if c.table == table]


def workload(spec):
    """Tables, generators and plan of a synthetic workload spec (see csrc/workloads.hpp)."""
    text = _text_call(lib().vc_workload_describe, _b(spec))
    w = Workload(spec=spec, template="", fact_table="", fact_rows=0, algo_bytes=0, probe_bytes=0)
    for line in text.splitlines():
        tag, _, rest = line.partition(" ")
        if tag == "template":
            w.template = rest
        elif tag == "fact":
            t, n = rest.split()
            w.fact_table, w.fact_rows = t, int(n)
        elif tag == "bytes":
            a, p = rest.split()
            w.algo_bytes, w.probe_bytes = int(a), int(p)
        elif tag == "table":
            t, n = rest.split()
            w.tables[t] = int(n)
        elif tag == "column":
            f = rest.split()
            w.columns.append(ColumnSpec(f[0], f[1], int(f[2]), int(f[3]), int(f[4]), int(f[5]), int(f[6]),
                                        float(f[7]), int(f[8]), int(f[9]), int(f[10]), int(f[11])))
        elif tag == "plan":
            w.plan = rest
    return w


def plan_columns(plan):
    """[(table, column)] the plan scans."""
    return [tuple(l.split()) for l in _text_call(lib().vc_plan_columns, _b(plan)).splitlines() if l]


def batch_specs(count, seed, min_rows=10_000, max_rows=60_000_000):
    return _text_call(lib().vc_workload_batch, count, seed, min_rows, max_rows).split()


def stream_read(device_ptr, nbytes, device_out, stream=None):
    """One plain streaming read of nbytes at device_ptr (the bandwidth floor of a scan)."""
    check(lib().vc_stream_read(ctypes.c_void_p(device_ptr), nbytes, ctypes.c_void_p(device_out), _stream_ptr(stream)))


def zipf_cdf(s, n):
    out = np.empty(n, dtype=np.float64)
    check(lib().vc_gen_zipf_cdf(s, n, out.ctypes.data))
    return out


def generate_host(col, begin=0, count=None, cdf=None):
    """The column's values for rows [begin, begin+count), generated on the host."""
    count = col.n - begin if count is None else count
    if col.type == STR:
        raw = np.zeros(count * STR_WIDTH, dtype=np.uint8)
        check(lib().vc_gen_host(col.kind, col.type, col.a, col.b, col.c, col.s, col.seed, col.n, None, begin, count,
                                raw.ctypes.data))
        rows = raw.reshape(count, STR_WIDTH).view(f"S{STR_WIDTH}").reshape(count)
        return np.array([r.decode() for r in rows], dtype=object)
    out = np.empty(count, dtype=col.dtype)
    if col.kind == GEN_KINDS["zipf"] and col.s != 0.0 and cdf is None:
        cdf = zipf_cdf(col.s, col.b)
    check(lib().vc_gen_host(col.kind, col.type, col.a, col.b, col.c, col.s, col.seed, col.n,
                            None if cdf is None else cdf.ctypes.data, begin, count, out.ctypes.data))
    return out


def generate_workload_host(w):
    """{table: {column: ndarray}} for every column of the workload."""
    data = {t: {} for t in w.tables}
    cdfs = {}
    for c in w.columns:
        cdf = None
        if c.kind == GEN_KINDS["zipf"] and c.s != 0.0:
            key = (c.s, c.b)
            if key not in cdfs:
                cdfs[key] = zipf_cdf(c.s, c.b)
            cdf = cdfs[key]
        data[c.table][c.name] = generate_host(c, cdf=cdf)
    return data


# ---------------------------------------------------------------------------- engine


class Engine:
    """A device (or, with offline=True, a compile-only) database of columns in HBM."""

    def __init__(self, device=0, offline=False, sms=148):
        h = ctypes.c_void_p()
        if offline:
            check(lib().vc_engine_create_offline(sms, ctypes.byref(h)))
        else:
            check(lib().vc_engine_create(device, ctypes.byref(h)))
        self._h = h
        self.offline = offline
        self.tables = {}

    def close(self):
        if self._h:
            check(lib().vc_engine_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def create_table(self, name, rows):
        check(lib().vc_table_create(self._h, _b(name), rows))
        self.tables[name] = {"rows": rows, "columns": {}}

    def add_column(self, table, name, type_, lo, hi):
        t = TYPES[type_] if isinstance(type_, str) else type_
        check(lib().vc_column_add(self._h, _b(table), _b(name), t, int(lo), int(hi)))
        self.tables[table]["columns"][name] = t

    def upload(self, table, name, array, stream=None):
        t = self.tables[table]["columns"][name]
        if t == STR:
            return self.upload_strings(table, name, array)
        a = np.ascontiguousarray(array, dtype=NP_TYPES[t])
        check(lib().vc_column_upload(self._h, _b(table), _b(name), a.ctypes.data, len(a), _stream_ptr(stream)))
        return a

    def upload_strings(self, table, name, strings):
        """Uploads a string column (dictionary-encoded by the engine)."""
        enc = [x.encode() if isinstance(x, str) else bytes(x) for x in strings]
        offsets = np.zeros(len(enc) + 1, dtype=np.int64)
        offsets[1:] = np.cumsum([len(x) for x in enc]) if enc else []
        blob = b"".join(enc) or b"\0"
        check(lib().vc_column_upload_strings(self._h, _b(table), _b(name), blob, offsets.ctypes.data, len(enc)))
        return strings

    def dict_string(self, code):
        """String of a dictionary code (string result columns hold codes in Query.result())."""
        return _text_call(lambda *a: lib().vc_dict_string(self._h, int(code), *a))

    def upload_ptr(self, table, name, host_ptr, rows, stream=None):
        check(lib().vc_column_upload(self._h, _b(table), _b(name), ctypes.c_void_p(host_ptr), rows,
                                     _stream_ptr(stream)))

    def download(self, table, name):
        t = self.tables[table]["columns"][name]
        out = np.empty(self.tables[table]["rows"], dtype=NP_TYPES[t])
        check(lib().vc_column_download(self._h, _b(table), _b(name), out.ctypes.data, len(out), None))
        return out

    def attach(self, table, name, device_ptr):
        check(lib().vc_column_attach(self._h, _b(table), _b(name), ctypes.c_void_p(device_ptr)))

    def column_info(self, table, name):
        """(type, lo, hi, rows) of a column: its type code, declared domain and table rows."""
        t, lo, hi, n = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        check(lib().vc_column_info(self._h, _b(table), _b(name), ctypes.byref(t), ctypes.byref(lo), ctypes.byref(hi),
                                   ctypes.byref(n)))
        return t.value, lo.value, hi.value, n.value

    def import_tbl(self, table, directory, schema, threads=0):
        """Imports <directory>/<table>.tbl (pipe-separated; schema "name:type,..." with types int,
        bigint, date, decN, char, or "-" to skip a field) through the <directory>/cached/ column
        cache.  Returns the row count."""
        n = ctypes.c_int64()
        check(lib().vc_table_import(self._h, _b(table), _b(directory), _b(schema), threads, ctypes.byref(n)))
        self.tables[table] = {"rows": n.value, "columns": {}}
        for item in schema.split(","):
            if item != "-":
                name = item.split(":")[0]
                self.tables[table]["columns"][name] = self.column_info(table, name)[0]
        return n.value

    def attach_host(self, table, name, host_ptr):
        """Reads the column in place from pinned host memory (queries created afterwards)."""
        check(lib().vc_column_attach_host(self._h, _b(table), _b(name), ctypes.c_void_p(host_ptr)))

    def device_ptr(self, table, name):
        p = ctypes.c_void_p()
        check(lib().vc_column_device_ptr(self._h, _b(table), _b(name), ctypes.byref(p)))
        return p.value

    def generate(self, col, cdf=None, stream=None):
        if col.kind == GEN_KINDS["zipf"] and col.s != 0.0 and cdf is None:
            cdf = zipf_cdf(col.s, col.b)
        check(lib().vc_column_generate(self._h, _b(col.table), _b(col.name), col.kind, col.a, col.b, col.c, col.s,
                                       col.seed, None if cdf is None else cdf.ctypes.data, _stream_ptr(stream)))

    def load_workload(self, w, data=None, on_device=True, stream=None):
        """Declares the workload's tables and fills them: from `data` ({table: {col: array}}),
        else with the device generator (on_device) or host generation + upload."""
        for t, rows in w.tables.items():
            self.create_table(t, rows)
        for c in w.columns:
            self.add_column(c.table, c.name, c.type, c.lo, c.hi)
            if self.offline:
                if c.type == STR:
                    self.generate(c)  # strings are encoded on the host: their codes type the plan
                continue
            if data is not None:
                self.upload(c.table, c.name, data[c.table][c.name], stream)
            elif on_device:
                self.generate(c, stream=stream)
            else:
                self.upload(c.table, c.name, generate_host(c), stream)

    def query(self, plan, flavor=""):
        return Query(self, plan, flavor)

    def describe(self, plan, flavor=""):
        """The plan's lowered pipelines (no compilation): vc_plan_describe as a dict."""
        import json
        return json.loads(_text_call(lib().vc_plan_describe, self._h, _b(plan), _b(flavor or "")))


class Query:
    """A compiled query: vc_query_new / run / reset / free."""

    def __init__(self, engine, plan, flavor=""):
        self.engine = engine
        h = ctypes.c_void_p()
        check(lib().vc_query_new(engine._h, _b(plan), _b(flavor or ""), ctypes.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            check(lib().vc_query_free(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, stream=None):
        check(lib().vc_query_run(self._h, _stream_ptr(stream)))
        return self

    def reset(self):
        check(lib().vc_query_reset(self._h))

    def shape(self):
        r = ctypes.c_int64()
        c = ctypes.c_int32()
        check(lib().vc_query_result_shape(self._h, ctypes.byref(r), ctypes.byref(c)))
        return r.value, c.value

    def result(self, out=None):
        """int64 array of shape (rows, cols), column-major (the C ABI's layout; no transpose).
        out: an int64 buffer of at least rows * cols elements to fill (reused across runs it
        saves the page faults of a fresh allocation); the result is then a view of it."""
        r, c = self.shape()
        if out is None or out.size < max(r * c, 1):
            out = np.empty(max(r * c, 1), dtype=np.int64)
        check(lib().vc_query_result_copy(self._h, out.ctypes.data, out.size))
        return out.reshape(-1)[: r * c].reshape(c, r).T

    def result_text(self):
        return _text_call(lib().vc_query_result_text, self._h)

    def result_lines(self):
        return sorted(l for l in self.result_text().split("\n") if l)

    def info(self):
        import json
        return json.loads(_text_call(lib().vc_query_info, self._h))

    def source(self):
        return _text_call(lib().vc_query_source, self._h)

    def profile(self, enable=True):
        check(lib().vc_query_profile(self._h, 1 if enable else 0))

    def time(self, reps=5, flush_l2=True, stream=None):
        """Device time (ms) of each of `reps` runs, L2 flushed before each."""
        ms = (ctypes.c_float * reps)()
        check(lib().vc_query_time(self._h, reps, 1 if flush_l2 else 0, _stream_ptr(stream), ms, reps))
        return [float(x) for x in ms]

    def timings(self):
        ms = (ctypes.c_float * 256)()
        n = ctypes.c_int()
        names = ctypes.create_string_buffer(1 << 16)
        check(lib().vc_query_timings(self._h, ms, 256, ctypes.byref(n), names, len(names)))
        kn = names.value.decode().split("\n")
        return [(kn[i], float(ms[i])) for i in range(n.value)]


class Batch:
    """Many queries in one persistent kernel (vc_batch_*); the queries keep their results.
    Queries with a pipeline of at least `solo_rows` rows (0 = none) run as their own launches
    right after the persistent kernel (vc_batch_new_split)."""

    def __init__(self, queries, flavors=None, threads=256, tiles_per_item=64, solo_rows=0):
        self.queries = list(queries)  # the queries must outlive the batch
        arr = (ctypes.c_void_p * len(self.queries))(*[q._h.value for q in self.queries])
        fl = None
        if flavors is not None:
            fl = (ctypes.c_char_p * len(self.queries))(*[_b(f) if f else None for f in flavors])
        h = ctypes.c_void_p()
        check(lib().vc_batch_new_split(arr, len(self.queries), fl, threads, tiles_per_item, int(solo_rows),
                                       ctypes.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            check(lib().vc_batch_free(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, stream=None):
        check(lib().vc_batch_run(self._h, _stream_ptr(stream)))
        return self

    def wait(self):
        check(lib().vc_batch_wait(self._h))

    def set_wait_limit(self, ns):
        """Longest wait (ns) of a work item on its dependency before the batch gives up."""
        check(lib().vc_batch_set_wait_limit(self._h, int(ns)))

    def hold_item(self, index, hold=True):
        """Test hook: work item `index` waits for a dependency that never completes."""
        check(lib().vc_batch_hold_item(self._h, int(index), 1 if hold else 0))

    def latencies_us(self):
        out = (ctypes.c_double * len(self.queries))()
        check(lib().vc_batch_latencies(self._h, out, len(self.queries)))
        return [float(x) for x in out]

    def info(self):
        import json
        return json.loads(_text_call(lib().vc_batch_info, self._h))

    def source(self):
        return _text_call(lib().vc_batch_source, self._h)

    ITEM_FIELDS = ("shape", "dep", "dep_target", "done", "nitems", "begin", "end", "params")

    def items(self):
        """The work queue in claim order: an (items, 8) int64 array, columns ITEM_FIELDS."""
        n = ctypes.c_int64()
        check(lib().vc_batch_items(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros((n.value, 8), dtype=np.int64)
        check(lib().vc_batch_items(self._h, out.ctypes.data, n.value, ctypes.byref(n)))
        return out


class Mlp:
    """The chooser's perceptron, trained and evaluated by the library's GPU kernels."""

    def __init__(self, n_in, n_hidden, n_out, seed=1, device=0):
        h = ctypes.c_void_p()
        check(lib().vc_mlp_create(device, n_in, n_hidden, n_out, seed, ctypes.byref(h)))
        self._h = h
        self.shape = (n_in, n_hidden, n_out)

    def close(self):
        if self._h:
            check(lib().vc_mlp_free(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def num_params(self):
        n = ctypes.c_int64()
        check(lib().vc_mlp_num_params(self._h, ctypes.byref(n)))
        return n.value

    def get_params(self):
        out = np.empty(self.num_params(), dtype=np.float32)
        check(lib().vc_mlp_get_params(self._h, out.ctypes.data, out.size))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(lib().vc_mlp_set_params(self._h, p.ctypes.data, p.size))

    @staticmethod
    def _f32(a):
        return None if a is None else np.ascontiguousarray(a, dtype=np.float32)

    def loss_grad(self, X, T, mask=None):
        X, T, M = self._f32(X), self._f32(T), self._f32(mask)
        loss = ctypes.c_float()
        g = np.empty(self.num_params(), dtype=np.float32)
        check(lib().vc_mlp_loss_grad(self._h, X.ctypes.data, T.ctypes.data, None if M is None else M.ctypes.data,
                                     X.shape[0], ctypes.byref(loss), g.ctypes.data))
        return float(loss.value), g

    def train(self, X, T, mask=None, epochs=200, batch=64, lr=1e-3, seed=1):
        X, T, M = self._f32(X), self._f32(T), self._f32(mask)
        loss = ctypes.c_float()
        check(lib().vc_mlp_train(self._h, X.ctypes.data, T.ctypes.data, None if M is None else M.ctypes.data,
                                 X.shape[0], epochs, batch, lr, seed, ctypes.byref(loss)))
        return float(loss.value)

    def predict(self, X):
        X = self._f32(X)
        Y = np.empty((X.shape[0], self.shape[2]), dtype=np.float32)
        check(lib().vc_mlp_predict(self._h, X.ctypes.data, X.shape[0], Y.ctypes.data))
        return Y
