"""CPU oracle for the hot path -- TEST INFRASTRUCTURE ONLY.

A numpy restatement of what the reference's generated pipelines compute for a relational
plan: scans, selections, projections, Join01/JoinN hash joins and hash / global
aggregations, with exact int64 arithmetic, emitting QueryResult text rows.  Only tests/,
__graft_entry__.smoke() and bench.py's cpu_baseline leg may use it, and only as the checker
(or the timed CPU port); the product path never calls it.

Pinned: tests/golden holds the reference's own outputs (its hyper and vectorwise flavors,
compiled from the reference sources by oracle/ref/Makefile and run by oracle/ref/ref_run)
for seeded workloads; tests/test_oracle_golden.py checks this oracle against them.

Semantics followed (reference file:line):
  - Scan: every row of the base table, columns named "table.col" (relalg_translator.cpp:202-272)
  - Select: rows whose predicate holds (seltrue + emit, relalg_translator.cpp:343-378;
    comparison primitives kernel_generator.py:414-454)
  - Project: visible columns become the projection list; assignments are visible to later
    entries of the same list (relalg_translator.cpp:275-341)
  - arithmetic: exact integers (the typing pass widens results so nothing wraps,
    typing_pass.cpp:164-176; vectorwise primitives compute in the result type,
    kernel_generator.py:439-445)
  - HashJoin: visible after the probe: probe columns, build keys (= probe key values),
    build payloads (relalg_translator.cpp:955-1012); JoinN emits one row per match,
    Join01 stops after the first match (:1032-1042)
  - HashAggr: groups by keys, sums and counts; a hidden count if none is given (:469-472);
    output = keys then visible aggregates for groups with count > 0 (:692-771); global
    aggregation is one group (:430-441) and is emitted only when its count is > 0
  - output text: decimal integers joined by '|', one line per row
    (voila_cast::to_cstr runtime.hpp:346-391, QueryResult::push_col runtime_framework.cpp:77-111),
    compared after sorting lines (Query::check_result, runtime_framework.cpp:220-280)
"""
import numpy as np

_FUNS = {
    "<=": "le", "<": "lt", ">=": "ge", ">": "gt", "=": "eq", "!=": "ne", "+": "add", "-": "sub", "*": "mul",
}


def parse_sexpr(text):
    """Plan text -> nested lists of atoms (strings)."""
    tokens = text.replace("(", " ( ").replace(")", " ) ").split()
    pos = 0

    def read():
        nonlocal pos
        t = tokens[pos]
        pos += 1
        if t == "(":
            out = []
            while tokens[pos] != ")":
                out.append(read())
            pos += 1
            return out
        if t == ")":
            raise ValueError("unexpected ')'")
        return t

    node = read()
    if pos != len(tokens):
        raise ValueError("trailing text after plan")
    return node


class Frame:
    """An ordered set of named columns of equal length (the reference's 'flow')."""

    def __init__(self, cols, n):
        self.cols = cols  # list of (name, ndarray int64)
        self.n = n

    def get(self, name):
        for k, v in reversed(self.cols):
            if k == name:
                return v
        raise KeyError(f"cannot find '{name}' among the visible columns")

    def take(self, idx):
        return Frame([(k, v[idx]) for k, v in self.cols], int(len(idx)))


def _eval(e, frame, env):
    head = e[0]
    if head == "const":
        try:
            return np.full(frame.n, int(e[1]), dtype=np.int64)
        except ValueError:  # a string constant
            return np.full(frame.n, e[1], dtype=object)
    if head == "col":
        if e[1] in env:
            return env[e[1]]
        return frame.get(e[1])
    if head == "fun":
        f = _FUNS.get(e[1], e[1])
        a = [_eval(x, frame, env) for x in e[2:]]
        if f == "extract_year":
            return _julian_year(a[0])
        if f == "contains":  # substring test (runtime.hpp:150-224)
            return np.fromiter((p in x for x, p in zip(a[0], a[1])), dtype=bool, count=frame.n)
        if f == "add":
            return a[0] + a[1]
        if f == "sub":
            return a[0] - a[1]
        if f == "mul":
            return a[0] * a[1]
        if f == "lt":
            return a[0] < a[1]
        if f == "le":
            return a[0] <= a[1]
        if f == "gt":
            return a[0] > a[1]
        if f == "ge":
            return a[0] >= a[1]
        if f == "eq":
            return a[0] == a[1]
        if f == "ne":
            return a[0] != a[1]
        if f == "and":
            return a[0] & a[1]
        if f == "or":
            return a[0] | a[1]
        raise ValueError(f"unknown function {e[1]}")
    raise ValueError(f"bad expression {e}")


def _julian_year(jd):
    """Gregorian year of Julian day numbers, in the unsigned 32-bit steps of the reference's
    splitJulianDay (runtime.hpp:128-148; the Calendar FAQ conversion)."""
    u = np.uint64(0xffffffff)
    a = (jd.astype(np.uint64) + np.uint64(32044)) & u
    b = ((np.uint64(4) * a + np.uint64(3)) & u) // np.uint64(146097)
    c = (a - ((np.uint64(146097) * b) & u) // np.uint64(4)) & u
    d = ((np.uint64(4) * c + np.uint64(3)) & u) // np.uint64(1461)
    e = (c - ((np.uint64(1461) * d) & u) // np.uint64(4)) & u
    m = ((np.uint64(5) * e + np.uint64(2)) & u) // np.uint64(153)
    return ((np.uint64(100) * b + d - np.uint64(4800) + m // np.uint64(10)) & u).astype(np.int64)


def _check_int64(arrs):
    # values are computed in int64; the product rejects plans whose declared ranges could
    # leave int64, so the oracle only needs to detect accidental overflow
    for a in arrs:
        if a.dtype == np.int64 and a.size and (a.max() > 2**62 or a.min() < -2**62):
            raise OverflowError("oracle value range close to int64 limits")


def _column(a):
    """A base column: int64 values, or Python strings (object array) for a string column."""
    a = np.asarray(a)
    return a if a.dtype == object else a.astype(np.int64)


def _py(x):
    return x if isinstance(x, str) else int(x)


def _exact(v):
    """v as int64 when its sums cannot leave int64, else as Python ints (exact 128-bit sums,
    the reference's i128 results, typing_pass.cpp:244-259)."""
    if v.size and int(np.abs(v).max()) * v.size >= 2**62:
        return v.astype(object)
    return v


def _pack_keys(cols):
    """Unique int64 code per key tuple (via np.unique on stacked keys)."""
    if len(cols) == 1:
        return cols[0]
    stacked = np.stack(cols, axis=1)
    _, inv = np.unique(stacked, axis=0, return_inverse=True)
    return inv.reshape(-1).astype(np.int64)


def _aggr_names(node, counter=None, names=None):
    """Output table name of every aggregation below the root, as the reference's translator
    numbers them: one id per hash join, taken before its build side is translated
    (relalg_translator.cpp:814), and two per aggregation, taken after its input (the build
    pass and the re-aggregation, :392 and :776-808); the re-aggregation's table names the
    visible columns <name>.key_<i> and <name>.aggr_<j> (:740-760)."""
    if counter is None:
        counter, names = [0], {}
    head = node[0]
    if head in ("select", "project"):
        _aggr_names(node[2], counter, names)
    elif head == "join":
        counter[0] += 1
        _aggr_names(node[7], counter, names)
        _aggr_names(node[4], counter, names)
    elif head == "aggr":
        _aggr_names(node[4], counter, names)
        counter[0] += 2
        names[id(node)] = f"aggr_ht{counter[0] - 1}"
    return names


def _aggregate(node, f):
    """Keys and visible aggregates of an aggregation over frame f: (key columns, aggregate
    columns), one entry per group with count > 0 (relalg_translator.cpp:469-472, :692-701)."""
    glob = node[1] == "global"
    keys = [_eval(k, f, {}) for k in node[2]]
    aggs = []
    for a in node[3]:
        if a[1] == "count":
            aggs.append(("count", None))
        else:
            aggs.append(("sum", _eval(a[2], f, {}).astype(np.int64)))
    _check_int64(keys + [v for _, v in aggs if v is not None])
    if f.n == 0:
        return [np.zeros(0, dtype=np.int64) for _ in keys], [np.zeros(0, dtype=np.int64) for _ in aggs]
    if glob:
        return [], [np.array([f.n if kind == "count" else _exact(v).sum()], dtype=object) for kind, v in aggs]
    # keys as integer codes per column (strings too), grouped on the stacked codes
    enc = [np.unique(k, return_inverse=True) for k in keys]
    stacked = np.stack([inv.reshape(-1) for _, inv in enc], axis=1)
    uniq, inv = np.unique(stacked, axis=0, return_inverse=True)
    inv = inv.reshape(-1)
    order = np.argsort(inv, kind="stable")
    bounds = np.concatenate([[0], np.nonzero(np.diff(inv[order]))[0] + 1])
    counts = np.diff(np.concatenate([bounds, [f.n]]))
    out = []
    for kind, v in aggs:
        if kind == "count":
            out.append(counts.astype(np.int64))
        else:
            out.append(np.add.reduceat(_exact(v)[order], bounds))
    return [enc[i][0][uniq[:, i]] for i in range(uniq.shape[1])], out


def _op(node, db, names=None):
    if names is None:
        names = _aggr_names(node)
    head = node[0]
    if head == "aggr":
        f = _op(node[4], db, names)
        keys, aggs = _aggregate(node, f)
        name = names[id(node)]
        cols = [(f"{name}.key_{i}", k) for i, k in enumerate(keys)]
        cols += [(f"{name}.aggr_{j}", a) for j, a in enumerate(aggs)]
        return Frame(cols, len(aggs[0]) if aggs else (len(keys[0]) if keys else 0))
    if head == "scan":
        table = node[1]
        cols = [(f"{table}.{c}", _column(db[table][c])) for c in node[2]]
        n = len(cols[0][1]) if cols else 0
        return Frame(cols, n)
    if head == "select":
        f = _op(node[2], db, names)
        m = _eval(node[1], f, {}).astype(bool)
        return f.take(np.nonzero(m)[0])
    if head == "project":
        f = _op(node[2], db, names)
        env = {}
        out = []
        for e in node[1]:
            if e[0] == "assign":
                v = _eval(e[2], f, env)
                env[e[1]] = v
                out.append((e[1], v))
            elif e[0] == "col":
                out.append((e[1], env[e[1]] if e[1] in env else f.get(e[1])))
            else:
                raise ValueError("projection entries must be columns or assignments")
        return Frame(out, f.n)
    if head == "join":
        join01 = node[1] == "join01"
        probe = _op(node[4], db, names)
        build = _op(node[7], db, names)
        pk = [_eval(k, probe, {}) for k in node[2]]
        bk = [_eval(k, build, {}) for k in node[5]]
        bpay = [(p[1], _eval(p, build, {})) for p in node[6]]
        # one code space for probe and build key tuples
        if len(pk) == 1:
            pc, bc = pk[0], bk[0]
        else:
            both = [np.concatenate([a, b]) for a, b in zip(pk, bk)]
            code = _pack_keys(both)
            pc, bc = code[:probe.n], code[probe.n:]
        order = np.argsort(bc, kind="stable")
        sb = bc[order]
        lo = np.searchsorted(sb, pc, side="left")
        hi = np.searchsorted(sb, pc, side="right")
        cnt = hi - lo
        if join01:
            cnt = np.minimum(cnt, 1)
        rows = np.repeat(np.arange(probe.n), cnt)
        starts = np.repeat(lo, cnt)
        offs = np.arange(len(rows)) - np.repeat(np.cumsum(cnt) - cnt, cnt)
        bidx = order[starts + offs] if len(rows) else np.zeros(0, dtype=np.int64)
        out = probe.take(rows)
        for i, k in enumerate(node[5]):
            # build keys take the probe key values (relalg_translator.cpp:965-975)
            out.cols.append((k[1], pk[i][rows]))
        for name, v in bpay:
            out.cols.append((name, v[bidx]))
        return out
    raise ValueError(f"unsupported operator {head}")


def run_plan(plan, db):
    """Result rows (list of tuples of ints) of plan text over db = {table: {col: array}}."""
    node = parse_sexpr(plan) if isinstance(plan, str) else plan
    names = _aggr_names(node)
    if node[0] != "aggr":
        f = _op(node, db, names)
        return [tuple(_py(v[i]) for _, v in f.cols) for i in range(f.n)]
    f = _op(node[4], db, names)
    keys, aggs = _aggregate(node, f)
    cols = keys + aggs
    n = len(cols[0]) if cols else 0
    return [tuple(_py(c[i]) for c in cols) for i in range(n)]


def result_lines(rows):
    """QueryResult text lines, sorted (the reference's order-insensitive comparison)."""
    return sorted("|".join(str(v) for v in r) for r in rows)
