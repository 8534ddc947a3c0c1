"""Shared test helpers: golden fixtures, checksums and running plans on the GPU and oracle."""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def manifest():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)


def golden_lines(case, flavor):
    path = os.path.join(GOLDEN, f"{case}.{flavor}.txt")
    with open(path) as f:
        return sorted(l for l in f.read().split("\n") if l)


def _mix64(z):
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xbf58476d1ce4e5b9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94d049bb133111eb)
    return z ^ (z >> np.uint64(31))


def _fnv1a(b):
    h = 0xcbf29ce484222325
    for x in b:
        h = ((h ^ x) * 0x100000001b3) & 0xffffffffffffffff
    return h


def data_checksum(w, data):
    """Same order-insensitive checksum the reference harness prints (oracle/ref/ref_data.cpp)."""
    total = np.uint64(0)
    with np.errstate(over="ignore"):
        for ti, t in enumerate(w.tables):
            for ci, c in enumerate(w.table_columns(t)):
                a = data[t][c.name]
                if a.dtype == object:  # strings: FNV-1a of their bytes, as the reference harness
                    a = np.array([_fnv1a(x.encode()) for x in a], dtype=np.uint64).view(np.int64)
                v = a.astype(np.int64).view(np.uint64)
                i = np.arange(len(v), dtype=np.uint64)
                x = v * np.uint64(31) + i * np.uint64(1000003) + np.uint64(ti * 131) + np.uint64(ci)
                total = total + _mix64(x).sum(dtype=np.uint64)
    return int(total)


# A join whose build side is itself a join (over the star workload's tables): customers are
# kept when their region is the weekday of one of the first three dates.  In a batch, the
# customer build probes the date table and must wait for the date build.
NESTED_BUILD_PLAN = (
    "(aggr global () ((fun sum (col lineorder.lo_revenue)) (fun count))"
    " (join join01 ((col lineorder.lo_custkey)) () (scan lineorder (lo_custkey lo_revenue))"
    "  ((col customer.c_custkey)) ()"
    "  (join join01 ((col customer.c_region)) () (scan customer (c_custkey c_region))"
    "   ((col date.d_weekday)) ()"
    "   (select (fun < (col date.d_datekey) (const 4)) (scan date (d_datekey d_weekday))))))")
