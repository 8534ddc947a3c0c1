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


def data_checksum(w, data):
    """Same order-insensitive checksum the reference harness prints (oracle/ref/ref_data.cpp)."""
    total = np.uint64(0)
    with np.errstate(over="ignore"):
        for ti, t in enumerate(w.tables):
            for ci, c in enumerate(w.table_columns(t)):
                v = data[t][c.name].astype(np.int64).view(np.uint64)
                i = np.arange(len(v), dtype=np.uint64)
                x = v * np.uint64(31) + i * np.uint64(1000003) + np.uint64(ti * 131) + np.uint64(ci)
                total = total + _mix64(x).sum(dtype=np.uint64)
    return int(total)
