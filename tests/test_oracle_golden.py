"""The oracle against the reference's own outputs (tests/golden, made by make_golden.py from
the reference's hyper and vectorwise flavors).  CPU only."""
import numpy as np
import pytest

from helpers import data_checksum, golden_lines, manifest
from oracle.voila_oracle import result_lines, run_plan
from vldb_voila_b200 import generate_workload_host, workload

CASES = sorted(manifest().items())


@pytest.mark.parametrize("name,entry", CASES, ids=[c[0] for c in CASES])
def test_oracle_matches_reference_vectorwise(name, entry):
    w = workload(entry["spec"])
    data = generate_workload_host(w)
    # the data is the reference loader's data, byte for byte
    assert str(data_checksum(w, data)) == entry["checksum"]
    plan = entry["plan"] or w.plan
    assert result_lines(run_plan(plan, data)) == golden_lines(name, "vectorwise")


@pytest.mark.parametrize("name,entry", CASES, ids=[c[0] for c in CASES])
def test_reference_flavors_agree_except_hyper_charge_wrap(name, entry):
    hyper = golden_lines(name, "hyper")
    vec = golden_lines(name, "vectorwise")
    if hyper == vec:
        return
    # Only the TPC-H Q1-shaped plan differs: the reference's hyper flavor evaluates
    # charge = disc_price * (100 + tax) as u32 * u8 in C++ (its typing pass types disc_price
    # as u32), so every product wraps modulo 2^32 before being summed.
    w = workload(entry["spec"])
    assert w.template == "sel_aggr" and entry["plan"] is None
    data = generate_workload_host(w)["lineitem"]
    keep = data["l_shipdate"].astype(np.int64) <= int(w.plan.split("(const ")[-1].split(")")[0])
    price = data["l_extendedprice"].astype(np.int64)[keep]
    disc = data["l_discount"].astype(np.int64)[keep]
    tax = data["l_tax"].astype(np.int64)[keep]
    rf = data["l_returnflag"].astype(np.int64)[keep]
    ls = data["l_linestatus"].astype(np.int64)[keep]
    charge_wrapped = ((price * (100 - disc)) * (100 + tax)) % (1 << 32)
    by_group = {}
    for k1, k2, c in zip(rf.tolist(), ls.tolist(), charge_wrapped.tolist()):
        by_group[(k1, k2)] = by_group.get((k1, k2), 0) + c
    expect = sorted(
        "|".join(f.split("|")[:5] + [str(by_group[(int(f.split("|")[0]), int(f.split("|")[1]))])] + f.split("|")[6:])
        for f in vec)
    assert hyper == expect
