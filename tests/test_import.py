"""Data import (vc_table_import): pipe-separated .tbl text through the reference's binary
column cache (<dir>/cached/<table>_<column>, raw arrays) into engine columns whose declared
domains are the observed min/max.  CPU part on a compile-only engine; the GPU part runs a
query over imported data against the oracle."""
import os

import numpy as np
import pytest

from vldb_voila_b200 import Engine, VoilaError

TBL = ("1|17|1996-03-13|7.5|N|O|x|\n"
       "2|-36|1992-01-01|-1.25|R|F|y|\r\n"
       "3|8|2000-02-29|0|A|F|z|\n"
       "\n"
       "4|28|1998-12-01|12345678.99|N|O|w|\n")
SCHEMA = "k:int,q:bigint,d:date,p:dec2,f:char,s:char,-"


def _write(tmp_path, text=TBL, name="li"):
    (tmp_path / f"{name}.tbl").write_text(text)
    return str(tmp_path)


def test_import_parses_types_and_writes_the_reference_cache(tmp_path):
    d = _write(tmp_path)
    e = Engine(offline=True)
    assert e.import_tbl("li", d, SCHEMA, threads=2) == 4
    cache = os.path.join(d, "cached")
    k = np.fromfile(os.path.join(cache, "li_k"), dtype=np.int32)
    q = np.fromfile(os.path.join(cache, "li_q"), dtype=np.int64)
    dd = np.fromfile(os.path.join(cache, "li_d"), dtype=np.int32)
    p = np.fromfile(os.path.join(cache, "li_p"), dtype=np.int64)
    f = np.fromfile(os.path.join(cache, "li_f"), dtype=np.uint8)
    assert k.tolist() == [1, 2, 3, 4] and q.tolist() == [17, -36, 8, 28]
    # Julian day numbers: 1992-01-01 is 2448623 (the workloads' ship-date origin)
    assert dd.tolist() == [2450156, 2448623, 2451604, 2451149]
    assert p.tolist() == [750, -125, 0, 1234567899]
    assert bytes(f) == b"NRAN"
    assert sorted(os.listdir(cache)) == ["li_d", "li_f", "li_k", "li_p", "li_q", "li_s"]
    assert e.column_info("li", "q")[1:] == (-36, 28, 4)
    assert e.column_info("li", "f")[:3] == (1, ord("A"), ord("R"))
    assert e.column_info("li", "d")[0] == 3 and e.column_info("li", "p")[0] == 4


def test_import_reads_the_cache_instead_of_the_text(tmp_path):
    d = _write(tmp_path)
    Engine(offline=True).import_tbl("li", d, SCHEMA)
    os.remove(os.path.join(d, "li.tbl"))
    e = Engine(offline=True)
    assert e.import_tbl("li", d, SCHEMA) == 4
    assert e.column_info("li", "p")[1:3] == (-125, 1234567899)


@pytest.mark.parametrize("text,msg", [("1|2|1996-13-01|1.0|N|O|x|\n", "cannot parse field d"),
                                      ("1|2|1996-01-01|1.005|N|O|x|\n", "cannot parse field p"),
                                      ("1|2|1996-01-01\n", "fewer fields"),
                                      ("99999999999|2|1996-01-01|1|N|O|x|\n", "cannot parse field k")])
def test_import_rejects_malformed_rows(tmp_path, text, msg):
    d = _write(tmp_path, text)
    with pytest.raises(VoilaError) as ex:
        Engine(offline=True).import_tbl("li", d, SCHEMA)
    assert ex.value.code == 1 and msg in str(ex.value)


def test_import_splits_large_files_across_threads(tmp_path):
    n = 60000
    rng = np.random.default_rng(1)
    a = rng.integers(-10**6, 10**6, n)
    lines = "".join(f"{i}|{v}|\n" for i, v in enumerate(a))
    d = _write(tmp_path, lines * 40, name="big")
    e = Engine(offline=True)
    assert e.import_tbl("big", d, "i:int,v:bigint", threads=7) == 40 * n
    v = np.fromfile(os.path.join(d, "cached", "big_v"), dtype=np.int64)
    assert np.array_equal(v, np.tile(a, 40))
    assert e.column_info("big", "v")[1:3] == (int(a.min()), int(a.max()))


@pytest.mark.gpu
def test_query_over_imported_data_matches_oracle(tmp_path):
    """A Q1-shaped query over a lineitem imported from .tbl text (written from the seeded
    sel_aggr generator, prices and discounts as decimals the way dbgen prints them) equals the
    oracle over the same values."""
    import datetime

    from oracle.voila_oracle import result_lines, run_plan
    from vldb_voila_b200 import generate_workload_host, workload
    w = workload("sel_aggr:rows=200000,seed=91")
    data = generate_workload_host(w)["lineitem"]
    names = ["l_quantity", "l_extendedprice", "l_discount", "l_tax", "l_returnflag", "l_linestatus", "l_shipdate"]
    base = datetime.date(1992, 1, 1).toordinal() - 2448623
    cols = [data["l_quantity"].astype(str), [f"{v // 100}.{v % 100:02d}" for v in data["l_extendedprice"].tolist()],
            [f"0.{v:02d}" for v in data["l_discount"].tolist()], data["l_tax"].astype(str),
            [chr(c) for c in data["l_returnflag"].tolist()], [chr(c) for c in data["l_linestatus"].tolist()],
            [datetime.date.fromordinal(int(x) + base).isoformat() for x in data["l_shipdate"].tolist()]]
    text = "\n".join("|".join(r) + "|" for r in zip(*cols)) + "\n"
    (tmp_path / "lineitem.tbl").write_text(text)
    e = Engine(0)
    e.import_tbl("lineitem", str(tmp_path), "l_quantity:int,l_extendedprice:dec2,l_discount:dec2,l_tax:int,"
                 "l_returnflag:char,l_linestatus:char,l_shipdate:date")
    imported = {"lineitem": {n: data[n] for n in names}}
    q = e.query(w.plan)
    q.run()
    assert q.result_lines() == result_lines(run_plan(w.plan, imported))
