"""The learned flavor chooser against the exhaustive autotuner (GPU): trained on autotuner
timings (the full knob grid of each workload's kind) of seeded workloads, evaluated on held-out
ones; and the explorer's sampled search logging to the reference's SQLite runs schema."""
import math
import sqlite3

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_learned_choice_is_close_to_exhaustive_and_beats_default(tmp_path):
    from vldb_voila_b200 import chooser as ch
    log = str(tmp_path / "tune.jsonl")
    train = ch.training_specs(24, seed=11, min_rows=200_000, max_rows=8_000_000)
    held = ch.training_specs(8, seed=12, min_rows=200_000, max_rows=8_000_000)
    for s in train:
        times = ch.autotune(s, reps=3, log_path=log)
        assert len(times) >= 0.8 * len(ch.candidates_for(ch.describe_spec(s)))
    records = ch.load_log(log)
    assert len(records) == len(train)
    test_records = []
    for s in held:
        test_records.append({"spec": s, "features": ch.features(s).tolist(), "times_ms": ch.autotune(s, reps=3)})
    c = ch.Chooser()
    loss = c.fit(records)
    assert math.isfinite(loss)
    res = ch.evaluate(c, test_records)
    ratio = np.exp(np.mean([math.log(r["chosen_ms"] / r["best_ms"]) for r in res]))
    assert ratio <= 1.10, res
    # what the network gains over the method without it (the default flavor)
    assert sum(r["chosen_ms"] for r in res) <= sum(r["default_ms"] for r in res) * 1.02, res


def test_explorer_samples_and_logs_to_the_runs_table(tmp_path):
    from vldb_voila_b200 import chooser as ch
    db = str(tmp_path / "voila.db")
    spec = "groupby:rows=400000,keys=50000,zipf=0.8,seed=5"
    times = ch.explore(spec, mode="sample", sample=6, seed=3, reps=2, sqlite_path=db)
    assert ch.DEFAULT in times and 2 <= len(times) <= 7
    con = sqlite3.connect(db)
    n, = con.execute("SELECT COUNT(*) FROM runs WHERE backend = 'cuda' AND result = 'OK'").fetchone()
    assert n == 2 * len(times)
    best = con.execute("SELECT full_blend, MIN(time_ms) FROM runs WHERE result = 'OK'").fetchone()
    assert best[0] in times


def test_per_pipeline_backtracking_never_loses_to_its_start(tmp_path):
    from vldb_voila_b200 import chooser as ch
    db = str(tmp_path / "voila.db")
    spec = "star:rows=2000000,custs=30000,supps=2000,parts=140000,seed=7"
    base = "cuda()"
    best, ms = ch.backtrack(spec, base=base, reps=3, sqlite_path=db)
    assert best.startswith(base)
    con = sqlite3.connect(db)
    base_ms = [r[0] for r in con.execute("SELECT time_ms FROM runs WHERE full_blend = ? AND result = 'OK'", (base,))]
    assert ms <= float(np.median(base_ms)) + 1e-9
    n, = con.execute("SELECT COUNT(*) FROM runs WHERE mode = 'backtrack'").fetchone()
    assert n >= 3 * len(ch.PIPE_GRID)
