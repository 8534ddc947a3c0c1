"""The learned flavor chooser against the exhaustive autotuner (GPU): trained on autotuner
timings of seeded workloads, evaluated on held-out ones."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_learned_choice_is_close_to_exhaustive_and_beats_default(tmp_path):
    from vldb_voila_b200 import chooser as ch
    log = str(tmp_path / "tune.jsonl")
    train = ch.training_specs(24, seed=11, min_rows=200_000, max_rows=8_000_000)
    held = ch.training_specs(8, seed=12, min_rows=200_000, max_rows=8_000_000)
    for s in train:
        ch.autotune(s, reps=3, log_path=log)
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
    assert sum(r["chosen_ms"] for r in res) <= sum(r["default_ms"] for r in res) * 1.02, res
