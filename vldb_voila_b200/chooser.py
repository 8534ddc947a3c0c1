"""Flavor selection for pipelines: the exhaustive autotuner and the learned chooser.

The reference explores its blend space by compiling and timing variants (explorer.cpp:111-134
per-pipeline backtracking, :352-426 random sampling; runs logged to SQLite, compiler.cpp:91-256).
Here:

  * `autotune` is the exhaustive search: every candidate CUDA flavor of a pipeline is compiled
    (NVRTC, cached by source) and timed on the GPU (device events, L2 flushed before every run);
    results are appended to a JSONL log so a search can be resumed and reused as training data.
  * `Chooser` is the learned part: a small MLP, trained and evaluated on the GPU by the library's
    own kernels (csrc/mlp.cu), maps per-pipeline features (row count, predicate selectivity,
    build size, key cardinality, Zipf skew, payload widths, operator counts) to the predicted
    relative time of every candidate flavor and picks the argmin.  Results never depend on the
    choice, only speed; the autotuner is its fallback and the yardstick of its choices.
"""
import json
import math
import os

import numpy as np

from .engine import Engine, Mlp, workload

# Candidate flavors (the computation_type=cuda(...) blends searched per pipeline).  Knobs
# that do not apply to a pipeline leave its generated code unchanged.
CANDIDATES = [
    "cuda()",
    "cuda(prefetch=0)",
    "cuda(rows=2,prefetch=0)",
    "cuda(rows=8,prefetch=0)",
    "cuda(load=tma,stages=2)",
    "cuda(lowcard=private)",
    "cuda(lowcard=private,prefetch=0)",
    "cuda(threads=128,lowcard=private,load=tma,stages=2)",
    "cuda(aggr=cache,cache=128)",
    "cuda(aggr=cache,cache=256,fill=75)",
    "cuda(fill=75)",
    "cuda(aggr=cache,cache=128,fill=75,prefetch=0)",
    "cuda(build=staged,prefetch=0)",
    "cuda(compact=-1,prefetch=0)",
    "cuda(threads=128)",
    "cuda(aggr=cache,cache=256,fill=75,prefetch=0)",
    "cuda(aggr=cache,cache=2048,fill=75,prefetch=0,threads=512)",
    "cuda(build=direct)",
]

DEFAULT = "cuda()"

FEATURE_NAMES = ["log2_rows", "selectivity", "log2_build_rows", "log2_key_domain", "zipf", "bytes_per_row",
                 "probes", "aggregates", "t_sel_aggr", "t_join_aggr", "t_groupby", "t_star"]


def _params(spec):
    tmpl, _, rest = spec.partition(":")
    out = {}
    for item in rest.split(","):
        if "=" in item:
            k, v = item.split("=", 1)
            out[k] = float(v)
    return tmpl, out


def features(spec):
    """Feature vector of a workload spec (see FEATURE_NAMES)."""
    w = workload(spec)
    tmpl, p = _params(spec)
    rows = max(w.fact_rows, 1)
    fact_cols = w.table_columns(w.fact_table)
    bpr = sum(np.dtype(c.dtype).itemsize for c in fact_cols)
    build_rows, domain, probes, aggs, sel, zipf = 0, 1, 0, 1, 1.0, 0.0
    if tmpl == "sel_aggr":
        sel = p.get("sel", 2436 / 2526.0)
        domain, aggs = 180, 5
    elif tmpl == "join_aggr":
        build_rows = w.tables["orders"]
        sel = p.get("sel", 0.2)
        domain, probes, aggs = build_rows, 1, 2
    elif tmpl == "groupby":
        domain = p.get("keys", 1500000)
        zipf = p.get("zipf", 0.0)
        aggs = 3
    elif tmpl == "star":
        build_rows = sum(n for t, n in w.tables.items() if t != w.fact_table)
        sel, domain, probes, aggs = 1 / 875.0, 35, 4, 2
    onehot = [float(tmpl == t) for t in ("sel_aggr", "join_aggr", "groupby", "star")]
    return np.array([math.log2(rows), sel, math.log2(build_rows + 1), math.log2(max(domain, 1)), zipf, bpr / 32.0,
                     probes, aggs / 8.0] + onehot, dtype=np.float32)


def autotune(spec, candidates=CANDIDATES, reps=5, log_path=None, engine=None, device=0):
    """Exhaustive search: {flavor: median device ms} for every candidate on the workload."""
    own = engine is None
    eng = engine or Engine(device)
    w = workload(spec)
    if own:
        eng.load_workload(w, on_device=True)
    times = {}
    for fl in candidates:
        q = eng.query(w.plan, fl)
        q.time(1)  # warm-up: module load, first-touch of tables
        times[fl] = float(np.median(q.time(reps)))
        q.close()
    if log_path:
        with open(log_path, "a") as f:
            f.write(json.dumps({"spec": spec, "features": features(spec).tolist(), "times_ms": times}) + "\n")
    if own:
        eng.close()
    return times


def load_log(path):
    rows = []
    if os.path.exists(path):
        with open(path) as f:
            for line in f:
                line = line.strip()
                if line:
                    rows.append(json.loads(line))
    return rows


class Chooser:
    """MLP over workload features predicting log2(time / median time) of each candidate."""

    def __init__(self, candidates=CANDIDATES, hidden=64, seed=7, device=0):
        self.candidates = list(candidates)
        self.hidden = hidden
        self.seed = seed
        self.device = device
        self.mlp = None
        self.mu = None
        self.sd = None

    def _targets(self, records):
        T = np.zeros((len(records), len(self.candidates)), dtype=np.float32)
        M = np.zeros_like(T)
        for i, r in enumerate(records):
            t = r["times_ms"]
            vals = [t[c] for c in self.candidates if c in t]
            med = float(np.median(vals))
            for j, c in enumerate(self.candidates):
                if c in t and t[c] > 0:
                    T[i, j] = math.log2(t[c] / med)
                    M[i, j] = 1.0
        return T, M

    def fit(self, records, epochs=400, batch=32, lr=2e-3):
        X = np.stack([np.asarray(r["features"], dtype=np.float32) for r in records])
        self.mu = X.mean(axis=0)
        self.sd = X.std(axis=0) + 1e-3
        Xn = (X - self.mu) / self.sd
        T, M = self._targets(records)
        self.mlp = Mlp(X.shape[1], self.hidden, len(self.candidates), seed=self.seed, device=self.device)
        return self.mlp.train(Xn, T, M, epochs=epochs, batch=batch, lr=lr, seed=self.seed)

    def predict(self, feats):
        X = (np.atleast_2d(np.asarray(feats, dtype=np.float32)) - self.mu) / self.sd
        return self.mlp.predict(X)

    def choose(self, spec_or_features):
        f = features(spec_or_features) if isinstance(spec_or_features, str) else spec_or_features
        return self.candidates[int(np.argmin(self.predict(f)[0]))]


def evaluate(chooser, records):
    """Per record: time of the chosen, exhaustive-best and default flavors."""
    out = []
    for r in records:
        t = r["times_ms"]
        pick = chooser.choose(np.asarray(r["features"], dtype=np.float32))
        best = min(t.values())
        out.append({"spec": r["spec"], "chosen": pick, "chosen_ms": t[pick], "best_ms": best,
                    "best": min(t, key=t.get), "default_ms": t[DEFAULT]})
    return out


def training_specs(count, seed, min_rows=100_000, max_rows=20_000_000):
    """Seeded workloads drawn like the mixed batch (sizes log-uniform, selectivities and
    skews uniform) plus star joins, for the autotuner to label."""
    from .engine import batch_specs
    specs = batch_specs(count, seed, min_rows, max_rows)
    rng = np.random.default_rng(seed)
    n_star = max(1, count // 8)
    for i in range(n_star):
        rows = int(math.exp(rng.uniform(math.log(min_rows), math.log(max_rows))))
        specs.append(f"star:rows={rows},seed={seed * 100 + i}")
    return specs
