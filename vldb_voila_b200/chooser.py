"""Flavor selection for pipelines: the exhaustive autotuner, the explorer and the learned chooser.

The reference explores its blend space by compiling and timing variants (explorer.cpp:111-134
per-pipeline backtracking, :352-426 random sampling; domains explorer_helper.cpp:6-21; runs
logged to the SQLite `runs` table, compiler.cpp:91-256).  Here:

  * the search space is a grid of CUDA-flavor knobs per pipeline kind (`GRIDS`): the kind of a
    query's fact pipeline -- a scan with a small-domain aggregation, one join probe, a chain of
    probes, a hash group-by -- decides which knobs can change its generated code, and the grid
    is their full product;
  * `autotune` is the exhaustive search over a kind's grid: every candidate is compiled
    (NVRTC, cached by source) and timed on the GPU (device events, L2 flushed before every
    run); candidates the device cannot run (shared memory) are skipped;
  * `explore` is the reference explorer's counterpart: the full grid or a seeded random sample
    of it, every run logged to a JSONL file and/or the reference's SQLite `runs` schema
    (backend 'cuda', the flavor string as the blend); `backtrack` is its per-pipeline
    backtracking, over "p<id>=cuda(...)" overrides of single pipelines;
  * `Chooser` is the learned part: a small MLP, trained and evaluated on the GPU by the
    library's own kernels (csrc/mlp.cu), maps a pipeline's features -- taken from the lowered
    plan (vc_plan_describe: rows, probes, rows of the probed builds, key domain, groups bound,
    aggregates, bytes per row, sink kind) plus the data statistics a caller knows (predicate
    selectivity, Zipf skew) -- to the predicted relative time of every grid candidate, and
    picks the argmin among the candidates of the query's kind.  Results never depend on the
    choice, only speed; the autotuner is its fallback and the yardstick of its choices.
"""
import itertools
import json
import math
import os
import sqlite3
import time

import numpy as np

from .engine import Engine, Mlp, VoilaError, workload

DEFAULT = "cuda()"


def _load_modes():
    # (load, prefetch, stages): vector loads with or without the next tile in flight, or the
    # bulk-copy ring at two depths
    return [("ldg", 1, None), ("ldg", 0, None), ("tma", None, 2), ("tma", None, 4)]


def _scan_grid():
    out = []
    for threads, rows, (load, pf, stages), lowcard in itertools.product(
            (128, 256), (4, 8), _load_modes(), ("combine", "private", "redux", "regs")):
        items = [f"threads={threads}", f"rows={rows}", f"load={load}", f"lowcard={lowcard}"]
        items += [f"prefetch={pf}"] if pf is not None else [f"stages={stages}"]
        out.append("cuda(" + ",".join(items) + ")")
    return out


def _hash_grid():
    out = []
    for threads, rows, pf, aggr, fill in itertools.product(
            (256, 512), (2, 4), (0, 1), ("global", "cache,cache=256", "cache,cache=2048"), (50, 75)):
        out.append(f"cuda(threads={threads},rows={rows},prefetch={pf},aggr={aggr},fill={fill})")
    # the partitioned group-by (histogram + scatter + shared-memory tables per partition)
    for threads, rows in itertools.product((256, 512), (4, 8)):
        out.append(f"cuda(threads={threads},rows={rows},aggr=part)")
    # the direct table (slot = packed key), alone or behind the shared-memory cache
    for threads, rows, aggr in itertools.product((256, 512), (2, 4), ("direct", "dcache,cache=256", "dcache,cache=2048")):
        out.append(f"cuda(threads={threads},rows={rows},prefetch=1,aggr={aggr})")
    return out


def _join_grid():
    out = []
    for threads, rows, pf, build in itertools.product((128, 256), (2, 4, 8), (0, 1), ("auto", "direct", "direct4")):
        b = "build=direct,probe=4" if build == "direct4" else f"build={build}"
        out.append(f"cuda(threads={threads},rows={rows},prefetch={pf},{b})")
    return out


def _star_grid():
    out = []
    for threads, rows, compact, pf, lowcard in itertools.product(
            (128, 256), (4, 8), ("auto", -1), (0, 1), ("combine", "private")):
        out.append(f"cuda(threads={threads},rows={rows},compact={compact},prefetch={pf},lowcard={lowcard})")
    return out


# the default flavor heads every grid: it is the chooser's "method without it"
GRIDS = {k: [DEFAULT] + g() for k, g in
         (("scan", _scan_grid), ("hash", _hash_grid), ("join", _join_grid), ("star", _star_grid))}
KINDS = tuple(GRIDS)
# every candidate of every kind (the chooser's outputs), the default first
CANDIDATES = [DEFAULT] + sorted({c for g in GRIDS.values() for c in g} - {DEFAULT})

FEATURE_NAMES = ["log2_rows", "log2_probed_build_rows", "log2_groups_bound", "log2_key_domain", "filters",
                 "probes", "probes_n", "aggregates", "bytes_per_row", "selectivity", "zipf",
                 "sink_global", "sink_dense", "sink_hash", "sink_emit"] + [f"kind_{k}" for k in KINDS]


def fact_pipeline(desc):
    """The pipeline that produces the query's result (the fact pipeline)."""
    pipes = desc["pipelines"]
    return next((p for p in pipes if p["result"]), max(pipes, key=lambda p: p["rows"]))


def kind_of(desc):
    """Pipeline kind of a lowered plan (see GRIDS)."""
    p = fact_pipeline(desc)
    if p["probes"] >= 2:
        return "star"
    if p["probes"] == 1:
        return "join"
    if p["sink"] == "aggr_hash":
        return "hash"
    return "scan"


def plan_features(desc, selectivity=1.0, zipf=0.0):
    """Feature vector (FEATURE_NAMES) of a lowered plan (Engine.describe / vc_plan_describe).
    selectivity (fraction of fact rows that reach the sink) and zipf (key skew) are data
    statistics the plan does not hold: the caller's estimates, else 1.0 and 0.0."""
    p = fact_pipeline(desc)
    rows = max(p["rows"], 1)
    kind = kind_of(desc)
    lg = lambda x: math.log2(max(float(x), 1.0))
    return np.array([lg(rows), lg(p["probed_build_rows"] + 1), lg(p["groups_bound"]), lg(p["key_domain"]),
                     p["filters"], p["probes"], p["probes_n"], p["aggregates"] / 8.0,
                     p["scan_bytes"] / rows / 32.0, float(selectivity), float(zipf),
                     float(p["sink"] == "aggr_global"), float(p["sink"] == "aggr_dense"),
                     float(p["sink"] == "aggr_hash"), float(p["sink"] == "emit")] +
                    [float(kind == k) for k in KINDS], dtype=np.float32)


def _spec_params(spec):
    tmpl, _, rest = spec.partition(":")
    out = {}
    for item in rest.split(","):
        if "=" in item:
            k, v = item.split("=", 1)
            out[k] = float(v)
    return tmpl, out


def spec_statistics(spec):
    """(selectivity, zipf) of a synthetic workload spec: the statistics its generator fixes."""
    tmpl, p = _spec_params(spec)
    if tmpl == "sel_aggr":
        return p.get("sel", 2436 / 2526.0), 0.0
    if tmpl == "join_aggr":
        return p.get("sel", 0.2), 0.0
    if tmpl == "groupby":
        return 1.0, p.get("zipf", 0.0)
    if tmpl == "star":
        return 1 / 875.0, 0.0
    return 1.0, 0.0


_describe_cache = {}


def describe_spec(spec):
    """Lowered-plan description of a workload spec (an offline engine: no device, no compile)."""
    if spec not in _describe_cache:
        w = workload(spec)
        e = Engine(offline=True)
        e.load_workload(w)
        _describe_cache[spec] = e.describe(w.plan)
        e.close()
    return _describe_cache[spec]


def features(spec):
    """Feature vector of a workload spec: its lowered plan plus the generator's statistics."""
    sel, zipf = spec_statistics(spec)
    return plan_features(describe_spec(spec), sel, zipf)


def candidates_for(desc):
    return GRIDS[kind_of(desc)]


# ---------------------------------------------------------------------------- run logging


class RunLog:
    """Run records in the reference's SQLite `runs` table (compiler.cpp:100-106; columns it has
    no counterpart for stay NULL) and/or a JSONL file."""

    def __init__(self, sqlite_path=None, jsonl_path=None):
        self.db = None
        self.jsonl = jsonl_path
        if sqlite_path:
            self.db = sqlite3.connect(sqlite_path)
            self.db.execute(
                "CREATE TABLE IF NOT EXISTS runs(id INTEGER PRIMARY KEY AUTOINCREMENT, t TIMESTAMP, mode TEXT, "
                "query TEXT, result TEXT, rep INTEGER, time_ms REAL NULL, tuples REAL NULL, cycles REAL NULL, "
                "instructions REAL NULL, L1misses REAL NULL, LLCmisses REAL NULL, branchmisses REAL NULL, "
                "taskclock REAL NULL, threads INTEGER, cgen_ms REAL NULL, ccomp_ms REAL NULL, default_blend TEXT, "
                "key_check_blend TEXT, aggregates_blend TEXT, backend TEXT, scale_factor INTEGER, "
                "pipeline_flavor TEXT, full_blend TEXT)")

    def record(self, mode, query, flavor, result, rep, time_ms, tuples, ccomp_ms=None):
        if self.db is not None:
            self.db.execute(
                "INSERT INTO runs(t, mode, query, result, rep, time_ms, tuples, threads, ccomp_ms, default_blend, "
                "backend, scale_factor, full_blend) VALUES (datetime('now','localtime'), ?, ?, ?, ?, ?, ?, 1, ?, ?, "
                "'cuda', 0, ?)", (mode, query, result, rep, time_ms, tuples, ccomp_ms, flavor, flavor))
            self.db.commit()

    def record_search(self, spec, times, feats):
        if self.jsonl:
            with open(self.jsonl, "a") as f:
                f.write(json.dumps({"spec": spec, "features": feats.tolist(), "times_ms": times}) + "\n")

    def close(self):
        if self.db is not None:
            self.db.close()
            self.db = None


# ---------------------------------------------------------------------------- search


def autotune(spec, candidates=None, reps=5, log_path=None, engine=None, device=0, sqlite_path=None, mode="full"):
    """Exhaustive search: {flavor: median device ms} over the workload kind's grid (or the
    given candidates); candidates the device rejects are left out."""
    own = engine is None
    eng = engine or Engine(device)
    w = workload(spec)
    if own:
        eng.load_workload(w, on_device=True)
    if candidates is None:
        candidates = candidates_for(describe_spec(spec))
    log = RunLog(sqlite_path, log_path)
    times = {}
    for fl in candidates:
        t0 = time.perf_counter()
        try:
            q = eng.query(w.plan, fl)
        except VoilaError as e:
            log.record(mode, spec, fl, f"EXCEPT '{e}'", 0, None, w.fact_rows)
            continue
        ccomp = (time.perf_counter() - t0) * 1e3
        q.time(1)  # warm-up: module load, first-touch of tables
        ts = q.time(reps)
        times[fl] = float(np.median(ts))
        for r, t in enumerate(ts):
            log.record(mode, spec, fl, "OK", r, float(t), w.fact_rows, ccomp)
        q.close()
    log.record_search(spec, times, features(spec))
    log.close()
    if own:
        eng.close()
    return times


def explore(spec, mode="full", sample=16, seed=1, reps=3, sqlite_path=None, log_path=None, engine=None):
    """The reference explorer's modes over the CUDA flavor grid: 'full' times every candidate
    of the workload's kind, 'sample' a seeded random subset of `sample` of them (the default
    flavor always included).  Returns {flavor: ms}."""
    cands = candidates_for(describe_spec(spec))
    if mode == "sample":
        rng = np.random.default_rng(seed)
        pick = rng.choice(len(cands), size=min(sample, len(cands)), replace=False)
        cands = [DEFAULT] + [cands[i] for i in sorted(pick) if cands[i] != DEFAULT]
    elif mode != "full":
        raise ValueError("mode must be full or sample")
    return autotune(spec, candidates=cands, reps=reps, log_path=log_path, engine=engine,
                    sqlite_path=sqlite_path, mode=mode)


# knobs a single pipeline may take (hash and graph stay query-wide)
PIPE_GRID = [f"cuda(threads={t},rows={r},prefetch={pf})" for t in (128, 256, 512) for r in (2, 4, 8) for pf in (0, 1)]


def backtrack(spec, base=None, reps=3, sqlite_path=None, log_path=None, engine=None, device=0):
    """The reference explorer's per-pipeline backtracking (explorer.cpp:111-134) over CUDA
    flavors: starting from `base` (default: the best of the workload kind's grid), each pipeline in
    turn tries every PIPE_GRID setting as a "p<id>=cuda(...)" override while the others keep
    their current choice, and keeps the fastest.  Returns (flavor string, ms)."""
    own = engine is None
    eng = engine or Engine(device)
    w = workload(spec)
    if own:
        eng.load_workload(w, on_device=True)
    log = RunLog(sqlite_path, log_path)
    if base is None:
        times = autotune(spec, reps=reps, engine=eng)
        base = min(times, key=times.get)

    def timed(fl):
        try:
            q = eng.query(w.plan, fl)
        except VoilaError as e:
            log.record("backtrack", spec, fl, f"EXCEPT '{e}'", 0, None, w.fact_rows)
            return None
        q.time(1)
        ts = q.time(reps)
        q.close()
        for r, t in enumerate(ts):
            log.record("backtrack", spec, fl, "OK", r, float(t), w.fact_rows)
        return float(np.median(ts))

    best, best_ms = base, timed(base)
    overrides = {}
    for pipe in range(len(eng.describe(w.plan, base)["pipelines"])):
        for cand in PIPE_GRID:
            trial = dict(overrides)
            trial[pipe] = cand
            fl = base + "".join(f";p{k}={v}" for k, v in sorted(trial.items()))
            ms = timed(fl)
            if ms is not None and ms < best_ms:
                best, best_ms, overrides = fl, ms, trial
    log.close()
    if own:
        eng.close()
    return best, best_ms


def load_log(path):
    rows = []
    if os.path.exists(path):
        with open(path) as f:
            for line in f:
                line = line.strip()
                if line:
                    rows.append(json.loads(line))
    return rows


# ---------------------------------------------------------------------------- learned chooser


class Chooser:
    """MLP over plan features predicting log2(time / median time) of each candidate."""

    def __init__(self, candidates=CANDIDATES, hidden=64, seed=7, device=0):
        self.candidates = list(candidates)
        self.index = {c: i for i, c in enumerate(self.candidates)}
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
            med = float(np.median(list(t.values())))
            for c, ms in t.items():
                j = self.index.get(c)
                if j is not None and ms > 0:
                    T[i, j] = math.log2(ms / med)
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

    def choose(self, spec_or_features, allowed=None):
        """The candidate with the lowest predicted time among `allowed` (default: the grid of
        the workload's kind when given a spec, else every candidate)."""
        if isinstance(spec_or_features, str):
            f = features(spec_or_features)
            allowed = allowed or candidates_for(describe_spec(spec_or_features))
        else:
            f = spec_or_features
        pred = self.predict(f)[0]
        idx = [self.index[c] for c in allowed if c in self.index] if allowed else range(len(self.candidates))
        return self.candidates[min(idx, key=lambda j: pred[j])]

    def choose_for_plan(self, engine, plan, selectivity=1.0, zipf=0.0):
        """Flavor for plan text on an engine holding its tables: featurized from the lowered plan."""
        desc = engine.describe(plan)
        return self.choose(plan_features(desc, selectivity, zipf), allowed=candidates_for(desc))


def evaluate(chooser, records):
    """Per record: time of the chosen, exhaustive-best and default flavors (the chooser picks
    among the candidates the record timed)."""
    out = []
    for r in records:
        t = r["times_ms"]
        pick = chooser.choose(np.asarray(r["features"], dtype=np.float32), allowed=list(t))
        best = min(t.values())
        out.append({"spec": r["spec"], "chosen": pick, "chosen_ms": t[pick], "best_ms": best,
                    "best": min(t, key=t.get), "default_ms": t.get(DEFAULT, max(t.values()))})
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
