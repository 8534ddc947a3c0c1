"""Benchmark of the CUDA flavor on VOILA's hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload config4] [--impl ours|reference]

A step is one run of the workload's query (all of its fused pipelines: dimension/join-table
builds, the fused probe chain + aggregation, result publication) over one batch of synthetic
input resident in HBM.  Default workload: the largest single-GPU configuration, the star join
over a 60,000,000-row fact table (4 dimension probes, group by year and region).  `value` is
fact rows per second over the whole job; between timed steps L2 is flushed by writing a
256 MiB buffer (the fact table, 1.92 GB, is also far larger than L2).  `e2e` is the same
metric through the public C ABI with the inputs uploaded from pinned host memory and the
result read back every step.

Under torchrun (N > 1) every rank runs the same query over its own fact shard (weak
scaling) and the partial aggregates are merged by the exchange step of shards.py (the
reference's flush2partitions + re-aggregation) inside the timed region.

--impl reference times the reference's own CPU implementation (its hyper and vectorwise
flavors compiled from source into oracle/_ref, all host threads) on the same workload; if
that build is not usable on this host it falls back to the numpy port of the oracle.

--workload config5 times the mixed batch (256 seeded pipelines) one query after another with
exhaustively tuned flavors against a batch with learned flavors.  Environment knobs:
VC_BATCH_N / VC_BATCH_MAX_ROWS (the mix), VC_TRAIN_N / VC_TUNE_REPS (the chooser's training
set and the autotuner's repetitions), VC_BATCH_SOLO_ROWS (queries with a pipeline of at least
this many rows run as their own launches after the persistent kernel; 0 = all inside it) and
VC_CONFIG5_FLAVORS=default (both arms on the default flavor, no tuning).
--device-only and --host-resident-only run just the query, --steps times, for a profiler.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

WORKLOADS = {
    "config1": "sel_aggr:rows=6000000,seed=1",
    "config2": "join_aggr:build=1500000,probe=6000000,sel=0.2,seed=2",
    "config3": "groupby:rows=6000000,keys=1500000,zipf=1.25,seed=3",
    "config4": "star:rows=60000000,seed=4",
}
REF_NAMES = {"sel_aggr": "sel_aggr", "join_aggr": "join_aggr", "groupby": "groupby", "star": "star"}
METRIC = "fact rows/s (fact pipeline)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--workload", default="config4")
    ap.add_argument("--flavor", default="")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--host-resident-only", action="store_true",
                    help="run only the query over host-resident columns, --steps times (for a profiler)")
    ap.add_argument("--device-only", action="store_true",
                    help="run only the query over device-resident columns, --steps times (for a profiler)")
    return ap.parse_args()


def spec_of(name, rank=0):
    spec = WORKLOADS.get(name, name)
    if rank:
        # each rank generates its own tables from its own seed
        spec = spec.replace("seed=", f"seed={rank}00")
    return spec


# ---------------------------------------------------------------------------- clocks


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        mhz, maxes, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                mhz.append(float(f[1]))
                maxes.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not mhz:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(mhz), "sm_max_mhz": max(maxes), "reasons": sorted(reasons),
                "samples": len(mhz)}


# ---------------------------------------------------------------------------- CPU baseline


def _ref_dir():
    d = os.path.join(REPO, "oracle", "_ref", "avx512")
    try:
        with open("/proc/cpuinfo") as f:
            if "avx512f" not in f.read():
                return None
    except OSError:
        return None
    return d if os.path.exists(os.path.join(d, "ref_run")) else None


def reference_cpu(spec, reps, warmup, threads=None):
    """Times the reference's generated query libraries (hyper and vectorwise) with ref_run.
    Returns ({flavor: [ms per rep]}, fact rows) or (None, None) when the reference build is
    unavailable.  Runs only the reference's own code: nothing of this package is loaded."""
    d = _ref_dir()
    if d is None:
        return None, None
    threads = threads or os.cpu_count()
    tmpl = spec.split(":")[0]
    out, rows = {}, None
    for fl in ("hyper", "vectorwise"):
        lib = os.path.join(d, f"q_{REF_NAMES[tmpl]}_{fl}.so")
        if not os.path.exists(lib):
            continue
        r = subprocess.run([os.path.join(d, "ref_run"), "--workload", spec, "--lib", lib, "--flavor", fl,
                            "--threads", str(threads), "--reps", str(reps + warmup), "--no-result", "1"],
                           capture_output=True, text=True, timeout=1800)
        if r.returncode != 0:
            continue
        info = json.loads(r.stdout.strip().splitlines()[-1])
        out[fl] = info["times_ms"][warmup:]
        rows = int(info["rows"])
    return (out or None), rows


def port_cpu(spec, reps):
    """Times the numpy oracle port (single process) on the workload."""
    from oracle.voila_oracle import run_plan
    from vldb_voila_b200 import generate_workload_host, workload
    w = workload(spec)
    data = generate_workload_host(w)
    times = []
    for _ in range(reps):
        t = time.perf_counter()
        run_plan(w.plan, data)
        times.append((time.perf_counter() - t) * 1e3)
    return times


def cpu_baseline(spec, fact_rows, reps=5, warmup=1):
    ref, _ = reference_cpu(spec, reps, warmup)
    if ref:
        best = min(ref, key=lambda k: statistics.median(ref[k]))
        ms = statistics.median(ref[best])
        return {"value": fact_rows / (ms / 1e3), "unit": "fact rows/s", "cores": os.cpu_count(),
                "kind": "reference", "flavor": best,
                "flavors_ms": {k: round(statistics.median(v), 3) for k, v in ref.items()},
                "sample": f"the full workload {spec}, {reps} hot runs (qrun interval, no result printing), "
                          f"median; reference built from source, -march=skylake-avx512"}
    ms = statistics.median(port_cpu(spec, max(1, reps // 2)))
    return {"value": fact_rows / (ms / 1e3), "unit": "fact rows/s", "cores": 1, "kind": "port",
            "sample": f"the full workload {spec} through the numpy oracle, median"}


# ---------------------------------------------------------------------------- reference arm


def run_reference_arm(args):
    """The reference's own CPU path on this host.  Only the reference's compiled code runs
    (ref_run + its generated query library); this package is imported only by the fallback
    to the numpy port, on hosts where the reference cannot run."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    spec = spec_of(args.workload)
    t0 = time.perf_counter()
    ref, fact_rows = reference_cpu(spec, args.steps, args.warmup)
    if ref:
        best = min(ref, key=lambda k: statistics.median(ref[k]))
        times = ref[best]
        kind, cores = "reference", os.cpu_count()
        sample = f"{spec}: each step one full hot run (qrun) of the reference's {best} flavor"
    else:
        from vldb_voila_b200 import workload
        fact_rows = workload(spec).fact_rows
        times = port_cpu(spec, args.steps)
        kind, cores, best = "port", 1, "numpy"
        sample = f"{spec}: each step one run of the numpy oracle port"
    ms = statistics.mean(times)
    value = fact_rows / (ms / 1e3)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "fact rows/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": spec, "template": spec.split(":")[0], "fact_rows": fact_rows, "flavor": best},
        "cpu_baseline": {"value": value, "unit": "fact rows/s", "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "fact rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": round(time.perf_counter() - t0, 1),
    }
    if ref:
        line["flavors_ms"] = {k: round(statistics.mean(v), 3) for k, v in ref.items()}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------- our arm


def run_host_resident_only(args):
    """The workload's query over columns left in pinned host memory, run --steps times: what a
    profiler captures to measure the PCIe bytes of a host-resident step."""
    import numpy as np
    import torch

    from vldb_voila_b200 import Engine, generate_workload_host, workload
    w = workload(spec_of(args.workload))
    host = generate_workload_host(w)
    eng = Engine(0)
    keep = []
    for t, rows in w.tables.items():
        eng.create_table(t, rows)
    for c in w.columns:
        eng.add_column(c.table, c.name, c.type, c.lo, c.hi)
        a = np.ascontiguousarray(host[c.table][c.name])
        keep.append(torch.from_numpy(a.view(np.uint8) if a.dtype != np.uint8 else a).pin_memory())
        eng.attach_host(c.table, c.name, keep[-1].data_ptr())
    q = eng.query(w.plan, args.flavor)
    for _ in range(args.steps):
        q.run()
        res = q.result()
    print(json.dumps({"workload": w.spec, "steps": args.steps, "result_rows": int(len(res))}))
    return 0


def run_device_only(args):
    """The workload's query over columns generated in HBM, run --steps times with no timing:
    what a profiler captures for a kernel's counters."""
    import torch

    from vldb_voila_b200 import Engine, workload
    w = workload(spec_of(args.workload))
    eng = Engine(0)
    eng.load_workload(w, on_device=True)
    torch.cuda.synchronize()
    q = eng.query(w.plan, args.flavor)
    for _ in range(args.steps):
        q.run()
    res = q.result()
    print(json.dumps({"workload": w.spec, "flavor": q.info()["flavor"], "steps": args.steps,
                      "result_rows": int(len(res))}))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.host_resident_only:
        return run_host_resident_only(args)
    if args.device_only:
        return run_device_only(args)

    import numpy as np
    import torch
    import torch.distributed as dist

    from vldb_voila_b200 import Engine, workload
    from vldb_voila_b200.engine import stream_read

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    spec = spec_of(args.workload, rank)
    w = workload(spec)
    eng = Engine(local)
    stream = torch.cuda.current_stream()
    eng.load_workload(w, on_device=True, stream=stream)
    torch.cuda.synchronize()
    q = eng.query(w.plan, args.flavor)
    info = q.info()
    kernels = [k["name"] for k in info["kernels"]]
    dom = [i for i, k in enumerate(info["kernels"]) if k["dominant"]][0]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def step():
        q.run(stream)

    from vldb_voila_b200.shards import merge_partials, plan_group_keys

    nkeys = plan_group_keys(w.plan)

    def combine():
        """Exchange step: merge the ranks' partial aggregates (vldb_voila_b200/shards.py)."""
        if world > 1:
            part = q.result()
            merge_partials(part, nkeys, part.shape[1], device="cuda")

    for i in range(args.warmup):
        flush.fill_(i & 0xff)
        step()
        combine()
    torch.cuda.synchronize()

    step_ms, dom_ms, all_ms = [], [], []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        # timed steps: device time of each step, the exchange step included (no per-kernel
        # events inside)
        for i in range(args.steps):
            flush.fill_((i + 1) & 0xff)
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            step()
            combine()
            ev1.record(stream)
            ev1.synchronize()
            step_ms.append(ev0.elapsed_time(ev1))
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        # profiled pass: per-kernel device times from events on the launch stream
        q.profile(True)
        for i in range(args.steps):
            flush.fill_((i + 1) & 0xff)
            step()
            combine()
            t = q.timings()
            dom_ms.append(t[dom][1])
            all_ms.append([x[1] for x in t])
        q.profile(False)
        # the floor: one plain streaming read (vc_stream_read) of the same byte count as the
        # dominant kernel's algorithmic bytes, L2 flushed the same way
        floor_buf = torch.empty(max(w.probe_bytes, 16), dtype=torch.uint8, device="cuda")
        floor_buf.fill_(1)
        floor_out = torch.zeros(1, dtype=torch.int64, device="cuda")
        floor_ms = []
        for i in range(min(args.steps, 50) + 3):
            flush.fill_((i + 3) & 0xff)
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            stream_read(floor_buf.data_ptr(), w.probe_bytes, floor_out.data_ptr(), stream)
            ev1.record(stream)
            ev1.synchronize()
            if i >= 3:
                floor_ms.append(ev0.elapsed_time(ev1))
        del floor_buf
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = statistics.mean(step_ms)
    if world > 1:
        tt = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    value = world * w.fact_rows / (ms / 1e3)

    # e2e through the public API: pinned host inputs uploaded every step, result read back
    from vldb_voila_b200.engine import generate_workload_host
    host = generate_workload_host(w)
    pinned = {}
    h2d = 0
    for c in w.columns:
        a = host[c.table][c.name]
        t = torch.from_numpy(a.view(np.uint8) if a.dtype != np.uint8 else a).pin_memory()
        pinned[(c.table, c.name)] = (t, len(a))
        h2d += a.nbytes
    e2e_ms = []
    d2h = 0
    # the caller's result buffer, reused across steps like any steady-state consumer would
    rr, rc = q.shape()
    resbuf = np.zeros(max(2 * rr * rc, 1), dtype=np.int64)
    for i in range(args.warmup + args.steps):
        flush.fill_(i & 0xff)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for (tb, cn), (t, n) in pinned.items():
            eng.upload_ptr(tb, cn, t.data_ptr(), n, stream)
        q.run(stream)
        res = q.result(out=resbuf)
        combine()
        t1 = time.perf_counter()
        d2h = res.nbytes + 16
        if i >= args.warmup:
            e2e_ms.append((t1 - t0) * 1e3)
    e2e_copy = statistics.mean(e2e_ms)

    # e2e with host-resident columns: the same pinned buffers registered as the columns of a
    # second engine, read in place by the kernels over PCIe (only the bytes a step touches
    # cross the bus), and the result read back every step
    engh = Engine(local)
    for t, rows in w.tables.items():
        engh.create_table(t, rows)
    for c in w.columns:
        engh.add_column(c.table, c.name, c.type, c.lo, c.hi)
        t, n = pinned[(c.table, c.name)]
        engh.attach_host(c.table, c.name, t.data_ptr())
    qh = engh.query(w.plan, args.flavor)
    e2eh_ms = []
    for i in range(args.warmup + args.steps):
        flush.fill_(i & 0xff)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        qh.run(stream)
        resh = qh.result(out=resbuf)
        combine()
        t1 = time.perf_counter()
        if i >= args.warmup:
            e2eh_ms.append((t1 - t0) * 1e3)
    e2e_host = statistics.mean(e2eh_ms)
    assert np.array_equal(np.sort(qh.result(), axis=0), np.sort(q.result(), axis=0)), "host-resident result differs"
    qh.close()
    engh.close()
    pcie = None
    ppath = os.path.join(REPO, "profiles", "pcie.json")
    if os.path.exists(ppath):
        with open(ppath) as f:
            pc = json.load(f).get(w.template)
        if pc:
            pcie = int(round(pc["read_bytes_per_fact_row"] * w.fact_rows))
    if world > 1:
        tt = torch.tensor([e2e_copy, e2e_host], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_copy, e2e_host = float(tt[0].item()), float(tt[1].item())
    e2e_modes = {
        "copy": {"value": world * w.fact_rows / (e2e_copy / 1e3), "unit": "fact rows/s", "ms_per_step": e2e_copy,
                 "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                 "mode": "every column copied from pinned host memory (cudaMemcpyAsync), then the query"},
        "host_resident": {"value": world * w.fact_rows / (e2e_host / 1e3), "unit": "fact rows/s",
                          "ms_per_step": e2e_host, "h2d_bytes_per_step": pcie if pcie is not None else h2d,
                          "h2d_bytes_measured": pcie is not None, "d2h_bytes_per_step": d2h,
                          "mode": "columns stay in pinned host memory; the kernels read what they need over PCIe"},
    }
    e2e_best = min(e2e_modes, key=lambda k: e2e_modes[k]["ms_per_step"])

    peaks = {}
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    dom_avg = statistics.mean(dom_ms)
    traffic = None
    tpath = os.path.join(REPO, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            t = json.load(f).get(w.template)
        # per-launch DRAM bytes of the dominant kernel (ncu), per fact row so that it scales
        # to the workload's size
        if isinstance(t, dict):
            traffic = int(round(t["bytes_per_fact_row"] * w.fact_rows))
        elif t is not None:
            traffic = int(t)
    # achieved bandwidth: the dominant kernel's algorithmic bytes (every column it scans, read
    # once) per launch time -- except where the kernel skips most of those bytes by design
    # (the star probe chain gathers the later columns only for rows that survive the first
    # probe): there the DRAM bytes ncu measured per launch are what it moves
    basis_bytes, basis = w.probe_bytes, "algorithmic bytes (scanned columns read once)"
    if traffic is not None and traffic < 0.8 * w.probe_bytes:
        basis_bytes, basis = traffic, "measured DRAM bytes per launch (ncu; the kernel skips unneeded column sectors)"
    achieved = basis_bytes / (dom_avg / 1e3) / 1e9
    floor_gbs = w.probe_bytes / (statistics.mean(floor_ms) / 1e3) / 1e9

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "fact rows/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "int64",
            "data": "synthetic (seeded generator, resident in HBM)",
            "config": {"workload": spec, "template": w.template, "fact_rows": w.fact_rows,
                       "flavor": info["flavor"], "l2": "flushed between timed steps (256 MiB write)",
                       "parallelism": f"dp{world}" if world > 1 else "single GPU"},
            "e2e": e2e_modes[e2e_best],
            "e2e_modes": e2e_modes,
            "roofline": {"bound": "hbm", "kernel": kernels[dom], "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "basis": basis,
                         "algorithmic_bytes": w.probe_bytes,
                         "logical_gbs": w.probe_bytes / (dom_avg / 1e3) / 1e9,
                         "kernel_ms": dom_avg,
                         "kernel_share_of_step": dom_avg / ms,
                         "kernel_rows_per_s": w.fact_rows / (dom_avg / 1e3),
                         "stream_read_floor": {"gbs": floor_gbs, "frac_of_peak": floor_gbs / peak,
                                               "kernel_over_floor": statistics.mean(floor_ms) / dom_avg,
                                               "method": "vc_stream_read over the algorithmic byte count, same L2 flush"},
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if "hbm_gbs" in peaks
                         else "fallback 6650 GB/s"},
            "gpu_launches": len(kernels) * args.steps,
            "kernel_ms": {k: round(statistics.mean(r[i] for r in all_ms), 5) for i, k in enumerate(kernels)},
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(spec, w.fact_rows)
        print(json.dumps(line))
    q.close()
    eng.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_config5(args):
    """The mixed batch: 256 seeded pipelines (sizes log-uniform 1e4..6e7 rows, selectivities
    1-100 %, Zipf 0-1.25) run (a) one query after another with exhaustively tuned flavors and
    (b) as one persistent-kernel batch with learned-chooser flavors.  Also reports the learned
    choices' time against the exhaustive best on these held-out pipelines."""
    import numpy as np
    import torch

    from vldb_voila_b200 import chooser as ch
    from vldb_voila_b200 import Engine, workload
    from vldb_voila_b200.engine import Batch, batch_specs

    torch.cuda.set_device(0)
    n = int(os.environ.get("VC_BATCH_N", "256"))
    max_rows = int(float(os.environ.get("VC_BATCH_MAX_ROWS", "60000000")))
    specs = batch_specs(n, 5, 10_000, max_rows)
    t0 = time.time()
    # VC_CONFIG5_FLAVORS=default: both arms run the default flavor (no tuning, no chooser), which
    # isolates batching from flavor choice
    tune = os.environ.get("VC_CONFIG5_FLAVORS", "tuned") != "default"
    reps = int(os.environ.get("VC_TUNE_REPS", "3"))
    train, loss, chooser = [], None, None
    if tune:
        # learned chooser: trained on autotuner timings of separate seeded workloads
        train = ch.training_specs(int(os.environ.get("VC_TRAIN_N", "48")), seed=21, min_rows=100_000,
                                  max_rows=20_000_000)
        records = [{"spec": s, "features": ch.features(s).tolist(), "times_ms": ch.autotune(s, reps=reps)}
                   for s in train]
        chooser = ch.Chooser()
        loss = chooser.fit(records)
    t_train = time.time() - t0

    engines, queries_tuned, tuned, learned, records5 = [], [], [], [], []
    for s in specs:
        w = workload(s)
        e = Engine(0)
        e.load_workload(w, on_device=True)
        if tune:
            times = ch.autotune(s, reps=reps, engine=e)
            best = min(times, key=times.get)
            pick = chooser.choose(s)
            records5.append({"spec": s, "best": best, "best_ms": times[best], "chosen": pick,
                             "chosen_ms": times[pick], "default_ms": times[ch.DEFAULT]})
        else:
            best = pick = ch.DEFAULT
        tuned.append(best)
        learned.append(pick)
        engines.append(e)
        queries_tuned.append(e.query(w.plan, best))
    torch.cuda.synchronize()
    t_tune = time.time() - t0 - t_train

    stream = torch.cuda.current_stream()
    # (a) per-pipeline launches, one query after another, tuned flavors
    for q in queries_tuned[:8]:
        q.run(stream)
    torch.cuda.synchronize()
    plain_ms, plain_lat = [], []
    for rep in range(args.steps):
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(len(queries_tuned) + 1)]
        evs[0].record(stream)
        for i, q in enumerate(queries_tuned):
            q.run(stream)
            evs[i + 1].record(stream)
        evs[-1].synchronize()
        plain_ms.append(evs[0].elapsed_time(evs[-1]))
        plain_lat = [evs[0].elapsed_time(e) * 1000.0 for e in evs[1:]]
        plain_each = [evs[i].elapsed_time(evs[i + 1]) for i in range(len(queries_tuned))]
    expect = [q.result_lines() for q in queries_tuned]

    # (b) one persistent kernel over all pipelines, learned flavors
    # batched pipelines build their join tables in place (dense or direct hash; one work
    # phase per table): a staged build becomes the automatic choice
    batch_flavors = [f.replace("build=staged", "build=auto") for f in learned]
    queries_learned = [e.query(workload(s).plan, f) for e, s, f in zip(engines, specs, batch_flavors)]
    # queries whose fact pipeline fills the GPU by itself run as their own launches after the
    # persistent kernel (vc_batch_new_split), the rest inside it
    solo_rows = int(float(os.environ.get("VC_BATCH_SOLO_ROWS", str(1 << 22))))

    def time_batch(bt):
        for _ in range(2):
            bt.run(stream)
            bt.wait()
        ms_list, lat = [], []
        for rep in range(args.steps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            bt.run(stream)
            b.record(stream)
            bt.wait()
            ms_list.append(a.elapsed_time(b))
            lat = bt.latencies_us()
        return ms_list, lat, all(q.result_lines() == e for q, e in zip(queries_learned, expect))

    batch = Batch(queries_learned, threads=256, tiles_per_item=16, solo_rows=solo_rows)
    batch_ms, batch_lat, exact = time_batch(batch)
    unsplit = None
    if solo_rows > 0:
        # the same queries all inside the persistent kernel, for comparison
        batch0 = Batch(queries_learned, threads=256, tiles_per_item=16)
        ms0, _, exact0 = time_batch(batch0)
        unsplit = {"batched_ms": statistics.median(ms0), "results_identical": exact0,
                   "value": statistics.median(plain_ms) / statistics.median(ms0)}
        exact = exact and exact0
        batch0.close()

    ratio = [r["chosen_ms"] / r["best_ms"] for r in records5]
    rows = sum(workload(s).fact_rows for s in specs)
    p = lambda xs, k: float(np.percentile(xs, k))
    line = {
        "metric": "mixed batch of pipelines: total time, batched persistent kernel vs per-pipeline launches",
        "value": statistics.median(plain_ms) / statistics.median(batch_ms), "unit": "x (per-pipeline / batched)",
        "higher_is_better": True, "n_gpus": 1, "steps": args.steps, "dtype": "int64", "data": "synthetic",
        "config": {"workload": f"{n} pipelines batch_specs(seed=5, 1e4..{max_rows:.0e} rows)", "fact_rows": rows,
                   "batch_info": batch.info()},
        "batched_ms": statistics.median(batch_ms), "per_pipeline_ms": statistics.median(plain_ms),
        "batched_rows_per_s": rows / (statistics.median(batch_ms) / 1e3),
        "latency_us": {"batched_p50": p(batch_lat, 50), "batched_p99": p(batch_lat, 99),
                       "per_pipeline_p50": p(plain_lat, 50), "per_pipeline_p99": p(plain_lat, 99)},
        "results_identical": exact,
        "solo_rows": solo_rows,
        "per_pipeline_ms_by_template": {t: round(sum(ms for s, ms in zip(specs, plain_each) if s.startswith(t)), 3)
                                        for t in sorted({s.split(":")[0] for s in specs})},
        "flavors": "per-pipeline arm: exhaustively tuned; batch: learned" if tune else "default flavor in both arms",
        "all_in_one_kernel": unsplit,
        "chooser": {"train_workloads": len(train), "train_loss": loss, "heldout_pipelines": len(records5),
                    "geomean_chosen_over_best": float(np.exp(np.mean(np.log(ratio)))),
                    "max_chosen_over_best": float(np.max(ratio)),
                    "within_10pct_fraction": float(np.mean([r <= 1.10 for r in ratio])),
                    "sum_chosen_ms": sum(r["chosen_ms"] for r in records5),
                    "sum_best_ms": sum(r["best_ms"] for r in records5),
                    "sum_default_ms": sum(r["default_ms"] for r in records5)} if records5 else None,
        "setup_s": {"train": round(t_train, 1), "tune": round(t_tune, 1)},
    }
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    if "--workload" in sys.argv and sys.argv[sys.argv.index("--workload") + 1] == "config5":
        sys.exit(run_config5(parse()))
    sys.exit(main())
