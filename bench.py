#!/usr/bin/env python
"""Benchmark: per-vertex triangle counting on one B200 (or N replicas).

Default workload: R-MAT scale 20 (1,048,576 vertices), edge factor 16,
(a,b,c,d) = (0.57, 0.19, 0.19, 0.05), seed 2; duplicates and self-loops
removed, symmetrised, int32 offsets / int32 sorted adjacency; plain
(per-vertex) mode: r, t, lcc and the global count.  A step is one complete
count of the graph (all launches of one gtc_count call) with the CSR resident
in HBM; L2 is flushed (a 256 MiB write) before every timed step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--config rmat20|er|rgg]

Prints one JSON line.  Under torchrun (N > 1) every rank counts its own
replica of the graph (no collective on the data path; "scaling": "weak") and
the time is the max over ranks.  --impl reference times the reference's own
CPU code (compiled from its sources into oracle/_ref) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "per-vertex TC edges/s"
UNIT = "undirected edges/s"
DTYPE = "int32 ids / int64 counts"
L2_FLUSH_BYTES = 256 << 20

CONFIGS = {
    "rmat20": dict(kind="rmat", scale=20, ef=16, seed=2,
                   label="R-MAT scale 20, edge factor 16, (0.57,0.19,0.19,0.05), seed 2"),
    "er": dict(kind="er", n=16384, deg=16, seed=1,
               label="Erdos-Renyi n=16384, mean degree 16, seed 1"),
    "rgg": dict(kind="rgg", n=1 << 22, deg=12, seed=3,
                label="2D RGG n=4194304, mean degree 12, Morton order, seed 3"),
    "serving": dict(kind="serving", pool=256, seed=5, rates=(1000, 5000, 20000),
                    arrivals_s=1.5,
                    label="Poisson arrivals at 1k, 5k and 20k requests/s; each request a graph "
                          "from the batched-workload generator (pool of 256, seed 5) or, with "
                          "probability 1%, an R-MAT scale 22 edge factor 16 graph; CSRs resident "
                          "in HBM"),
    "ops": dict(kind="ops", pool=256, seed=5, vertices=1 << 16,
                label="the reference-compatible operators on R-MAT scale 20 (kernelCall with int64 "
                      "ids, its vertex-list overload on 65,536 vertices, CSR validation) and the "
                      "pack + batched count of a 256-graph pool of the batched generator (seed 5)"),
    "batched": dict(kind="batched", graphs=4096, seed=4,
                    label="4,096 graphs, n log-uniform in [256, 262144], half ER (mean degree "
                          "U[8,32]), half R-MAT (0.57,0.19,0.19,0.05, edge factor U[8,16]), seed 4; "
                          "concatenated CSR, int64 offsets, int32 graph-local ids"),
}


# DRAM bytes (read + write) of one complete count, summed over its launches
# from one ncu capture of the same workload (dram__bytes_read.sum +
# dram__bytes_write.sum, cold L2 before each launch), read from the committed
# per-workload ncu summary under profiles/ (its "traffic per count:" line).  Far below B_alg: the forward lists and the per-vertex records stay
# in the 126 MB L2, so most probe reads never reach HBM.
def dram_traffic(workload: str) -> dict | None:
    path = os.path.join(ROOT, "profiles", f"dram_per_kernel_{workload}.md")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic per count:"):
                    parts = line.split(":", 1)[1].split()
                    return {"bytes": int(parts[0].replace(",", "")), "source": os.path.relpath(path, ROOT)}
    except OSError:
        pass
    return None


def make_graph(cfg: dict, device):
    from gputrianglecounting_b200 import graphs as G
    if cfg["kind"] == "rmat":
        return G.rmat(cfg["scale"], cfg["ef"], cfg["seed"], device=device)
    if cfg["kind"] == "er":
        return G.erdos_renyi(cfg["n"], cfg["deg"], cfg["seed"], device=device)
    return G.rgg2d(cfg["n"], cfg["deg"], cfg["seed"], device=device)


def graph_config(workload: str, cfg: dict, g, world: int) -> dict:
    """The `config` object of a single-graph line (identical for both arms)."""
    return {"workload": workload, "graph": cfg["label"], "n": g.n, "nnz": g.nnz, "m": g.m,
            "mode": "plain (r, t, lcc, global)", "offsets": "int32",
            "l2": f"GPU arm: flushed before every timed step ({L2_FLUSH_BYTES >> 20} MiB write)",
            "parallelism": f"{world} independent replica(s)"}


def algorithmic_bytes(host_graph) -> dict:
    """B_alg = 4 W + 4 (n+1) + 4 nnz + 8 n + 8 n, W = sum over undirected
    edges of min(d_u, d_v) (the per-unit work model of the hot path)."""
    off = host_graph.off.astype(np.int64)
    ind = host_graph.ind.astype(np.int64)
    n = off.shape[0] - 1
    deg = np.diff(off)
    row = np.repeat(np.arange(n, dtype=np.int64), deg)
    upper = row < ind
    W = int(np.minimum(deg[row[upper]], deg[ind[upper]]).sum())
    nnz = ind.shape[0]
    return {"W": W, "B_alg": 4 * W + 4 * (n + 1) + 4 * nnz + 16 * n}


def measured_peaks() -> tuple[float, str]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks / throttle reasons during timing."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.result = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if self.proc is None:
            return False
        time.sleep(0.2)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) != 6:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[2:]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if sm:
            self.result = {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                           "reasons": sorted(reasons), "samples": len(sm)}
        return False


# --------------------------------------------------------------- reference

class ReferenceTimer:
    """The reference's CPU count timed on the host cores: count_all_trianglesCPU
    (vertex-list overload, src/clusteringCount.cpp:125-155, compiled unchanged
    into oracle/_ref) on the workload's int32 CSR, row by row, with the rows
    spread over all host threads by OpenMP (dynamic, 1) in units: each heavy
    row (cost >= total / (256 threads)) is a unit of its own, the other rows
    form units of up to 64 consecutive ids (the granularity of a
    schedule(dynamic, 64) row loop).  Per-unit times are measured, so the
    full-graph wall time can be estimated without running the whole graph
    every step:

        T_full = max((sum of heavy-unit times + k * sum of sampled light-unit
                      times) / threads, largest unit time)

    which is the lower bound of any schedule on `threads` cores (optimistic
    for the reference).  The heavy units are measured once (calibrate);
    each step times a systematic 1-in-k sample of the light units in order
    of cost (phase = step index), k chosen so a step lasts about step_s.
    A graph whose whole count fits in step_s runs whole every step, and
    T_full is simply its wall time.  Unit cost model (merge steps of the
    reference's count_intersectionsReg for a row): d(v)^2 + sum_{u in N(v)} d(u).
    """

    CHUNK = 64

    def __init__(self, host_graph, threads: int, step_s: float = 2.0):
        from oracle import oracle as O
        self.O = O
        self.threads = threads
        self.step_s = step_s
        off = np.asarray(host_graph.off, np.int64)
        self.off32 = np.ascontiguousarray(off, np.int32)
        self.ind32 = np.ascontiguousarray(host_graph.ind, np.int32)
        self.m = host_graph.m
        n = off.shape[0] - 1
        deg = np.diff(off).astype(np.float64)
        row = np.repeat(np.arange(n, dtype=np.int64), np.diff(off))
        cost = deg * deg + np.bincount(row, weights=deg[self.ind32], minlength=n) + 1.0
        total = float(cost.sum())
        heavy = np.nonzero(cost >= total / (256.0 * threads))[0]
        heavy = heavy[np.argsort(-cost[heavy], kind="stable")]
        is_heavy = np.zeros(n, bool)
        is_heavy[heavy] = True
        light_rows = np.nonzero(~is_heavy)[0]
        chunk_of = light_rows // self.CHUNK
        starts = np.nonzero(np.r_[True, chunk_of[1:] != chunk_of[:-1]])[0] if n else np.zeros(0, int)
        # unit table: heavy rows one per unit, then the light chunks
        self.unit_rows = np.concatenate([heavy, light_rows]).astype(np.int64)
        self.unit_off = np.concatenate([np.arange(heavy.shape[0] + 1),
                                        heavy.shape[0] + np.r_[starts[1:], light_rows.shape[0]]]
                                       ).astype(np.int64) if n else np.zeros(1, np.int64)
        self.n_heavy = int(heavy.shape[0])
        light_cost = np.add.reduceat(cost[light_rows], starts) if light_rows.size else np.zeros(0)
        self.light_units = self.n_heavy + np.argsort(-light_cost, kind="stable")   # cost order
        self.cost_heavy = float(cost[heavy].sum())
        self.cost_light = float(light_cost.sum())
        self.tri = np.zeros(self.ind32.shape[0], np.int64)
        self.r = np.zeros(n, np.int64)
        self.whole = False
        self.k = 1
        self.heavy_ns = np.zeros(0, np.int64)
        self.heavy_wall = 0.0

    def _run(self, units):
        t0 = time.perf_counter()
        ns, _ = self.O.ref_units_timed(self.off32, self.ind32, self.unit_rows, self.unit_off,
                                       units, self.threads, tri=self.tri, r=self.r)
        return ns, time.perf_counter() - t0

    def calibrate(self) -> None:
        """Time the heavy units once and a pilot light sample; choose k."""
        heavy_units = np.arange(self.n_heavy, dtype=np.int64)
        if self.n_heavy:
            self.heavy_ns, self.heavy_wall = self._run(heavy_units)
        nl = self.light_units.shape[0]
        pilot_k = max(1, nl // 512)
        ns, _ = self._run(self.light_units[::pilot_k])
        sample_cost = self.cost_light / pilot_k if nl else 0.0
        rate = (ns.sum() / sample_cost) if sample_cost > 0 else 0.0          # ns per cost unit
        light_est_s = rate * self.cost_light / 1e9
        heavy_s = self.heavy_ns.sum() / 1e9
        est_whole = max((heavy_s + light_est_s) / self.threads,
                        self.heavy_ns.max() / 1e9 if self.n_heavy else 0.0)
        if est_whole <= self.step_s:
            self.whole = True
            self.k = 1
        else:
            self.k = max(1, int(math.ceil(light_est_s / self.threads / self.step_s)))

    def step(self, index: int) -> dict:
        """One timed step; returns its wall time and the full-graph estimate."""
        if self.whole:
            units = np.arange(self.unit_off.shape[0] - 1, dtype=np.int64)
            ns, wall = self._run(units)
            return {"wall_s": wall, "full_s": wall, "units": int(units.shape[0])}
        units = self.light_units[index % self.k::self.k]
        ns, wall = self._run(units)
        hv = self.heavy_ns
        serial = hv.sum() + self.k * ns.sum()
        longest = max(hv.max() if hv.size else 0, ns.max() if ns.size else 0)
        full = max(serial / self.threads, longest) / 1e9
        return {"wall_s": wall, "full_s": full, "units": int(units.shape[0])}

    def describe(self) -> str:
        if self.whole:
            return (f"the whole graph every step: the reference's count_all_trianglesCPU "
                    f"(vertex-list overload, int32 CSR) over all rows, OpenMP dynamic over "
                    f"{self.unit_off.shape[0] - 1} units on {self.threads} threads")
        return (f"the reference's count_all_trianglesCPU (vertex-list overload, int32 CSR) on "
                f"{self.threads} threads; {self.n_heavy} heavy rows (one unit each) timed once "
                f"({self.heavy_wall:.2f} s wall), then each step a systematic 1-in-{self.k} "
                f"sample of the {self.light_units.shape[0]} light 64-row units in cost order; "
                f"full-graph time = max((heavy + {self.k} x sampled unit time) / threads, "
                f"longest unit), a lower bound for any schedule")


def cpu_baseline(host_graph, threads: int) -> dict:
    """The reference's CPU count on this host (calibration + one sampled step)."""
    rt = ReferenceTimer(host_graph, threads)
    rt.calibrate()
    st = rt.step(0)
    return {"value": host_graph.m / st["full_s"], "unit": UNIT, "cores": threads,
            "kind": "reference", "sample": rt.describe(),
            "full_graph_s_estimate": st["full_s"], "step_wall_s": st["wall_s"]}


def run_reference(args, cfg, rank: int) -> None:
    import torch  # noqa: F401  (same environment as the GPU arm)
    from oracle import oracle as O
    if rank != 0:
        return
    threads = O.max_threads()
    if cfg["kind"] in ("batched", "serving"):
        run_reference_batched(args, CONFIGS["batched"], threads)
        return
    if cfg["kind"] == "ops":                # the operators' graph: R-MAT scale 20
        cfg = CONFIGS["rmat20"]
    g = int32_offsets(make_graph(cfg, "cpu").numpy())
    rt = ReferenceTimer(g, threads)
    t0 = time.perf_counter()
    rt.calibrate()
    calib_s = time.perf_counter() - t0
    for w in range(args.warmup):
        rt.step(w)
    steps = [rt.step(args.warmup + k) for k in range(args.steps)]
    full = statistics.mean(st["full_s"] for st in steps)
    wall = statistics.mean(st["wall_s"] for st in steps)
    value = g.m / full
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": wall * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": DTYPE, "data": "synthetic",
        "config": graph_config(args.config, cfg, g, world=args.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": rt.describe(), "full_graph_s_estimate": full,
                         "calibration_s": calib_s},
        "reference_timing": {"ms_per_step": "wall time of each step's sample",
                             "value": "undirected edges / estimated full-graph time",
                             "full_graph_ms_estimate": full * 1e3},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference_batched(args, cfg, threads: int) -> None:
    """Reference CPU code on a bounded sample of the batched workload: every
    64th graph spec (same generator and seeds as the GPU arm, realised with
    the host RNG), each counted whole by the reference's vertex-list
    overload."""
    from gputrianglecounting_b200 import graphs as G
    from oracle import oracle as O
    specs = G.batched_specs(cfg["graphs"], cfg["seed"])[::64]
    sample = [G.make_spec_graph(s, "cpu").numpy() for s in specs]
    preps = [O.ref_prepared(h.off, h.ind) for h in sample]
    m_s = sum(h.m for h in sample)

    def one_pass():
        t0 = time.perf_counter()
        for (o, i) in preps:
            tri = np.zeros(i.shape[0], np.int64)
            r = np.zeros(o.shape[0] - 1, np.int64)
            O.ref_rows_prepared(o, i, None, tri, r, threads)
        return time.perf_counter() - t0
    for _ in range(min(args.warmup, 1)):
        one_pass()
    times = [one_pass() for _ in range(max(1, min(args.steps, 3)))]
    value = m_s / statistics.mean(times)
    line = {
        "impl": "reference", "metric": "batched per-vertex TC edges/s", "value": value,
        "unit": UNIT, "n_gpus": args.gpus, "steps": len(times), "warmup": args.warmup,
        "ms_per_step": statistics.mean(times) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": "batched", "graph": cfg["label"], "sample_graphs": len(sample),
                   "sample_edges": m_s},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"every 64th graph of the batch ({len(sample)} graphs, "
                                   f"{m_s} edges) per step"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ b200

def run_b200(args, name: str, rank: int, world: int, with_baseline: bool = True):
    import torch
    import torch.distributed as dist
    from gputrianglecounting_b200 import api
    from gputrianglecounting_b200 import dist as gdist
    from gputrianglecounting_b200._lib import load as load_lib
    load_lib()

    cfg = CONFIGS[name]
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # generated on the host (deterministic per seed, identical for both arms);
    # int32 offsets, as the workload specifies its CSR
    host = int32_offsets(make_graph(cfg, "cpu").numpy())
    g = host.to(dev)
    torch.cuda.synchronize()
    counter = api.TriangleCounter(dev)
    out = None
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()

    # warm-up (also validates the input once); the launch shape comes from the
    # autotuner (staged search, cached per degree profile), chosen before any
    # timed step
    reason, why = api.validate_csr(g.off, g.ind)
    if reason != 0:
        raise RuntimeError(f"generated graph invalid: {why}")
    from gputrianglecounting_b200 import autotune
    t_tune = time.perf_counter()
    tuning = autotune.autotune(g.off, g.ind, counter=counter, search="staged",
                               cache_path=args.tune_cache)
    tune_s = time.perf_counter() - t_tune
    tune_entry = autotune.tuned_entry(g.off, g.nnz) or {}
    for _ in range(args.warmup):
        out = counter.count(g.off, g.ind, out=out, tuning=tuning)
    torch.cuda.synchronize()

    # device-timed steps, one event pair per step, L2 flushed between steps
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.fill_(k & 0xff)
            evs[k][0].record(stream)
            out = counter.count(g.off, g.ind, out=out, tuning=tuning)
            evs[k][1].record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = gdist.max_over_ranks(sum(step_ms), dev)
    T = out.triangles

    # phase breakdown of one count (events between the pipeline phases)
    phases = phase_breakdown(counter, g, flush, tuning)

    # end to end through the public API with host buffers (pinned), copies
    # inside the timed region
    h_off = torch.from_numpy(host.off).pin_memory()
    h_ind = torch.from_numpy(host.ind).pin_memory()
    h_r = torch.empty(host.n, dtype=torch.int64).pin_memory()
    h_lcc = torch.empty(host.n, dtype=torch.float64).pin_memory()
    h_glob = torch.empty(3, dtype=torch.int64).pin_memory()
    d_off = torch.empty_like(g.off)
    d_ind = torch.empty_like(g.ind)
    e2e_evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
    for k in range(args.warmup + args.steps):
        flush.fill_(k & 0xff)
        if k >= args.warmup:
            e2e_evs[k - args.warmup][0].record(stream)
        d_off.copy_(h_off, non_blocking=True)
        d_ind.copy_(h_ind, non_blocking=True)
        res = counter.count(d_off, d_ind, outputs=("r", "lcc"), tuning=tuning)
        h_r.copy_(res.r, non_blocking=True)
        h_lcc.copy_(res.lcc, non_blocking=True)
        h_glob.copy_(res.global_counts, non_blocking=True)
        if k >= args.warmup:
            e2e_evs[k - args.warmup][1].record(stream)
    torch.cuda.synchronize()
    e2e_ms = gdist.max_over_ranks(sum(a.elapsed_time(b) for a, b in e2e_evs), dev)
    assert int(h_glob[0]) == T, "end-to-end result differs from the device-resident run"
    h2d = host.off.nbytes + host.ind.nbytes
    d2h = h_r.numel() * 8 + h_lcc.numel() * 8 + 3 * 8

    if rank != 0:
        return None
    m = host.m
    edges_all = m * world * args.steps
    value = edges_all / (total_ms / 1e3)
    ms_per_step = total_ms / args.steps
    work = algorithmic_bytes(host)
    traffic = dram_traffic(name)
    peak, peak_kind = measured_peaks()
    achieved = work["B_alg"] / (ms_per_step / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": DTYPE, "data": "synthetic",
        "config": graph_config(name, cfg, host, world),
        "result": {"triangles": T},
        "tuning": {"launch_shape": tuning, "search_s": tune_s,
                   "untuned_ms": tune_entry.get("default_ms"),
                   "tuned_ms": tune_entry.get("ms")},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": (traffic or {}).get("bytes"),
                     "traffic_unit": "bytes per count (ncu capture of this workload: "
                                     f"{(traffic or {}).get('source')})",
                     "scope": "one complete count (all launches of one gtc_count call)",
                     "work_model": f"B_alg = 4W + 4(n+1) + 4nnz + 16n = {work['B_alg']} bytes, "
                                   f"W = sum_undirected min(d_u, d_v) = {work['W']}",
                     "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)",
                     "note": "B_alg counts the full-list merge work of the reference's "
                             "algorithm; the degree-ordered kernels probe far fewer "
                             "elements and serve them mostly from L2 (traffic is the DRAM "
                             "measurement), so frac above 1.0 means fewer bytes than the "
                             "work model, not more than HBM delivers"},
        "phases_ms": phases,
        "e2e": {"value": m * world * args.steps / (e2e_ms / 1e3), "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_ms / args.steps},
        "clocks": clk.result,
        "gpu_launches": launches_per_count(host.n, host.nnz, tuning) * args.steps,
    }
    if with_baseline and not args.no_cpu_baseline:
        from oracle import oracle as O
        line["cpu_baseline"] = cpu_baseline(host, O.max_threads())
    return line


def launches_per_count(n: int, nnz: int, tuning: dict | None = None) -> int:
    """Kernels of one plain count with every output (the library's own plan:
    5 with vertex-id labels, 6 from 2^18 rows on, 11 with degree-rank
    labels)."""
    from gputrianglecounting_b200 import api
    return api.launch_plan(n, nnz, tuning=tuning)["launches"]


def int32_offsets(host_graph):
    """The same CSR with int32 offsets (the single-graph workloads specify an
    int32 CSR; every one of them has fewer than 2^31 entries)."""
    from gputrianglecounting_b200.graphs import CSRGraph
    assert host_graph.nnz < (1 << 31)
    return CSRGraph(np.ascontiguousarray(host_graph.off, dtype=np.int32), host_graph.ind,
                    host_graph.name)


def phase_breakdown(counter, g, flush, tuning: dict | None = None) -> dict:
    """Per-phase device time of one count with this tuning, from events the
    library records between its phases (forward build / group kernel / block
    kernel / epilogue), averaged over 3 runs."""
    import ctypes

    import torch
    from gputrianglecounting_b200 import _lib
    fn = _lib.load().gtc_count_phase_times
    n, nnz = g.off.numel() - 1, g.ind.numel()
    off_bits = 32 if g.off.dtype == torch.int32 else 64
    ws = counter._workspace(counter.workspace_bytes(n, nnz, off_bits))
    tun = _lib.Tuning(**{k: int(v) for k, v in tuning.items()}) if tuning else None
    res = []
    for k in range(3):
        flush.fill_(k)
        times = (ctypes.c_float * 4)()
        st = fn(g.off.data_ptr(), off_bits, g.ind.data_ptr(), n, nnz, ws.data_ptr(), ws.numel(),
                ctypes.cast(times, ctypes.c_void_p), ctypes.byref(tun) if tun else None)
        _lib.check(st, "gtc_count_phase_times")
        res.append(list(times))
    torch.cuda.synchronize()
    avg = [sum(r[i] for r in res) / len(res) for i in range(4)]
    return {"forward_build": avg[0], "group_kernel": avg[1], "block_kernel": avg[2],
            "epilogue": avg[3]}


# ------------------------------------------------------------------ batched

def batch_launches(total_n: int, total_nnz: int, tuning: dict | None = None) -> int:
    """Entry starts + globalize + the pipeline without its global-count
    kernel + per-graph T; with degree-rank labels the batch's graph-major
    ranks take a histogram, a 3-launch scan and a rank kernel in place of the
    single graph's 3 rank launches (+2)."""
    from gputrianglecounting_b200 import api
    extra = 2 if api.launch_plan(total_n, total_nnz, tuning=tuning)["labels"] == "degree-rank" \
        else 0
    return 2 + (launches_per_count(total_n, total_nnz, tuning) - 1) + 1 + extra


def run_batched(args, cfg, rank: int, world: int):
    """4,096 graphs: one persistent-pipeline run per step, replayed as a
    captured CUDA graph, against the same engine called once per graph."""
    import torch
    import torch.distributed as dist
    from gputrianglecounting_b200 import api, graphs as G
    from gputrianglecounting_b200 import dist as gdist
    from gputrianglecounting_b200._lib import load as load_lib
    load_lib()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    specs = G.batched_specs(cfg["graphs"], cfg["seed"])
    t0 = time.perf_counter()
    graphs = [G.make_spec_graph(s, dev) for s in specs]
    batch = G.concat_graphs(graphs, dev)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    m_total = batch.total_nnz // 2
    bc = api.BatchCounter(dev)
    out = bc.alloc_outputs(batch, ("r", "lcc", "graph_T"))
    # tuning for this batch's degree profile (staged search, cached), chosen
    # before any timed step
    from gputrianglecounting_b200 import autotune
    t0 = time.perf_counter()
    tuning = autotune.autotune_batch(bc, batch, out=out, cache_path=args.tune_cache)
    tune_s = time.perf_counter() - t0
    tune_entry = autotune.batch_entry(batch)
    stream = torch.cuda.Stream(dev)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            bc.count(batch, out=out, tuning=tuning, stream=stream)
    stream.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        bc.count(batch, out=out, tuning=tuning, stream=stream)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                evs[k][0].record(stream)
                graph.replay()
                evs[k][1].record(stream)
        torch.cuda.synchronize()
    step_ms = sorted(a.elapsed_time(b) for a, b in evs)
    total_ms = gdist.max_over_ranks(sum(step_ms), dev)
    graph_T = out.graph_T.clone()

    # one call per graph, same engine, same outputs (views of one buffer per
    # output, so that the whole result compares in one go)
    tc = api.TriangleCounter(dev)
    r_one = torch.empty_like(out.r)
    lcc_one = torch.empty_like(out.lcc)
    g_one = torch.empty(len(graphs), 3, dtype=torch.int64, device=dev)
    vs = batch.vstart.cpu().tolist()
    per = [api.TriangleCounts(r=r_one[vs[i]:vs[i + 1]], t=None, lcc=lcc_one[vs[i]:vs[i + 1]],
                              global_counts=g_one[i])
           for i in range(len(graphs))]
    for g, o in zip(graphs, per):                      # warm-up: workspace, caches
        tc.count(g.off, g.ind, out=o)
    torch.cuda.synchronize()
    base_ms = []
    for _ in range(2):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for g, o in zip(graphs, per):
            tc.count(g.off, g.ind, out=o)
        b.record()
        torch.cuda.synchronize()
        base_ms.append(a.elapsed_time(b))
    # every per-vertex r and lcc and every per-graph T of the batch equals the
    # graph counted alone
    assert torch.equal(g_one[:, 0], graph_T), "batched and per-graph T differ"
    assert torch.equal(r_one, out.r), "batched and per-graph r differ"
    assert torch.equal(lcc_one.view(torch.int64), out.lcc.view(torch.int64)), "lcc differ"
    del graph
    if rank != 0:
        return None
    value = m_total * world * args.steps / (total_ms / 1e3)
    base_value = m_total / (min(base_ms) / 1e3)
    p = lambda q: step_ms[min(len(step_ms) - 1, int(round(q * (len(step_ms) - 1))))]
    line = {
        "metric": "batched per-vertex TC edges/s", "value": value, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32 ids / int64 counts", "data": "synthetic",
        "config": {"workload": "batched", "graph": cfg["label"], "graphs": len(graphs),
                   "total_n": batch.total_n, "total_nnz": batch.total_nnz, "m": m_total,
                   "triangles": int(graph_T.sum().item()),
                   "l2": "inputs (13 GB adjacency) far larger than L2",
                   "generation_s": gen_s, "parallelism": f"{world} independent replica(s)"},
        "batched": {"form": "one gtc_count_batch per step, captured CUDA graph, persistent kernels",
                    "tuning": tuning, "tuning_search_s": tune_s,
                    "untuned_step_ms": tune_entry["default_ms"] if tune_entry else None,
                    "edges_per_s": value, "step_ms_p50": p(0.5), "step_ms_p99": p(0.99),
                    "per_graph_ms": min(base_ms), "per_graph_edges_per_s": base_value,
                    "speedup_vs_one_call_per_graph": value / world / base_value},
        "clocks": clk.result,
        "gpu_launches": batch_launches(batch.total_n, batch.total_nnz, tuning) * args.steps,
    }
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        sample = list(range(0, len(graphs), 64))
        t0 = time.perf_counter()
        m_s = 0
        for i in sample:
            h = graphs[i].numpy()
            O.ref_rows(h.off, h.ind, None, O.max_threads())
            m_s += h.m
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": m_s / dt, "unit": UNIT, "cores": O.max_threads(),
                                "kind": "reference",
                                "sample": f"{len(sample)} of {len(graphs)} graphs (every 64th), "
                                          f"{m_s} edges in {dt:.2f} s"}
    return line


# ------------------------------------------------------------------ serving

def run_ops(args, cfg, rank: int, world: int):
    """Device time per call of the library's other operators: the reference's
    kernelCall<int64_t> argument list on the whole R-MAT 20 graph (int64 ids
    narrowed on the device), its vertex-list overload on 65,536 seeded
    vertices, CSR validation, and gtc_batch_pack + gtc_count_batch of a pool
    of 256 device-resident graphs."""
    import torch
    from gputrianglecounting_b200 import api, graphs as G
    from gputrianglecounting_b200._lib import load as load_lib
    load_lib()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    host = int32_offsets(make_graph(CONFIGS["rmat20"], "cpu").numpy())
    off = torch.from_numpy(host.off).to(dev)
    ind = torch.from_numpy(host.ind).to(dev)
    off64, ind64 = off.to(torch.int64), ind.to(torch.int64)
    out64 = torch.empty(host.n, dtype=torch.int64, device=dev)
    rng = np.random.default_rng(cfg["seed"])
    verts = torch.from_numpy(rng.integers(0, host.n, cfg["vertices"]).astype(np.int64)).to(dev)
    vout = torch.empty(cfg["vertices"], dtype=torch.int64, device=dev)
    pool = [G.make_spec_graph(s, dev) for s in G.batched_specs(cfg["pool"], cfg["seed"])]
    bc = api.BatchCounter(dev)
    tun = {"group": 16, "labels": 2, "region": 4, "big_chunk": 4096, "item_len": 1024}
    ops = {
        "kernelCall_i64": lambda: api.kernelCall(1, 256, host.n, off64, ind64, out64, 1, 256, 0),
        "kernelCall_vertex_i64": lambda: api.kernelCall(1, 256, cfg["vertices"], off64, ind64, vout,
                                                       1, 256, 0, vertex=verts),
        "validate_csr": lambda: api.validate_csr(off, ind),
        "batch_pack_and_count": lambda: bc.count(bc.pack(pool), tuning=tun),
    }
    res = {}
    for name, fn in ops.items():
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(args.steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        res[name] = {"ms": statistics.mean(ms), "ms_min": min(ms)}
    if rank != 0:
        return None
    pool_m = sum(g.nnz for g in pool) // 2
    return {"metric": "operator device time per call", "value": res["kernelCall_i64"]["ms"],
            "unit": "ms", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": res["kernelCall_i64"]["ms"], "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPE, "data": "synthetic",
            "config": {"workload": "ops", "graph": cfg["label"], "n": host.n, "nnz": host.nnz,
                       "pool_graphs": len(pool), "pool_m": pool_m},
            "ops": res}


def run_serving(args, cfg, rank: int, world: int):
    """Continuous batching under Poisson load: p50/p99 latency and sustained
    edges/s per arrival rate (each rank serves its own stream)."""
    import torch
    from gputrianglecounting_b200 import graphs as G, serve
    from gputrianglecounting_b200._lib import load as load_lib
    load_lib()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    specs = G.batched_specs(cfg["pool"], cfg["seed"])
    pool = [G.make_spec_graph(s, dev) for s in specs]
    big = [G.rmat(22, 16, cfg["seed"] * 10 + k, device=dev) for k in range(2)]
    graphs = pool + big
    torch.cuda.synchronize()
    # launch shape tuned once on the pool's union (the typical admitted batch)
    from gputrianglecounting_b200 import api, autotune
    tuning = autotune.autotune_batch(api.BatchCounter(dev), G.concat_graphs(pool, dev),
                                     cache_path=args.tune_cache)
    server = serve.CountServer(graphs, dev, slots=3, budget_bytes=4 << 30, max_graphs=512,
                               tuning=tuning)
    # warm-up: every graph once, to size the slots' workspaces
    warm = [serve.Request(i, i, 0.0) for i in range(len(graphs))]
    server.run(warm)
    per_rate = {}
    rng = np.random.default_rng(cfg["seed"])
    with ClockSampler(local) as clk:
        for rate in cfg["rates"]:
            count = int(rate * cfg["arrivals_s"])
            arr = serve.poisson_arrivals(float(rate), count, seed=cfg["seed"] + rate)
            pick = rng.random(count) < 0.01
            gid = np.where(pick, len(pool) + rng.integers(0, len(big), count),
                           rng.integers(0, len(pool), count))
            reqs = [serve.Request(i, int(g), float(t)) for i, (g, t) in enumerate(zip(gid, arr))]
            server.batches = 0
            done = server.run(reqs, timeout_s=300)
            st = serve.latency_stats(done)
            st["batches"] = server.batches
            st["large_requests"] = int(pick.sum())
            per_rate[str(rate)] = st
    if rank != 0:
        return None
    top = per_rate[str(cfg["rates"][-1])]
    line = {
        "metric": "serving sustained edges/s (p50/p99 latency per rate)",
        "value": top["sustained_edges_per_s"] * world, "unit": UNIT, "n_gpus": world,
        "steps": len(cfg["rates"]), "warmup": 1, "ms_per_step": top["p50_ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32 ids / int64 counts", "data": "synthetic",
        "config": {"workload": "serving", "graph": cfg["label"], "slots": 3,
                   "slot_budget_gb": 4, "max_graphs_per_batch": 512, "tuning": tuning},
        "serving": per_rate, "clocks": clk.result,
    }
    return line


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--config", choices=sorted(CONFIGS), default="rmat20")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tune-cache", default=None,
                    help="JSON file caching the autotuner's launch shapes per degree profile "
                         "(read if present, written after a search)")
    ap.add_argument("--no-extras", action="store_true",
                    help="default workload only: skip the batched and serving sub-runs")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    cfg = CONFIGS[args.config]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference(args, cfg, rank)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        if args.config == "batched":
            line = run_batched(args, cfg, rank, world)
        elif args.config == "ops":
            line = run_ops(args, cfg, rank, world)
        elif args.config == "serving":
            line = run_serving(args, cfg, rank, world)
        else:
            line = run_b200(args, args.config, rank, world)
            if args.config == "rmat20" and not args.no_extras:
                # the other single-graph workloads, each with its own roofline
                # and CPU baseline, then the headline metric's other two parts:
                # batched speedup and served latency
                sub = argparse.Namespace(**vars(args))
                sub.steps, sub.warmup = 20, 3
                for other in ("rgg", "er"):
                    o = run_b200(sub, other, rank, world)
                    if line is not None:
                        line[other] = {"edges_per_s": o["value"], "ms": o["ms_per_step"],
                                       "steps": o["steps"], "config": o["config"],
                                       "result": o["result"], "tuning": o["tuning"],
                                       "roofline": o["roofline"],
                                       "phases_ms": o["phases_ms"], "e2e": o["e2e"],
                                       "clocks": o["clocks"]}
                        if "cpu_baseline" in o:
                            line[other]["cpu_baseline"] = o["cpu_baseline"]
                sub.steps = 30
                b = run_batched(sub, CONFIGS["batched"], rank, world)
                srv_cfg = dict(CONFIGS["serving"], arrivals_s=1.0)
                sv = run_serving(sub, srv_cfg, rank, world)
                if line is not None:
                    line["batched"] = dict(b["batched"], workload=b["config"]["graph"],
                                           graphs=b["config"]["graphs"], m=b["config"]["m"])
                    if "cpu_baseline" in b:
                        line["batched"]["cpu_baseline"] = b["cpu_baseline"]
                    line["serving"] = dict(sv["serving"], workload=sv["config"]["graph"])
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
