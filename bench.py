#!/usr/bin/env python3
"""Headline benchmark: exact triangle count of the 34.7M-edge power-law (R-MAT scale 22) graph on one B200.

Workload (seeded synthetic stand-in for the reference's com-LiveJournal measurement, same edge count): R-MAT
scale 22, (a,b,c,d) = (.57,.19,.19,.05), 8.52 * 2^22 samples symmetrised with self loops and duplicates removed
(about 34.7M undirected edges), ids permuted from the seed, oriented by (degree, id) into CSR like the reference's
graph.h. One step = one triangle count of the whole graph with the CSR and its derived index resident in HBM.

Reported (one JSON line, rank 0):
  value        algorithmic GB/s = B_alg / kernel time, B_alg = 4(n+1) + 8m + 4 * sum over oriented edges (u,v) of
               (d+(u) + d+(v)) (the bytes a two-list merge streams), whole job over all ranks;
  e2e          the same metric through the public C ABI from pinned host buffers: ga_graph_create (H2D copy and
               validation), ga_graph_prepare, ga_tc_count (8-byte D2H) and ga_graph_destroy, every step;
  roofline     B_alg per launch / CUDA-event launch time vs the measured HBM copy bandwidth;
  cpu_baseline the reference's own cpu_triangles_omp (oracle/_ref, compiled from its sources) on the host cores.
``--impl reference`` times the reference's CPU implementation alone with the same metric (its graph built by the
library's generator alone, libga_gen.so, and the reference's own build_graph_from_edges).

After the headline (outside its timed region) the default run adds the secondary workloads to the same line under
"workloads", each with parity against the reference's CPU code and its own CPU baseline: hk2 (Holme-Kim n 1.70M,
count + batch peeling at three eps), rmat22-full (per-edge supports and (k, triangle)-cores of the headline graph),
batch (4,096 graphs in one launch vs per-graph launches) and serve (Poisson arrivals into the request loop, p50/p99).
``--workload NAME`` runs one of them alone as its own line; ``--legs`` picks which the default run adds.
Multi-GPU (torchrun, one rank per GPU): replicas by default - every rank counts its own copy of the graph, no
collective on the data path; the max over ranks of the device time gives the whole-job value (weak scaling). With
--shard the ranks count ONE graph together, rank r its shard r of N (ga_tc_count_shard), summed by one 8-byte
all-reduce (strong scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "TC ms & GB/s (% HBM peak), 35M-edge power-law; batched vs plain graphs/s, p99"
SCALE, EDGE_FACTOR, SEED = 22, 8.52, 1
RMAT = (0.57, 0.19, 0.19)
L2_FLUSH_BYTES = 256 << 20
REF_ARM_BUDGET_S = 150.0   # wall time the reference arm's warm-up + timed steps may take


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_graph(ga, scale=SCALE, ef=EDGE_FACTOR, seed=SEED):
    t0 = time.time()
    pairs = ga.gen_rmat(scale, int(ef * (1 << scale)), *RMAT, seed=seed)
    g = ga.graph_from_pairs(1 << scale, pairs)
    log(f"graph: R-MAT scale {scale} ef {ef} seed {seed}: n={g.n} m={g.m} max_out_degree={g.max_out_degree} "
        f"({time.time() - t0:.1f} s on the host)")
    return g


def reference_graph(scale=SCALE, ef=EDGE_FACTOR, seed=SEED):
    """The same R-MAT graph as make_graph, built without the CUDA library: the samples come from libga_gen.so (the
    library's generator alone), the clean-up (self loops dropped, (min, max), unique) is numpy's, and the oriented CSR
    is the reference's own build_graph_from_edges (graph.h:38-67, oracle/_ref). Returns the reference's Graph fields."""
    import ctypes as C
    from oracle import Reference
    lib = C.CDLL(os.path.join(ROOT, "graph_analyzer_b200", "_lib", "libga_gen.so"))
    lib.ga_gen_rmat.argtypes = [C.c_uint32, C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_void_p]
    lib.ga_permute_ids.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint64]
    t0 = time.time()
    ns = int(ef * (1 << scale))
    pairs = np.zeros(2 * ns, np.uint32)
    if lib.ga_gen_rmat(scale, ns, *RMAT, seed, pairs.ctypes.data) or lib.ga_permute_ids(pairs.ctypes.data, ns,
                                                                                          1 << scale, seed):
        raise RuntimeError("libga_gen: generation failed")
    p = pairs.reshape(-1, 2).astype(np.uint64)
    lo, hi = np.minimum(p[:, 0], p[:, 1]), np.maximum(p[:, 0], p[:, 1])
    keys = np.unique((lo << np.uint64(32) | hi)[lo != hi])
    edges = np.stack([keys >> np.uint64(32), keys & np.uint64(0xFFFFFFFF)], 1).astype(np.uint32)
    g = Reference().build_graph_from_edges(1 << scale, edges)
    log(f"graph (reference build): R-MAT scale {scale} ef {ef} seed {seed}: n={g.n} m={g.m} "
        f"max_out_degree={g.max_out_degree} ({time.time() - t0:.1f} s on the host)")
    return g


def headline_config(scale, g, triangles, b_alg, parallelism):
    """The `config` of the headline line, identical in keys (and in everything but `parallelism`) in both arms."""
    return {"workload": f"rmat{scale}_tc", "n": g.n, "m": g.m, "edge_factor": EDGE_FACTOR, "seed": SEED,
            "rmat_abc": list(RMAT), "triangles": triangles, "b_alg_bytes": b_alg,
            "l2": f"256 MiB written between timed steps (untimed); col alone is {4 * g.m / 1e6:.0f} MB",
            "parallelism": parallelism}


def algorithmic_bytes(g) -> int:
    """B_alg = 4(n+1) + 8m + 4 * sum_{(u,v)} (d+(u) + d+(v))."""
    d = np.diff(g.rowptr.astype(np.int64))
    s_u = int((d * d).sum())                              # sum over edges of d+(src) = sum_u d+(u)^2
    s_v = int(d[g.col.astype(np.int64)].sum())            # sum over edges of d+(dst)
    return 4 * (g.n + 1) + 8 * g.m + 4 * (s_u + s_v)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self) -> dict:
        rows = []
        for line in (getattr(self, "out", "") or "").splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def read_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return {"hbm_gbs": float(p["hbm_gbs"]), "source": "measured"}
    except (OSError, KeyError, ValueError):
        return {"hbm_gbs": 6650.0, "source": "fallback"}


def read_traffic(workload: str):
    """DRAM bytes per launch of the count kernel from the committed ncu summary (None if absent)."""
    path = os.path.join(ROOT, "profiles", f"tc_hash_{workload}.md")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch:"):
                return int(float(line.split(":", 1)[1].strip()))
    except OSError:
        pass
    return None


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        return dist, world, rank, local
    return None, 1, 0, 0


def max_over_ranks(dist, x: float, device=None) -> float:
    """Max of a per-rank time over all ranks (NCCL: a device tensor; gloo: a host tensor); x itself on one rank."""
    if dist is None:
        return x
    import torch
    on = device if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=on)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def algorithmic_bytes_rows(g, u1: int) -> int:
    """B_alg of the rows [0, u1): the bytes a merge count of those rows streams (same formula as the whole graph)."""
    d = np.diff(g.rowptr.astype(np.int64))
    e1 = int(g.rowptr[u1])
    return 4 * (u1 + 1) + 8 * e1 + 4 * (int((d[:u1] * d[:u1]).sum()) + int(d[g.col[:e1].astype(np.int64)].sum()))


def cpu_reference_baseline(g, b_alg: int, steps: int = 1) -> dict:
    """The reference's cpu_triangles_omp (oracle/_ref) with all host threads, full graph, best of `steps`."""
    from oracle import Reference
    ref = Reference()
    best = None
    T = None
    with ref.resident(g) as rg:
        for _ in range(steps):
            t0 = time.perf_counter()
            T = rg.triangles_omp()
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
    return {"value": b_alg / best / 1e9, "unit": "GB/s", "cores": ref.num_threads(), "kind": "reference",
            "sample": f"whole graph, cpu_triangles_omp (graph.h:123) best of {steps}, {best * 1e3:.1f} ms, "
                      f"T={T}", "ms": best * 1e3, "triangles": T}


def run_reference_arm(args):
    """--impl reference: the reference's own CPU implementation, same metric and config, on rank 0 only."""
    dist, world, rank, _ = dist_setup(args)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0
    from oracle import Reference
    ref = Reference()
    g = reference_graph(args.scale)
    b_alg = algorithmic_bytes(g)
    rg = ref.resident(g)
    # one whole count (untimed) sizes the sample: every step counts the rows [0, u1), chosen so that the whole
    # warm-up + timed run stays within REF_ARM_BUDGET_S (the whole graph when it fits); vertex ids are permuted, so a
    # row prefix is a random vertex sample
    t0 = time.perf_counter()
    T_full = rg.triangles_omp()
    t_full = time.perf_counter() - t0
    frac = min(1.0, REF_ARM_BUDGET_S / max(1e-9, t_full * (args.warmup + args.steps)))
    if frac >= 1.0:
        u1, b_step = g.n, b_alg
    else:
        d = np.diff(g.rowptr.astype(np.int64))
        per_row = d * d + np.bincount(g.src.astype(np.int64), weights=d[g.col.astype(np.int64)], minlength=g.n)
        u1 = int(np.searchsorted(np.cumsum(per_row), frac * per_row.sum())) + 1
        u1 = min(max(u1, 1), g.n)
        b_step = algorithmic_bytes_rows(g, u1)
    step = (lambda: rg.triangles_omp()) if u1 == g.n else (lambda: rg.triangles_omp_rows(0, u1))
    for _ in range(args.warmup):
        step()
    times = []
    T = None
    for _ in range(args.steps):
        t0 = time.perf_counter()
        T = step()
        times.append(time.perf_counter() - t0)
    rg.close()
    ms = 1e3 * sum(times) / len(times)
    value = b_step / (ms / 1e3) / 1e9
    sample = ("whole graph per step" if u1 == g.n else
              f"rows [0, {u1}) of {g.n} per step ({100 * b_step / b_alg:.1f}% of the algorithmic bytes)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": headline_config(args.scale, g, T_full, b_alg,
                                  f"host threads x{ref.num_threads()} (OpenMP)"),
        "sample": {"step_triangles": T, "step_b_alg_bytes": b_step, "full_count_ms": t_full * 1e3,
                   "graph_build": "libga_gen samples + the reference's build_graph_from_edges"},
        "cpu_baseline": {"value": value, "unit": "GB/s", "cores": ref.num_threads(), "kind": "reference",
                         "sample": f"{sample}, cpu_triangles_omp (graph.h:123), {args.steps} steps"},
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def run_ours(args):
    dist, world, rank, local = dist_setup(args)
    import torch
    import graph_analyzer_b200 as ga
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    g = make_graph(ga, args.scale)
    b_alg = algorithmic_bytes(g)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)
    d_out = torch.zeros(1, dtype=torch.int64, device=dev)

    # ---- device-resident: one count per step on the prepared, resident graph ----
    dg = ga.DeviceGraph(g, device=local, stream=stream.cuda_stream)
    if args.tc_kernel != "auto":   # e.g. under a profiler, whose overheads can sway the autotuner's timing
        dg.set_option(ga.OPT_TC_KERNEL, {"plain": 1, "hash": 2}[args.tc_kernel])
    t0 = time.perf_counter()
    dg.prepare()
    torch.cuda.synchronize(dev)
    prep_ms = (time.perf_counter() - t0) * 1e3
    T = dg.tc_count()
    tuning = dg.tuning()
    shard = dist is not None and args.shard   # strong scaling: rank r counts shard r of world, one sum at the end
    count_async = ((lambda p: dg.tc_count_shard_async(rank, world, p)) if shard else dg.tc_count_async)
    for _ in range(args.warmup):
        count_async(d_out.data_ptr())
    torch.cuda.synchronize(dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clk:
        for s in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()                                   # L2 flush between steps (not timed)
            evs[s][0].record(stream)
            count_async(d_out.data_ptr())
            evs[s][1].record(stream)
        torch.cuda.synchronize(dev)
        time.sleep(0.25)
    if dist:
        dist.barrier()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    if shard:
        total = d_out.clone()
        dist.all_reduce(total)   # the one exchange of a sharded count: 8 bytes
        got = int(total.item())
    else:
        got = int(d_out.item())
    if got != T:
        raise RuntimeError(f"count changed between launches: {got} vs {T}")
    ms = max_over_ranks(dist, sum(step_ms) / len(step_ms), dev)
    value = (1 if shard else world) * b_alg / (ms / 1e3) / 1e9

    # ---- end to end through the public API from pinned host memory ----
    rp_h = torch.from_numpy(g.rowptr.view(np.int32)).pin_memory()
    col_h = torch.from_numpy(g.col.view(np.int32)).pin_memory()
    e2e_times = []
    for s in range(args.warmup + args.steps):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        h = ga.lib()
        import ctypes as C
        hd = C.c_void_p()
        ga._check(h.ga_graph_create(rp_h.data_ptr(), col_h.data_ptr(), g.n, g.m, local, stream.cuda_stream,
                                    C.byref(hd)))
        ga._check(h.ga_graph_prepare(hd))
        out = C.c_uint64(0)
        if shard:
            ga._check(h.ga_tc_count_shard(hd, rank, world, C.byref(out)))
            part = torch.tensor([out.value], dtype=torch.int64, device=dev)
            dist.all_reduce(part)
            out = C.c_uint64(int(part.item()))
        else:
            ga._check(h.ga_tc_count(hd, C.byref(out)))
        ga._check(h.ga_graph_destroy(hd))
        dt = time.perf_counter() - t0
        if out.value != T:
            raise RuntimeError("end-to-end count differs")
        if s >= args.warmup:
            e2e_times.append(dt)
    e2e_ms = max_over_ranks(dist, 1e3 * sum(e2e_times) / len(e2e_times), dev)
    e2e_value = (1 if shard else world) * b_alg / (e2e_ms / 1e3) / 1e9

    if rank != 0:
        dg.close()
        if dist:
            dist.destroy_process_group()
        return 0
    peaks = read_peaks()
    achieved = b_alg / (ms / 1e3) / 1e9
    cpu = cpu_reference_baseline(g, b_alg) if world == 1 and not args.no_cpu else None
    if cpu and cpu["triangles"] != T:
        raise RuntimeError(f"GPU count {T} differs from the reference CPU count {cpu['triangles']}")
    line = {
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "strong" if shard else "weak", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic",
        "config": headline_config(args.scale, g, T, b_alg,
                                  f"shards x{world} (one 8-byte all-reduce)" if shard else f"replicas x{world}"),
        "prep_ms": prep_ms, "oriented_edges_per_s": (1 if shard else world) * g.m / (ms / 1e3), "tuning": tuning,
        "e2e": {"value": e2e_value, "unit": "GB/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": int(rp_h.numel() * 4 + col_h.numel() * 4), "d2h_bytes_per_step": 8,
                "path": "ga_graph_create + ga_graph_prepare + ga_tc_count + ga_graph_destroy"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": read_traffic(f"rmat{args.scale}"),
                     "peak_source": peaks["source"], "kernel": "k_tc_hash<COUNT>"},
        "cpu_baseline": ({k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")} if cpu else None),
        "clocks": clk.summary(),
        "gpu_launches": args.steps,
    }
    dg.close()
    del flush, d_out
    if world == 1 and args.legs:
        # the secondary workloads, after the headline's timed region and with its graph released from the device
        line["workloads"] = run_legs(args, g)
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


# ---- secondary workloads -----------------------------------------------------------------------------------------
# Each leg returns one dict: its GPU times (plain launches vs the autotuned, graph-captured form), parity of the
# device results with the reference's own CPU code (oracle/_ref) or with the full-size records that code made
# (tests/golden/fullsize.json), and the reference's CPU times on this host. The default run adds every leg to the
# headline line under "workloads" (after the headline is measured; nothing here is inside its timed region);
# ``--workload NAME`` prints one leg as its own line.

FULLSIZE = os.path.join(ROOT, "tests", "golden", "fullsize.json")


def _timed(torch, fn, reps=1):
    """Device-synchronised wall time of fn() in ms (mean over reps) and its last result."""
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = None
    for _ in range(reps):
        r = fn()
    torch.cuda.synchronize()
    return (time.perf_counter() - t0) * 1e3 / reps, r


def _cpu_timed(fn):
    t0 = time.perf_counter()
    r = fn()
    return (time.perf_counter() - t0) * 1e3, r


def _peel_key(p):
    return (int(p.best_num), int(p.best_den), int(p.best_round), int(p.rounds))


def _sha(a) -> str:
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _fullsize(part: str):
    try:
        with open(FULLSIZE) as f:
            return json.load(f).get(part)
    except (OSError, ValueError):
        return None


def leg_hk2(args) -> dict:
    """Holme-Kim n = 1.70M, 6-7 edges per new vertex (mean 6.54), p = 0.3: TC and batch peeling at eps 1/20, 1/10,
    1/2. GPU: (a) plain one-kernel-per-launch count and host-driven peeling (one sync per round, re-enumeration
    updates) vs (b) the autotuned kernel with the peeling loop captured as a CUDA graph. Parity: every PeelResult field
    and the whole removed_round of both forms against the reference's cpu_batch_peel (densest.h:138-160), serial and
    OpenMP, and the count against cpu_triangles_serial. CPU: those reference calls timed on this host."""
    import torch
    import graph_analyzer_b200 as ga
    from oracle import Reference
    ref = Reference()
    t0 = time.time()
    g = ga.graph_from_pairs(1_700_000, ga.gen_holme_kim(1_700_000, 6, 7, 0.54, 0.3, seed=SEED))
    log(f"graph: Holme-Kim n={g.n} m={g.m} ({time.time() - t0:.1f} s on the host)")
    plain = ga.DeviceGraph(g)
    for opt, v in ((ga.OPT_TC_KERNEL, 1), (ga.OPT_LOOP_MODE, 1), (ga.OPT_UPDATE_MODE, 1)):
        plain.set_option(opt, v)
    tuned = ga.DeviceGraph(g)
    tuned.set_option(ga.OPT_LOOP_MODE, 2)
    plain.prepare()
    tuned.prepare()
    out = {"workload": "hk1.7M_tc_peel", "n": g.n, "m": g.m, "tc_ms": {}, "peel_ms": {}}
    T = {}
    for name, d in (("plain", plain), ("tuned", tuned)):
        for _ in range(args.warmup):
            d.tc_count()
        out["tc_ms"][name], T[name] = _timed(torch, d.tc_count, args.steps)
    out["tuning"] = tuned.tuning()
    out["first_peel_ms_tuned"], _ = _timed(torch, lambda: tuned.batch_peel(1, 10, want_removed=False))
    gpu = {}
    for num, den in ((1, 20), (1, 10), (1, 2)):
        key = f"{num}/{den}"
        for name, d in (("plain", plain), ("tuned", tuned)):
            gpu[(key, name)] = d.batch_peel(num, den)        # untimed: the full result, removed_round included
            # timed like the reference's gpu_densest time_ms: the loop, without downloading removed_round
            ms, r = _timed(torch, lambda: d.batch_peel(num, den, want_removed=False), max(1, args.steps // 2))
            out["peel_ms"].setdefault(key, {})[name] = ms
            assert _peel_key(r) == _peel_key(gpu[(key, name)])
    plain.close()
    tuned.close()
    # the reference's CPU code on the same graph: parity and baseline
    cpu = {"serial": {}, "omp": {}}
    cpu["serial"]["tc"], Ts = _cpu_timed(lambda: ref.triangles_serial(g))
    cpu["omp"]["tc"], To = _cpu_timed(lambda: ref.triangles_omp(g))
    parity = {"tc": T["plain"] == T["tuned"] == Ts == To}
    for num, den in ((1, 20), (1, 10), (1, 2)):
        key = f"{num}/{den}"
        cpu["serial"][key], rs = _cpu_timed(lambda: ref.batch_peel(g, num, den, use_omp=False))
        cpu["omp"][key], ro = _cpu_timed(lambda: ref.batch_peel(g, num, den, use_omp=True))
        ok = rs.ok and ro.ok and _peel_key(rs) == _peel_key(ro) and np.array_equal(rs.removed_round, ro.removed_round)
        for name in ("plain", "tuned"):
            r = gpu[(key, name)]
            ok &= _peel_key(r) == _peel_key(rs) and np.array_equal(r.removed_round, rs.removed_round)
        parity[f"peel_{key}"] = bool(ok)
        out["peel_ms"][key]["result"] = list(_peel_key(rs))
    tot = {k: out["tc_ms"][k] + sum(v[k] for v in out["peel_ms"].values()) for k in ("plain", "tuned")}
    cpu_tot = {k: sum(v.values()) for k, v in cpu.items()}
    threads = ref.num_threads()
    out.update({
        "metric": "TC + batch peel (3 eps) ms, plain vs autotuned graph-captured", "value": tot["tuned"], "unit": "ms",
        "higher_is_better": False, "plain_ms": tot["plain"], "speedup_vs_plain": tot["plain"] / tot["tuned"],
        "triangles": T["tuned"],
        "parity": {"against": "the reference's cpu_batch_peel (serial and OpenMP) and cpu_triangles_serial, every "
                              "PeelResult field and the whole removed_round", **parity,
                   "all": all(parity.values())},
        "cpu_baseline": {"value": cpu_tot["omp"], "unit": "ms", "cores": threads, "kind": "reference",
                         "sample": "whole graph: cpu_triangles_omp + cpu_batch_peel(OpenMP) at eps 1/20, 1/10, 1/2 "
                                   "(graph.h:123, densest.h:138)", "per_call_ms": cpu["omp"]},
        "cpu_serial": {"value": cpu_tot["serial"], "unit": "ms", "cores": 1, "kind": "reference",
                       "sample": "whole graph: cpu_triangles_serial + cpu_batch_peel(serial) at the same eps "
                                 "(graph.h:110, densest.h:138)", "per_call_ms": cpu["serial"]},
        "speedup_vs_cpu_omp": cpu_tot["omp"] / tot["tuned"], "speedup_vs_cpu_serial": cpu_tot["serial"] / tot["tuned"],
    })
    return out


def leg_rmat22(args, g=None) -> dict:
    """R-MAT scale 22 (34.7M edges): TC, per-edge uint32 supports and the full (k, triangle)-core decomposition.
    GPU: plain launches (one-thread-per-edge kernel, host-driven rounds) vs autotuned + graph-captured. Parity: every
    per-edge support against the oracle's for_each_triangle restatement (dsg.h:67-79, OpenMP) and the reference's
    record (fullsize.json); every core number, kmax and the round count against the oracle's restatement of
    core_decomp_loop_inc (dsg.h:724-751) and the reference's core_decomposition record (Alg 3, dsg.h:125-166).
    CPU: cpu_triangles_serial on a bounded row sample and cpu_triangles_omp on the whole graph (the reference's),
    the oracle's support and core passes."""
    import torch
    import graph_analyzer_b200 as ga
    from oracle import Oracle, Reference
    ref, orc = Reference(), Oracle()
    g = g if g is not None else make_graph(ga, args.scale)
    b_alg = algorithmic_bytes(g)
    plain = ga.DeviceGraph(g)
    for opt, v in ((ga.OPT_TC_KERNEL, 1), (ga.OPT_LOOP_MODE, 1)):
        plain.set_option(opt, v)
    tuned = ga.DeviceGraph(g)
    tuned.set_option(ga.OPT_LOOP_MODE, 2)
    plain.prepare()
    tuned.prepare()
    d_sup = torch.zeros(g.m, dtype=torch.int32, device="cuda")
    out = {"workload": f"rmat{args.scale}_tc_esup_cores", "n": g.n, "m": g.m}
    sup = {}
    for name, d in (("plain", plain), ("tuned", tuned)):
        d.tc_count()
        out[f"tc_ms_{name}"], T = _timed(torch, d.tc_count, args.steps)
        d.support_edges_device(d_sup.data_ptr())
        out[f"esup_ms_{name}"], _ = _timed(torch, lambda: d.support_edges_device(d_sup.data_ptr()), 2)
        sup[name] = d_sup.cpu().numpy().view(np.uint32).copy()
    out["tuning"] = tuned.tuning()
    out["first_cores_ms_tuned"], _ = _timed(torch, lambda: tuned.core_decomposition(want_core=False))  # lists
    res = {}
    out["cores_ms_tuned_runs"] = []
    for _ in range(3):
        ms, res["tuned"] = _timed(torch, lambda: tuned.core_decomposition(), 1)
        out["cores_ms_tuned_runs"].append(ms)
    out["cores_ms_tuned"] = min(out["cores_ms_tuned_runs"])
    out["cores_ms_plain"], res["plain"] = _timed(torch, lambda: plain.core_decomposition(), 1)
    plain.close()
    tuned.close()
    del d_sup
    # parity: the oracle now, the reference's own records (made offline by tests/golden/make_fullsize.py)
    cpu = {}
    cpu["esup_oracle_omp_ms"], (To, sup_o) = _cpu_timed(lambda: orc.edge_support(g, use_omp=True))
    cpu["cores_oracle_ms"], (core_o, kmax_o, rounds_o) = _cpu_timed(lambda: orc.core_levels_inc(g))
    parity = {
        "tc": T == To,
        "esup_vs_oracle": all(np.array_equal(sup[k], sup_o) for k in sup),
        "cores_vs_oracle": all((r.kmax, r.rounds) == (kmax_o, rounds_o) and np.array_equal(r.core, core_o)
                               for r in res.values()),
    }
    rec = _fullsize("rmat")
    if rec and (rec["n"], rec["m"]) == (g.n, g.m) and args.scale == rec["config"]["scale"]:
        parity["tc_vs_reference_record"] = T == rec["triangles"]
        parity["esup_vs_reference_record"] = _sha(sup["tuned"]) == rec["edge_support_sha256"]
        parity["cores_vs_reference_record"] = (_sha(res["tuned"].core) == rec["core_sha256"]
                                               and res["tuned"].kmax == rec["kmax"])
    # the reference's counters on this host: OpenMP on the whole graph, serial on a bounded row sample
    with ref.resident(g) as rg:
        cpu["tc_omp_ms"], T_omp = _cpu_timed(rg.triangles_omp)
        parity["tc_vs_reference_omp"] = T_omp == T
        d = np.diff(g.rowptr.astype(np.int64))
        per_row = d * d + np.bincount(g.src.astype(np.int64), weights=d[g.col.astype(np.int64)], minlength=g.n)
        # rows whose serial count takes about 10 s: the OpenMP time x threads x 10 s / (that product) of the work
        frac = min(1.0, 10.0 / max(1e-3, cpu["tc_omp_ms"] / 1e3 * ref.num_threads()))
        u1 = min(g.n, int(np.searchsorted(np.cumsum(per_row), frac * per_row.sum())) + 1)
        cpu["tc_serial_sample_ms"], _ = _cpu_timed(lambda: rg.triangles_serial_rows(0, u1))
    b_rows = algorithmic_bytes_rows(g, u1)
    parity["all"] = all(parity.values())
    out.update({
        "metric": "TC, per-edge supports, (k,triangle)-cores ms",
        "value": out["tc_ms_tuned"] + out["esup_ms_tuned"] + out["cores_ms_tuned"], "unit": "ms",
        "higher_is_better": False, "triangles": T, "kmax": res["tuned"].kmax, "rounds": res["tuned"].rounds,
        "parity": {"against": "oracle (for_each_triangle supports, core_decomp_loop_inc restated) now, and the "
                              "reference's for_each_triangle / core_decomposition records", **parity},
        "cpu_baseline": {"value": b_alg / (cpu["tc_omp_ms"] / 1e3) / 1e9, "unit": "GB/s",
                         "cores": ref.num_threads(), "kind": "reference",
                         "sample": f"whole graph, cpu_triangles_omp (graph.h:123): {cpu['tc_omp_ms']:.0f} ms"},
        "cpu_serial": {"value": b_rows / (cpu["tc_serial_sample_ms"] / 1e3) / 1e9, "unit": "GB/s", "cores": 1,
                       "kind": "reference",
                       "sample": f"cpu_triangles_serial's loop (graph.h:110) on rows [0, {u1}) "
                                 f"({100 * b_rows / b_alg:.1f}% of the algorithmic bytes): "
                                 f"{cpu['tc_serial_sample_ms']:.0f} ms"},
        "cpu_oracle": {"esup_omp_ms": cpu["esup_oracle_omp_ms"], "cores_ms": cpu["cores_oracle_ms"],
                       "cores": ref.num_threads(), "kind": "port",
                       "sample": "whole graph: or_edge_support_omp, or_core_levels_inc (incidence lists, OpenMP "
                                 "listing and updates)"},
    })
    return out


def leg_batch(args) -> dict:
    """4,096 Holme-Kim graphs (n log-uniform in [64, 262144], mean degree U[4, 32], p U[0.1, 0.7]) packed as one
    concatenated CSR: TC + eps = 1/10 batch peeling of every graph by one count launch and one graph-captured peeling
    loop, against 4,096 per-graph runs of (a) the same kernels (autotuned count, graph-captured loop per graph) and
    (b) plain launches (one-thread-per-edge count, host-driven rounds). Parity: every graph's count, PeelResult and
    removed_round against the reference's records (fullsize.json, fullsize_batch.npz) and, on a sample of graphs, the
    reference's cpu_triangles_serial + cpu_batch_peel run now on all host threads (the CPU baseline)."""
    import concurrent.futures as cf
    import torch
    import graph_analyzer_b200 as ga
    from oracle import Reference
    ref = Reference()
    G = args.graphs
    t0 = time.time()
    b = ga.gen_holme_kim_batch(G, 64, 262144, 4.0, 32.0, 0.1, 0.7, seed=SEED)
    N, M = int(b.vtx_off[-1]), int(b.edge_off[-1])
    log(f"batch: {G} graphs, N={N} M={M} ({time.time() - t0:.1f} s on the host)")
    out = {"workload": f"batch{G}_hk_tc_peel", "graphs": G, "N": N, "M": M}
    t0 = time.perf_counter()
    db = ga.DeviceBatch(b)
    out["create_ms"] = (time.perf_counter() - t0) * 1e3
    t_leg = time.time()
    # timed without downloading removed_round (N entries), as the per-graph runs below
    out["first_batch_ms"], r0 = _timed(torch, lambda: db.tc_peel(1, 10, want_removed=False))   # autotune, lists, capture
    out["batch_ms"], r = _timed(torch, lambda: db.tc_peel(1, 10, want_removed=False), max(1, args.steps // 2))
    full = db.tc_peel(1, 10)                                                  # untimed: with removed_round
    out["device_bytes"] = db.device_bytes()
    out["tuning"] = db.tuning()
    db.close()
    ok_batch = np.array_equal(r.triangles, r0.triangles) and np.array_equal(full.best_num, r.best_num)
    parity = {"status_ok": bool(np.all(full.status == 0)), "repeat_identical": bool(ok_batch)}
    rec = _fullsize("batch")
    if rec and G == rec["config"]["graphs"] and (N, M) == (rec["N"], rec["M"]):
        with np.load(os.path.join(ROOT, "tests", "golden", rec["per_graph"])) as z:
            want = {k: z[k] for k in z.files}
        parity["vs_reference_record"] = bool(
            np.array_equal(full.triangles, want["triangles"]) and np.array_equal(full.best_num, want["best_num"])
            and np.array_equal(full.best_den, want["best_den"]) and np.array_equal(full.best_round, want["best_round"])
            and np.array_equal(full.rounds, want["rounds"]) and _sha(full.removed_round) == rec["removed_round_sha256"])
    log(f"batch: one-launch runs and records checked in {time.time() - t_leg:.1f} s")
    rp = torch.from_numpy(b.rowptr.view(np.int32)).cuda()
    cl = torch.from_numpy(b.col.view(np.int32)).cuda()

    # the per-graph arms run on every stride-th graph (all of them with --per-graph-stride 1); graph sizes come out
    # of the generator in random order, so the sample's time scaled by G / len(sample) estimates the whole batch's
    sample_idx = list(range(0, G, max(1, args.per_graph_stride)))
    scale = G / len(sample_idx)

    def per_graph_arm(options):
        t_arm = time.time()
        handles = []
        for i in sample_idx:
            v0, e0 = int(b.vtx_off[i]), int(b.edge_off[i])
            n, m = int(b.vtx_off[i + 1]) - v0, int(b.edge_off[i + 1]) - e0
            d = ga.DeviceGraph.from_device(rp.data_ptr() + 4 * (v0 + i), cl.data_ptr() + 4 * e0, n, m)
            for opt, v in options:
                d.set_option(opt, v)
            d.prepare()
            handles.append(d)
        mismatches = 0

        def run_all():
            nonlocal mismatches
            mismatches = 0
            for i, d in zip(sample_idx, handles):
                t = d.tc_count()
                p = d.batch_peel(1, 10, want_removed=False)
                if t != full.triangles[i] or _peel_key(p) != (full.best_num[i], full.best_den[i], full.best_round[i],
                                                              full.rounds[i]):
                    mismatches += 1
        log(f"batch per-graph arm {options}: {len(handles)} handles prepared in {time.time() - t_arm:.1f} s")
        t0 = time.time()
        run_all()                                  # warm-up: loop state, lists and graph capture per graph
        log(f"  warm-up {time.time() - t0:.1f} s")
        ms, _ = _timed(torch, run_all, 1)
        t0 = time.time()
        for d in handles:
            d.close()
        log(f"  timed {ms / 1e3:.2f} s, closed in {time.time() - t0:.1f} s")
        return ms * scale, mismatches

    out["per_graph_same_kernels_ms"], mm1 = per_graph_arm([(ga.OPT_LOOP_MODE, 2)])
    out["per_graph_plain_ms"], mm2 = per_graph_arm([(ga.OPT_TC_KERNEL, 1), (ga.OPT_LOOP_MODE, 1),
                                                   (ga.OPT_UPDATE_MODE, 1)])
    del rp, cl
    parity["per_graph_same_kernels_identical"] = mm1 == 0
    parity["per_graph_plain_identical"] = mm2 == 0
    # the reference's CPU code on a sample of graphs (every 16th), all host threads, one graph per thread
    sample = list(range(0, G, 16))
    threads = os.cpu_count() or 1

    def one(i):
        gi = b.graph(i)
        t = ref.triangles_serial(gi)
        p = ref.batch_peel(gi, 1, 10)
        v0, v1 = int(b.vtx_off[i]), int(b.vtx_off[i + 1])
        return (t == full.triangles[i] and _peel_key(p) == (full.best_num[i], full.best_den[i], full.best_round[i],
                                                             full.rounds[i])
                and np.array_equal(p.removed_round, full.removed_round[v0:v1]))
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(threads) as ex:
        oks = list(ex.map(one, sample))
    cpu_s = time.perf_counter() - t0
    log(f"batch: reference on {len(sample)} graphs in {cpu_s:.1f} s")
    parity["sample_vs_reference_now"] = all(oks)
    parity["all"] = all(parity.values())
    edges_sample = int(sum(int(b.edge_off[i + 1] - b.edge_off[i]) for i in sample))
    out.update({
        "metric": "batched vs plain graphs/s (TC + eps=1/10 batch peel)", "value": G / (out["batch_ms"] / 1e3),
        "unit": "graphs/s", "higher_is_better": True,
        "per_graph_same_kernels_graphs_per_s": G / (out["per_graph_same_kernels_ms"] / 1e3),
        "per_graph_plain_graphs_per_s": G / (out["per_graph_plain_ms"] / 1e3),
        "speedup_vs_per_graph_same_kernels": out["per_graph_same_kernels_ms"] / out["batch_ms"],
        "speedup_vs_per_graph_plain": out["per_graph_plain_ms"] / out["batch_ms"],
        "per_graph_sample": (f"all {G} graphs" if len(sample_idx) == G else
                             f"every {args.per_graph_stride}th graph ({len(sample_idx)}), time scaled by "
                             f"{scale:.2f}"),
        "triangles": int(full.triangles.sum()),
        "parity": {"against": "the reference's per-graph records (all graphs) and its CPU code now (sample)",
                   **parity},
        "cpu_baseline": {"value": len(sample) / cpu_s, "unit": "graphs/s", "cores": threads, "kind": "reference",
                         "sample": f"every 16th graph ({len(sample)} graphs, {100 * edges_sample / M:.1f}% of the "
                                   f"edges), cpu_triangles_serial + cpu_batch_peel per graph, one graph per thread"},
    })
    return out


def _serve_trace(ga, R, rng):
    """Request trace: 60% TC, 30% batch peel (eps = 1/10), 10% (k, triangle)-cores; 30% of requests re-query one of the
    32 most recently used graphs, the others go to a new graph - 95% Holme-Kim from the batch generator above, 5% R-MAT
    at scales 20-23 (a new registration of one pre-built graph per scale, so it is uploaded like a new graph)."""
    t0 = time.time()
    hk = ga.gen_holme_kim_batch(R, 64, 262144, 4.0, 32.0, 0.1, 0.7, seed=SEED + 7)
    rmat = {sc: make_graph(ga, sc, EDGE_FACTOR, SEED + sc) for sc in (20, 21, 22, 23)}
    graphs, used, trace, hk_next = [], [], [], 0
    for _ in range(R):
        if used and rng.random() < 0.3:
            gi = used[-1 - int(rng.integers(0, min(len(used), 32)))]
        else:
            if rng.random() < 0.05:
                graphs.append(rmat[int(rng.integers(20, 24))])
            else:
                graphs.append(hk.graph(hk_next))
                hk_next += 1
            gi = len(graphs) - 1
            used.append(gi)
        u = rng.random()
        trace.append((gi, 0 if u < 0.6 else 1 if u < 0.9 else 2))
    log(f"serve trace: {R} requests on {len(graphs)} graphs ({time.time() - t0:.1f} s on the host)")
    return graphs, trace


def _serve_value(ga, kind, r):
    if kind == ga.REQ_TC:
        return (r.triangles,)
    if kind == ga.REQ_PEEL:
        return (r.peel.best_num, r.peel.best_den, r.peel.best_round, r.peel.rounds)
    return r.core


def _serve_run(ga, graphs, trace, arrivals_s, slots=0):
    """Submits the trace at the given arrival times (open loop) to a fresh server; returns per-request latency (ms,
    submit to completion), results, wall time of the run and the server statistics."""
    with ga.Server(slots=slots) as s:
        ids = [s.add_graph(g) for g in graphs]
        tickets = []
        t0 = time.perf_counter()
        for (gi, kind), at in zip(trace, arrivals_s):
            dt = t0 + at - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            tickets.append(s.submit(ids[gi], kind, 1, 10))
        res = [s.wait(t) for t in tickets]
        wall = time.perf_counter() - t0
        st = s.stats()
    lat = np.array([r.queue_ms + r.run_ms for r in res])
    return lat, res, wall, st


def _fifo_latency(service_s, arrivals_s):
    """Latency (ms) of a single serial server (FIFO) given measured service times and arrival times."""
    free, lat = 0.0, []
    for sv, at in zip(service_s, arrivals_s):
        start = max(free, at)
        free = start + sv
        lat.append((free - at) * 1e3)
    return np.array(lat)


def leg_serve(args) -> dict:
    """Serving: open-loop Poisson arrivals (rate swept) into the request loop (admission under a 150 GB HBM budget,
    resident graphs for re-queries, small requests folded into batch launches, 4 + 2 concurrent streams), against
    serial plain launches of the same library (one request at a time: uploaded, counted with the kernel the autotuner
    picks, its peeling or core rounds driven from the host, freed), so the comparison isolates what the serving loop
    adds: concurrency, residency, folding and page-locked uploads.
    Results of every request must be identical in both."""
    import torch
    import graph_analyzer_b200 as ga
    R = args.requests
    rng = np.random.default_rng(SEED)
    graphs, trace = _serve_trace(ga, R, rng)
    # every run below uses a fresh server (no graph resident yet); one idle server held open for the whole workload
    # keeps the device's memory pool mapped between them, as in a long-lived serving process
    holder = ga.Server()
    # warm-up, untimed: one pass of the whole trace through a server fills the kernel-choice cache (one timing per
    # degree-distribution signature) and the memory pool, so neither side below pays those first-time costs
    _serve_run(ga, graphs, trace, np.zeros(R), args.slots)
    # serial plain launches: measured service time of every request in trace order
    service, plain_vals = [], []
    for gi, kind in trace:
        t0 = time.perf_counter()
        with ga.DeviceGraph(graphs[gi]) as d:
            d.set_option(ga.OPT_LOOP_MODE, 1)
            if kind == ga.REQ_TC:
                val = (d.tc_count(),)
            elif kind == ga.REQ_PEEL:
                val = _peel_key(d.batch_peel(1, 10, want_removed=False))
            else:
                c = d.core_decomposition(want_core=False)
                val = (c.kmax, c.rounds)
        torch.cuda.synchronize()
        service.append(time.perf_counter() - t0)
        plain_vals.append(val)
    serial_s = float(sum(service))
    # closed-loop bursts (all requests at t = 0): the server's capacity, median of three runs (run-to-run spread on a
    # shared host is large; every run is reported)
    bursts = [_serve_run(ga, graphs, trace, np.zeros(R), args.slots) for _ in range(3)]
    walls = [b[2] for b in bursts]
    lat, res, wall, st = bursts[int(np.argsort(walls)[1])]
    capacity = R / wall
    # where the time goes, per request class (graph family x kind): serial service vs the server's run time
    names = ("tc", "peel", "core")
    by_class = {}
    for (gi, kind), sv, r in zip(trace, service, res):
        c = ("rmat_" if graphs[gi].n > (1 << 19) else "hk_") + names[kind]
        e = by_class.setdefault(c, {"count": 0, "serial_ms": 0.0, "server_run_ms": 0.0})
        e["count"] += 1
        e["serial_ms"] += sv * 1e3
        e["server_run_ms"] += r.run_ms
    log("per class: " + json.dumps(by_class))
    identical = all(_serve_value(ga, k, r) == v and r.status == 0 for (_, k), r, v in zip(trace, res, plain_vals))
    for b in bursts:
        identical &= all(_serve_value(ga, k, r) == v and r.status == 0
                         for (_, k), r, v in zip(trace, b[1], plain_vals))
    burst = {"req_s": capacity, "runs_req_s": [R / w for w in walls], "p50_ms": float(np.percentile(lat, 50)),
             "p99_ms": float(np.percentile(lat, 99)), "folded_launches": st["folded_launches"],
             "evictions": st["evictions"], "peak_reserved_gb": st["peak_reserved_bytes"] / 1e9}
    sweep = []
    for frac in args.rate_fracs:
        rate = frac * capacity
        arr = np.cumsum(rng.exponential(1.0 / rate, R))
        arr -= arr[0]
        lat, res, wall, st = _serve_run(ga, graphs, trace, arr, args.slots)
        identical &= all(_serve_value(ga, k, r) == v and r.status == 0
                         for (_, k), r, v in zip(trace, res, plain_vals))
        slat = _fifo_latency(service, arr)
        sweep.append({"offered_req_s": rate, "achieved_req_s": R / wall,
                      "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                      "serial_plain_p50_ms": float(np.percentile(slat, 50)),
                      "serial_plain_p99_ms": float(np.percentile(slat, 99)),
                      "folded_launches": st["folded_launches"], "evictions": st["evictions"],
                      "peak_reserved_gb": st["peak_reserved_bytes"] / 1e9})
        log(f"serve: offered {rate:.1f} req/s -> p50 {sweep[-1]['p50_ms']:.2f} ms p99 {sweep[-1]['p99_ms']:.2f} ms "
            f"(serial plain p99 {sweep[-1]['serial_plain_p99_ms']:.1f} ms)")
    kinds = np.bincount([k for _, k in trace], minlength=3)
    line = {"workload": "serve_poisson", "metric": "serving requests/s and p50/p99 latency vs serial plain launches",
            "value": capacity, "unit": "req/s", "higher_is_better": True, "serial_plain_req_s": R / serial_s,
            "speedup_vs_serial_plain": capacity / (R / serial_s), "requests": R, "graphs": len(graphs),
            "mix": {"tc": int(kinds[0]), "peel_eps_1_10": int(kinds[1]), "cores": int(kinds[2])},
            "hbm_budget_gb": 150, "slots": args.slots or 4, "burst": burst, "sweep": sweep, "by_class": by_class,
            "bit_identical": bool(identical)}
    holder.close()
    return line

def leg_passes(args) -> dict:
    """Each triangle pass of the hash kernel on R-MAT scale 22 timed alone (device-synchronised wall time, mean of
    --steps calls after the warm-up): the count, per-edge supports (into device memory), per-vertex supports (with the
    download of the n counters), and a batch peel at eps 1/2, whose first call builds the incidence lists with the
    LIST pass (timed apart from the later, list-reusing calls). Checked against the count: both supports sum to 3T.
    Also the short command the per-pass ncu captures run."""
    import torch
    import graph_analyzer_b200 as ga
    g = make_graph(ga, args.scale)
    d = ga.DeviceGraph(g)
    d.set_option(ga.OPT_TC_KERNEL, 2)
    d.prepare()
    d_sup = torch.zeros(g.m, dtype=torch.int32, device="cuda")
    T = d.tc_count()
    out = {"workload": f"rmat{args.scale}_passes", "n": g.n, "m": g.m, "triangles": T}
    for _ in range(args.warmup):
        d.tc_count()
        d.support_edges_device(d_sup.data_ptr())
    out["count_ms"], _ = _timed(torch, d.tc_count, args.steps)
    out["esup_ms"], Ts = _timed(torch, lambda: d.support_edges_device(d_sup.data_ptr()), args.steps)
    out["vsup_ms"], (Tv, deg) = _timed(torch, d.support_vertices, args.steps)
    out["first_peel_ms"], _ = _timed(torch, lambda: d.batch_peel(1, 2, want_removed=False))   # LIST pass + rounds
    out["peel_ms"], _ = _timed(torch, lambda: d.batch_peel(1, 2, want_removed=False), args.steps)
    sup_total = int(d_sup.cpu().numpy().view(np.uint32).astype(np.int64).sum())
    d.close()
    ok = Ts == T and Tv == T and sup_total == 3 * T and int(deg.astype(np.int64).sum()) == 3 * T
    out.update({"metric": "triangle passes of the hash kernel, ms", "value": out["count_ms"], "unit": "ms",
                "higher_is_better": False, "parity": {"against": "the count (supports sum to 3T)", "all": ok}})
    return out


LEGS = {"hk2": leg_hk2, "rmat22-full": leg_rmat22, "batch": leg_batch, "serve": leg_serve}


def run_legs(args, g_rmat=None) -> dict:
    """Every secondary leg in turn (in the default run, after the headline), each under a wall-time budget and with
    its failure recorded instead of raised, so that a leg can never cost the headline line."""
    out, t_start = {}, time.time()
    for name in args.legs:
        if time.time() - t_start > args.legs_budget_s:
            out[name] = {"skipped": f"wall-time budget of {args.legs_budget_s:.0f} s for the secondary legs spent"}
            continue
        t0 = time.time()
        try:
            out[name] = LEGS[name](args, g_rmat) if name == "rmat22-full" else LEGS[name](args)
        except Exception as e:   # recorded in the line, never raised
            out[name] = {"error": f"{type(e).__name__}: {e}"}
        out[name]["leg_wall_s"] = time.time() - t0
        log(f"leg {name}: {out[name]['leg_wall_s']:.1f} s")
    return out


def run_leg(args) -> int:
    """--workload NAME: one secondary leg as its own JSON line (exit 1 when its parity fails)."""
    line = LEGS[args.workload](args)
    print(json.dumps(line), flush=True)
    par = line.get("parity", {})
    ok = par.get("all", True) if isinstance(par, dict) else True
    return 0 if ok and line.get("bit_identical", True) else 1


def _write_edge_text(g, path):
    """The graph as a SNAP-style text edge list ("u<TAB>v" per oriented edge)."""
    with open(path, "w") as f:
        f.write(f"# n={g.n} m={g.m}\n")
        step = 1 << 22
        for i in range(0, g.m, step):
            f.write("\n".join(f"{a}\t{b}" for a, b in zip(g.src[i:i + step].tolist(), g.col[i:i + step].tolist())))
            f.write("\n")


def _csv_rows(text):
    return [ln.split(",") for ln in text.splitlines() if ln and not ln.startswith(("#", "impl"))]


def run_reference_gpu(args):
    """The reference's own GPU drivers (baseline/_ref/bin, built from its sources for sm_100a by
    baseline/build_reference_gpu.py) against this library's drivers, on the same text files and the same GPU:
    gpu_tc vs ga_tc on R-MAT 22 (kernels v1-v9), gpu_densest vs ga_densest (eps 1/10, with the greedy peel rows) on
    the Holme-Kim n 1.70M graph, gpu_dsg vs ga_dsg (core decomposition) on the Holme-Kim n 8,298 graph, and gpu_dsg
    vs ga_dsg's whole densest-subgraph pipeline on the Holme-Kim n 8,298 and n 1.70M graphs. Every program verifies its own results (the
    reference's against its CPU code); the triangle counts, peel results, core rows and pipeline subgraphs must
    agree."""
    import tempfile
    import graph_analyzer_b200 as ga
    ref_bin = os.path.join(ROOT, "baseline", "_ref", "bin")
    our_bin = os.path.join(ROOT, "graph_analyzer_b200", "_bin")
    if not os.path.exists(os.path.join(ref_bin, "gpu_tc")):
        print(json.dumps({"workload": "reference_gpu", "unavailable": "baseline/_ref/bin not built "
                          "(python baseline/build_reference_gpu.py)"}), flush=True)
        return 0
    tmp = tempfile.mkdtemp(prefix="ga_refgpu_")
    out = {"workload": "reference_gpu", "metric": "reference GPU drivers vs this library's drivers, same files, same GPU"}
    runs = [
        ("tc_rmat22", lambda: make_graph(ga), ["gpu_tc", "ga_tc"], lambda p: [p, str(max(3, args.steps // 2))]),
        ("peel_hk1.7M", lambda: ga.graph_from_pairs(1_700_000, ga.gen_holme_kim(1_700_000, 6, 7, 0.54, 0.3, seed=SEED)),
         ["gpu_densest", "ga_densest"], lambda p: [p, "1", "10", "--repeats", "3"]),
        ("cores_hk8298", lambda: ga.graph_from_pairs(8298, ga.gen_holme_kim(8298, 12, 12, 0.0, 0.5, seed=SEED)),
         ["gpu_dsg", "ga_dsg"], lambda p: [p, "--repeats", "3", "--no-exact", "--no-greedy", "--no-greedypp"]),
        # the whole densest-subgraph pipeline: cores, greedy lower bound, prune, Greedy++ (10 passes), seeded CoreExact
        ("dsg_hk8298", lambda: ga.graph_from_pairs(8298, ga.gen_holme_kim(8298, 12, 12, 0.0, 0.5, seed=SEED)),
         ["gpu_dsg", "ga_dsg"], lambda p: [p, "--repeats", "3"]),
        ("dsg_hk1.7M", lambda: ga.graph_from_pairs(1_700_000, ga.gen_holme_kim(1_700_000, 6, 7, 0.54, 0.3, seed=SEED)),
         ["gpu_dsg", "ga_dsg"], lambda p: [p, "--repeats", "3"]),
    ]
    ok = True
    for name, make, (ref_prog, our_prog), argv in runs:
        g = make()
        path = os.path.join(tmp, name + ".txt")
        t0 = time.time()
        _write_edge_text(g, path)
        log(f"{name}: n={g.n} m={g.m} written ({time.time() - t0:.1f} s)")
        res = {}
        for who, exe in (("reference", os.path.join(ref_bin, ref_prog)), ("ours", os.path.join(our_bin, our_prog))):
            t0 = time.time()
            r = subprocess.run([exe, *argv(path)], capture_output=True, text=True, timeout=1800)
            log(f"{name} {who}: rc {r.returncode} in {time.time() - t0:.1f} s")
            if r.returncode != 0:
                log(r.stderr[-2000:])
                ok = False
            res[who] = _csv_rows(r.stdout)
        out[name] = res
        os.remove(path)
    os.rmdir(tmp)
    # headline comparison: best kernel time of each side on the TC file
    tc = out.get("tc_rmat22", {})
    if tc.get("reference") and tc.get("ours"):
        ref_best = min(tc["reference"], key=lambda r: float(r[5]))
        our_best = min(tc["ours"], key=lambda r: float(r[5]))
        out["tc_best"] = {"reference": {"impl": ref_best[0], "kernel_ms": float(ref_best[5])},
                          "ours": {"impl": our_best[0], "kernel_ms": float(our_best[5])},
                          "speedup": float(ref_best[5]) / float(our_best[5]),
                          "same_triangles": len({r[4] for r in tc["reference"] + tc["ours"]}) == 1}
        ok &= out["tc_best"]["same_triangles"]
    # the greedy peel beside the batch peel (the quality baseline of gpu_densest): same best density, both times
    pk = out.get("peel_hk1.7M", {})
    if pk.get("reference") and pk.get("ours"):
        a = {r[0]: r for r in pk["reference"]}.get("cpu_greedy_peel")
        b = {r[0]: r for r in pk["ours"]}.get("greedy_peel")
        if a and b:
            out["greedy_peel_hk1.7M"] = {"reference_ms": float(a[8]), "ours_ms": float(b[8]),
                                         "same_result": a[2:6] == b[2:6]}
            ok &= out["greedy_peel_hk1.7M"]["same_result"]
    # densest-subgraph pipeline: stage times side by side (the reference's CPU stages vs this library's) and the
    # results, which must be the same subgraphs
    stages = [("gpu_core_decomp", "gpu_core_decomp"), ("cpu_greedy", "greedy"), ("prune_kcore", "prune_kcore"),
              ("cpu_greedy_pp_pruned", "greedy_pp_pruned"),
              ("cpu_core_exact_pruned_seeded", "core_exact_pruned_seeded"), ("pipeline_gpu_core", "pipeline_gpu_core")]
    for name in ("dsg_hk8298", "dsg_hk1.7M"):
        d = out.get(name, {})
        if not (d.get("reference") and d.get("ours")):
            continue
        ref_rows = {r[0]: r for r in d["reference"]}
        our_rows = {r[0]: r for r in d["ours"]}
        summ = {}
        for rn, on in stages:
            if rn in ref_rows and on in our_rows:
                a, b = ref_rows[rn], our_rows[on]
                summ[on] = {"reference_ms": float(a[7]), "ours_ms": float(b[7]), "same_result": a[2:6] == b[2:6]}
                ok &= summ[on]["same_result"]
        if "pipeline_gpu_core" in summ:
            p = summ["pipeline_gpu_core"]
            p["speedup"] = p["reference_ms"] / max(p["ours_ms"], 1e-9)
        out[name + "_stages"] = summ
    out["all_verified"] = bool(ok)
    print(json.dumps(out), flush=True)
    return 0 if ok else 1


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--workload", choices=["rmat22", "hk2", "rmat22-full", "batch", "serve", "reference-gpu",
                                           "passes"],
                    default="rmat22",
                    help="rmat22 (default, the headline line) or a secondary workload")
    ap.add_argument("--graphs", type=int, default=4096, help="graphs in the batch workload")
    ap.add_argument("--per-graph-stride", type=int, default=0,
                    help="batch workload: per-graph arms on every k-th graph (0: all graphs when the batch runs alone, "
                         "every 8th in the default run's legs)")
    ap.add_argument("--tc-kernel", choices=["auto", "plain", "hash"], default="auto",
                    help="count kernel of the headline's timed steps (auto: the autotuner's choice)")
    ap.add_argument("--shard", action="store_true",
                    help="with N > 1 GPUs: count ONE graph split into N shards (strong scaling) instead of N replicas")
    ap.add_argument("--scale", type=int, default=SCALE,
                    help="R-MAT scale of the headline workload (22; smaller only for quick checks)")
    ap.add_argument("--requests", type=int, default=600, help="requests in the serve workload")
    ap.add_argument("--slots", type=int, default=0, help="serve workload: concurrent requests (0 = the default 4)")
    ap.add_argument("--rate-fracs", type=float, nargs="+", default=[0.25, 0.5, 0.75, 0.9],
                    help="serve workload: offered Poisson rates as fractions of the measured burst capacity")
    ap.add_argument("--legs", nargs="*", choices=list(LEGS), default=list(LEGS),
                    help="secondary workloads the default (headline) run adds to its line, after the headline "
                         "(none: --legs with no names)")
    ap.add_argument("--legs-budget-s", type=float, default=900.0,
                    help="wall time after which the remaining secondary legs are skipped (recorded as skipped)")
    args = ap.parse_args()
    if args.warmup < 3:
        log("warm-up raised to 3 steps")
        args.warmup = 3
    if not args.per_graph_stride:
        args.per_graph_stride = 1 if args.workload == "batch" else 8
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "passes":
        line = leg_passes(args)
        print(json.dumps(line), flush=True)
        return 0 if line["parity"]["all"] else 1
    if args.workload in LEGS:
        return run_leg(args)
    if args.workload == "reference-gpu":
        return run_reference_gpu(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
