#!/usr/bin/env python3
"""SSSP throughput benchmark (GTEPS) of the B200 persistent consolidation kernel:
the learned-policy kernel against the plain autotuned kernel on the same graph.

Workload (default): R-MAT scale 22 (4,194,304 vertices), edge factor 16
(67,108,864 generated edges, duplicates and self-loops removed), a=0.57 b=0.19
c=0.19, uint32 weights uniform in [1,255], seeded synthetic graph (seed 1000),
source = highest-out-degree vertex.  One step = one full SSSP from that source.

  plain    the autotuner picks fixed parameters on this graph (outside the timed
           region); K steps of that configuration are timed first
  value    GTEPS = m_r / kernel time (m_r = out-edges of reached vertices) of the
           learned-policy kernel (nested-parallelism_b200/policy_weights.npz; the MLP
           chooses bucket widths and levels, a short autotune of its own picks the
           degree threshold and block shape); graph
           resident in HBM, L2 flushed between steps, CUDA events on the launch stream
  e2e      the same metric through the public host-buffer call nps.sssp(): pinned
           host CSR -> device, kernel, distances -> host, every step
  roofline B_alg = 12 m_r + 12 n_r + 4 n bytes per SSSP over the measured HBM peak
  cpu_baseline  the reference's SSSP_CPU (heap Dijkstra, built from its sources
           into oracle/_ref) timed on this host, one full SSSP of the workload;
           its distances must equal both GPU arms'

`--impl reference` times the reference's CPU SSSP (oracle/_ref, else the oracle
restatement) on all host cores: the K steps run concurrently, one process each.
Multi-GPU (torchrun): replicas only for one graph -- every rank solves its own
copy, the value is the sum of edges over the max device time across ranks;
`--workload batch64` shards the 64-instance batch over the ranks instead.
"""
from __future__ import annotations

import argparse
import contextlib
import dataclasses
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (kind, args, description)
    "rmat22": ("rmat_eval", dict(scale=22, edge_factor=16, seeds=tuple(range(1000, 1010)), tune_seed=999),
               "R-MAT scale 22, edge factor 16, a=.57 b=.19 c=.19, w in [1,255], deduped, source = highest "
               "out-degree vertex; the learned policy's ten held-out evaluation graphs, seeds 1000-1009"),
    "rmat20": ("rmat", dict(scale=20, edge_factor=16, seed=1),
               "R-MAT scale 20, edge factor 16, a=.57 b=.19 c=.19, w in [1,255], seed 1, deduped"),
    "grid4096": ("grid", dict(rows=4096, cols=4096, drop=0.05, wmax=1000, seed=1),
                 "4096x4096 4-neighbour grid, 5% pairs dropped, w in [1,1000], seed 1, source (0,0)"),
    "uniform16k": ("uniform", dict(n=16384, m=131072, wmax=100, seed=1),
                   "uniform random 16,384 vertices / 131,072 edges, w in [1,100], seed 1, source 0"),
    "degree22": ("degree", dict(scale=22, edge_factor=16, seed=1000),
                 "degree statistics (the reference's graph analyzer) of R-MAT scale 22, edge factor 16, "
                 "seed 1000: extremes, totals, 8-bin histogram and full distribution"),
    "solutions22": ("solutions", dict(scale=22, edge_factor=16, seed=1000),
                    "ablation: SSSP_GPU solutions 0-6 (thread queue, dual queue, shared / global delayed "
                    "buffer, naive / per-block nested launch, consolidation plain and learned) on R-MAT scale 22, "
                    "edge factor 16, seed 1000"),
    "bfs22": ("bfs", dict(scale=22, edge_factor=16, seed=1000),
              "breadth-first levels (bfs-rec's bfs_rec_dp_cons_gpu) on R-MAT scale 22, edge factor 16, "
              "seed 1000, source 0; unit edge weights, no weight array read"),
    "spmv22": ("spmv", dict(scale=22, edge_factor=16, seed=1000),
               "y = A x in double (the SpMV application's spmv_np_consolidate_gpu) for the R-MAT scale 22, "
               "edge factor 16, seed 1000 matrix with the reference's data: val[i] = i%13+0.5, x[i] = i%17+0.5"),
    "bc14": ("bc", dict(scale=14, edge_factor=16, seed=1000),
             "betweenness centrality (the bc application's bc_np_consolidate_gpu) of R-MAT scale 14, edge "
             "factor 16, seed 1000, every vertex a source in id order, as the reference computes it"),
    "color22": ("color", dict(scale=22, edge_factor=16, seed=1000),
                "graph coloring (the graph-color application's gclr_np_consolidate_gpu) of R-MAT scale 22, "
                "edge factor 16, seed 1000 (1,295 colors, so 1,295 reference iterations)"),
    "batch64": ("batch", dict(count=64, seed=7),
                "64 R-MAT instances (a=.57 b=.19 c=.19), scale U{12..18}, edge factor {4,8,16,32}, "
                "w in [1,255], random sources, seed 7; one persistent CUDA-graph launch per shard"),
}

METRIC = "SSSP GTEPS on 1 B200: learned-policy vs plain, % of HBM roofline, bit-exact"
LEARNED_AXES = {"threshold": [16, 32, 64, 128], "block_size": [256, 512]}
LEARNED_TUNE_BUDGET = 8

# autotuner seed configuration per workload class (--delta / --level pin it instead)
DEFAULT_PARAMS = {
    "rmat": dict(level=2, threshold=64, delta=0, block_size=512),
    "grid": dict(level=2, threshold=64, delta=4096, block_size=256),
    "uniform": dict(level=2, threshold=64, delta=64, block_size=256),
}


def make_graph(nps, name):
    kind, a, _ = WORKLOADS[name]
    if kind == "rmat":
        return nps.gen_rmat(a["scale"], a["edge_factor"], seed=a["seed"])
    if kind == "grid":
        return nps.gen_grid(a["rows"], a["cols"], a["drop"], a["wmax"], a["seed"])
    return nps.gen_uniform(a["n"], a["m"], a["wmax"], a["seed"])


def _traffic(key):
    """DRAM bytes of one launch of the workload's dominant kernel, from the ncu capture recorded
    in profiles/traffic.json (null when none was recorded)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f).get(key)


def host_call_h2d_bytes(n, m, wmax):
    """Bytes one host-pointer nps.sssp call copies to the device: the row offsets and
    columns as given, the weights packed to 1 or 2 bytes when the largest fits and the
    graph has at least 2^20 edges (the library's rule), else 4 bytes each."""
    wb = 4
    if m >= 1 << 20:
        wb = 1 if wmax <= 0xFF else (2 if wmax <= 0xFFFF else 4)
    return 4 * (n + 1) + 4 * m + wb * m


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, copy)"
    return 6650.0, "fallback 6.65 TB/s"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            time.sleep(0.25)
            self.p.terminate()
            self.p.wait()

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ---------------------------------------------------------------------------
# reference arm: the reference's CPU SSSP on all host cores

_REF_GRAPH = None


def _ref_init(path):
    """Pool initializer: load the graph once per worker process (outside the timed region)."""
    global _REF_GRAPH
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    z = np.load(path)
    _REF_GRAPH = (z["row"], z["col"], z["w"])


def _ref_ready(_):
    return _REF_GRAPH is not None


def _ref_worker(args):
    src, use_ref = args
    import oracle
    row, col, w = _REF_GRAPH
    if use_ref:
        d, t = oracle.ref_sssp_cpu(row, col, w, src)
    else:
        d, t = oracle.timed(oracle.sssp_heap, row, col, w, src)
    return t, oracle.fnv1a(d)


def run_reference(a, nps, g, m_r, n_r, cfg):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import multiprocessing as mp
    import oracle
    use_ref = oracle.have_reference()
    cores = os.cpu_count() or 1
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = 64 << 30
    per_proc = (g.m * 8 + g.n * 12) * 3 + (m_r * 8) + (110 << 20)
    procs = max(1, min(a.steps, cores, int(avail * 0.6 // per_proc)))
    with tempfile.TemporaryDirectory(dir="/dev/shm" if os.path.isdir("/dev/shm") else None) as td:
        path = os.path.join(td, "g.npz")
        np.savez(path, row=g.row_ptr, col=g.col, w=g.w)
        ctx = mp.get_context("spawn")
        with ctx.Pool(procs, initializer=_ref_init, initargs=(path,)) as pool:
            # warm-up: every worker has loaded the graph and imported the oracle before timing
            assert all(pool.map(_ref_ready, range(procs * a.warmup), chunksize=1))
            t0 = time.perf_counter()
            res = pool.map(_ref_worker, [(g.source, use_ref)] * a.steps, chunksize=1)
            wall = time.perf_counter() - t0
    times = [r[0] for r in res]
    value = a.steps * m_r / wall / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * statistics.mean(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": procs,
                         "kind": "reference" if use_ref else "port",
                         "sample": f"{a.steps} full SSSPs of the workload run concurrently, one process "
                                   f"each ({procs} at a time), "
                                   + ("the reference's SSSP_CPU (apps/sssp/src/cpu/sssp.cpp) built from "
                                      "its sources" if use_ref else "the oracle's restatement of SSSP_CPU")},
        "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "warmup_note": "warm-up = each worker process loads the graph and the library before timing",
    }
    return line


# ---------------------------------------------------------------------------
# batched workload: every rank solves its LPT shard of the 64 instances in one
# persistent launch replayed from a CUDA graph (weak in instances per launch,
# no exchange during the solve; results all-gathered at the end)

BATCH_AXES = {"level": [1, 2, 3], "threshold": [32, 64, 128], "delta": [0, 32, 128, 1024],
              "block_size": [256, 512]}


def _batch_reference(a, B, count, seed, cfg):
    """--impl reference for the batch: the reference's SSSP_CPU over all instances,
    one process per host core, each step = the whole batch."""
    import multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    use_ref = oracle.have_reference()
    items = B.rmat_batch(count, seed)
    m_r_total = 0
    with tempfile.TemporaryDirectory(dir="/dev/shm" if os.path.isdir("/dev/shm") else None) as td:
        paths = []
        for it in items:
            d0 = oracle.sssp_heap(it.graph.row_ptr, it.graph.col, it.graph.w, it.source)
            m_r_total += oracle.reached(it.graph.row_ptr, d0)[1]
            path = os.path.join(td, f"g{it.index}.npz")
            np.savez(path, row=it.graph.row_ptr, col=it.graph.col, w=it.graph.w, src=it.source)
            paths.append(path)
        cores = os.cpu_count() or 1
        ctx = mp.get_context("spawn")
        with ctx.Pool(min(cores, count)) as pool:
            for _ in range(a.warmup):
                pool.map(_batch_ref_worker, [(p, use_ref) for p in paths[:min(cores, count)]], chunksize=1)
            t0 = time.perf_counter()
            for _ in range(a.steps):
                pool.map(_batch_ref_worker, [(p, use_ref) for p in paths], chunksize=1)
            wall = time.perf_counter() - t0
    value = a.steps * m_r_total / wall / 1e9
    return {"impl": "reference", "metric": "sssp_batch_gteps", "value": value, "unit": "GTEPS", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * wall / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": min(cores, count),
                             "kind": "reference" if use_ref else "port",
                             "sample": f"each step: all {count} instances, one SSSP_CPU per instance, "
                                       f"{min(cores, count)} processes"},
            "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def _batch_ref_worker(args):
    path, use_ref = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    z = np.load(path)
    if use_ref:
        d, t = oracle.ref_sssp_cpu(z["row"], z["col"], z["w"], int(z["src"]))
    else:
        d, t = oracle.timed(oracle.sssp_heap, z["row"], z["col"], z["w"], int(z["src"]))
    return t


def bench_batch(a, nps, ws, rank, local, desc):
    import torch
    import torch.distributed as dist
    B = importlib.import_module("nested-parallelism_b200.batch")
    at = importlib.import_module("nested-parallelism_b200.autotune")
    _, args, _ = WORKLOADS[a.workload]
    count, seed = args["count"], args["seed"]
    cfg = {"workload": a.workload, "description": desc, "instances": count}
    if a.impl == "reference":
        if rank == 0:
            cfg["parallelism"] = "host cores"
            print(json.dumps(_batch_reference(a, B, count, seed, cfg)))
        return 0
    if ws > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    mine = B.shard_indices(count, seed, ws, rank)
    items = B.rmat_batch(count, seed, only=mine)
    dgs = [at.to_device(it.graph, it.source, dev) for it in items]
    params, tune_ms, tune_log = at.autotune(dgs, repeats=2, budget=a.tune_budget, axes=BATCH_AXES, batch=True)
    params.device = local
    insts = [nps.Instance(d.row_ptr, d.col, d.w, d.dist, d.n, d.m, d.src) for d in dgs]
    stream = torch.cuda.Stream(dev)
    sptr = stream.cuda_stream
    with torch.cuda.stream(stream):
        for _ in range(a.warmup):
            nps.sssp_batch(insts, params, use_graph=True, stream=sptr)
    torch.cuda.synchronize(dev)
    dists = [d.dist.cpu().numpy().view(np.uint32).copy() for d in dgs]
    m_r = n_r = 0
    b_alg = 0
    for it, dd in zip(items, dists):
        reached = dd < nps.INF
        mr = int(np.diff(it.graph.row_ptr)[reached].sum())
        nr = int(reached.sum())
        m_r += mr
        n_r += nr
        b_alg += 12 * mr + 12 * nr + 4 * it.graph.n
    flush = torch.empty(256 << 20, dtype=torch.int8, device=dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            for i in range(a.steps):
                flush.fill_(i & 0x7F)
                evs[i][0].record(stream)
                nps.sssp_batch(insts, params, use_graph=True, stream=sptr)
                evs[i][1].record(stream)
        torch.cuda.synchronize(dev)
    if ws > 1:
        dist.barrier()
    kern_ms = sum(s.elapsed_time(e) for s, e in evs)
    clocks = clk.summary()

    # e2e: host CSR (pinned) -> device, one batch launch, distances -> host, every step
    host = []
    for it in items:
        g = it.graph
        host.append([torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).pin_memory()
                     for x in (g.row_ptr, g.col, g.w)] + [torch.empty(g.n, dtype=torch.int32).pin_memory()])
    h2d = sum(sum(t.numel() * 4 for t in h[:3]) for h in host)
    d2h = sum(h[3].numel() * 4 for h in host)
    e2e_steps = a.e2e_steps or a.steps

    def e2e_step():
        with torch.cuda.stream(stream):
            for h, d in zip(host, dgs):
                d.row_ptr.copy_(h[0], non_blocking=True)
                d.col.copy_(h[1], non_blocking=True)
                d.w.copy_(h[2], non_blocking=True)
            nps.sssp_batch(insts, params, use_graph=True, stream=sptr)
            for h, d in zip(host, dgs):
                h[3].copy_(d.dist, non_blocking=True)
        stream.synchronize()

    e2e_step()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / e2e_steps
    e2e_ok = all(np.array_equal(h[3].numpy().view(np.uint32), dd) for h, dd in zip(host, dists))

    tot = torch.tensor([kern_ms, e2e_ms, float(m_r), float(b_alg)], dtype=torch.float64, device=dev)
    mx = tot.clone()
    sm = tot.clone()
    if ws > 1:
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    kern_max, e2e_max, m_r_all = float(mx[0]), float(mx[1]), float(sm[2])
    results = B.gather_results([{"index": it.index, "fnv1a": nps.fnv1a(dd)} for it, dd in zip(items, dists)])

    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        t_cpu = 0.0
        m_s = 0
        exact = True
        sample = items[:8]
        for it, dd in zip(sample, dists[:8]):
            if oracle.have_reference():
                ref, t = oracle.ref_sssp_cpu(it.graph.row_ptr, it.graph.col, it.graph.w, it.source)
            else:
                ref, t = oracle.timed(oracle.sssp_heap, it.graph.row_ptr, it.graph.col, it.graph.w, it.source)
            t_cpu += t
            m_s += int(np.diff(it.graph.row_ptr)[ref < nps.INF].sum())
            exact = exact and bool(np.array_equal(ref, dd))
        cpu = {"value": m_s / t_cpu / 1e9, "unit": "GTEPS", "cores": 1,
               "kind": "reference" if oracle.have_reference() else "port",
               "sample": "instances 0..7 of the batch, one SSSP_CPU each, 1 thread", "seconds": t_cpu,
               "bit_exact_vs_gpu": exact}
    peak, peak_src = load_peaks()
    per_launch = kern_ms / a.steps * 1e-3
    if rank == 0:
        cfg.update({"parallelism": f"{ws} shards (LPT by n + edges)" if ws > 1 else "1 GPU",
                    "instances_rank0": len(items), "m_reached": int(m_r_all), "params": dataclasses.asdict(params),
                    "autotune": {"evaluations": len(tune_log), "best_ms": tune_ms},
                    "l2": "flushed between steps (256 MB write)", "result_hashes": len(results)})
        line = {"metric": "sssp_batch_gteps", "value": a.steps * m_r_all / (kern_max * 1e-3) / 1e9, "unit": "GTEPS",
                "n_gpus": ws, "steps": a.steps, "warmup": a.warmup, "ms_per_step": kern_max / a.steps,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "int32",
                "data": "synthetic", "config": cfg,
                "roofline": {"bound": "hbm", "achieved": b_alg / per_launch / 1e9, "peak": peak, "unit": "GB/s",
                             "frac": b_alg / per_launch / 1e9 / peak, "traffic": None, "peak_source": peak_src,
                             "b_alg_bytes": b_alg},
                "e2e": {"value": m_r_all / (e2e_max * 1e-3) / 1e9, "unit": "GTEPS", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "ms_per_step": e2e_max, "bit_exact_vs_device_run": e2e_ok,
                        "call": "sssp_batch on device copies of pinned host CSR, distances back to pinned host"},
                "gpu_launches": a.steps, "clocks": clocks, "cpu_baseline": cpu}
        print(json.dumps(line))
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def bench_degree(a, nps, ws, rank, local, desc):
    """Degree statistics of the R-MAT scale-22 graph through nps_degree_stats on device
    row offsets (two streaming passes: statistics, then the distribution).  value =
    bytes of row offsets streamed per second; each call is synchronous, so the time
    includes the two launches and the host round trips."""
    _, args, _ = WORKLOADS[a.workload]
    g = nps.gen_rmat(args["scale"], args["edge_factor"], seed=args["seed"])
    cfg = {"workload": a.workload, "description": desc, "n": g.n, "m": g.m}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if a.impl == "reference":
        if rank == 0:
            times = []
            for _ in range(a.warmup):
                oracle.degree_stats(g.row_ptr)
            for _ in range(a.steps):
                _, t = oracle.timed(oracle.degree_stats, g.row_ptr)
                times.append(t)
            bytes_ = 8 * (g.n + 1)
            value = bytes_ * a.steps / sum(times) / 1e9
            print(json.dumps({"impl": "reference", "metric": "degree_stats_gbs", "value": value, "unit": "GB/s",
                              "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
                              "ms_per_step": 1e3 * sum(times) / a.steps, "higher_is_better": True,
                              "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
                              "config": cfg,
                              "cpu_baseline": {"value": value, "unit": "GB/s", "cores": 1, "kind": "port",
                                               "sample": "the oracle's numpy restatement of getStatInfo()"},
                              "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}))
        return 0
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    row = torch.from_numpy(g.row_ptr.view(np.int32)).to(dev)
    want = oracle.degree_stats(g.row_ptr)
    for _ in range(a.warmup):
        st = nps.degree_stats(row, device=local)
    exact = bool(np.array_equal(st["dist"], want["dist"]) and st["max_degree_node"] == want["max_degree_node"])
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        st = nps.degree_stats(row, device=local)
    dt = (time.perf_counter() - t0) / a.steps
    t0 = time.perf_counter()
    for _ in range(a.steps):
        nps.degree_stats(g, device=local)
    dt_e2e = (time.perf_counter() - t0) / a.steps
    bytes_ = 8 * (g.n + 1)  # row offsets, read by both passes
    peak, peak_src = load_peaks()
    if rank == 0:
        cpu = None
        if not a.no_cpu_baseline:
            _, tcpu = oracle.timed(oracle.degree_stats, g.row_ptr)
            cpu = {"value": bytes_ / tcpu / 1e9, "unit": "GB/s", "cores": 1, "kind": "port",
                   "sample": "one run of the oracle's numpy restatement of getStatInfo() on the same graph"}
        print(json.dumps({"metric": "degree_stats_gbs", "value": bytes_ / dt / 1e9, "unit": "GB/s", "n_gpus": ws,
                          "steps": a.steps, "warmup": a.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
                          "config": dict(cfg, exact_vs_oracle=exact, timing="host wall clock per synchronous call"),
                          "roofline": {"bound": "hbm", "achieved": bytes_ / dt / 1e9, "peak": peak, "unit": "GB/s",
                                       "frac": bytes_ / dt / 1e9 / peak, "traffic": None, "peak_source": peak_src},
                          "e2e": {"value": bytes_ / dt_e2e / 1e9, "unit": "GB/s", "h2d_bytes_per_step": 4 * (g.n + 1),
                                  "d2h_bytes_per_step": 8 * (st["max_degree"] + 1), "ms_per_step": dt_e2e * 1e3},
                          "gpu_launches": 2 * a.steps, "cpu_baseline": cpu}))
    return 0


def bench_solutions(a, nps, ws, rank, local, desc):
    """Every case of SSSP_GPU()'s switch on the R-MAT scale-22 bench graph, device
    arrays resident, distances checked against the oracle.  Per solution: median
    device time of the call's iteration loop (CUDA events), GTEPS = reached
    out-edges / that time, and how much work it did.  value = consolidation with
    the learned policy (the headline path); the other solutions are the ablation."""
    _, args, _ = WORKLOADS[a.workload]
    g = nps.gen_rmat(args["scale"], args["edge_factor"], seed=args["seed"])
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    ref = oracle.sssp_heap(g.row_ptr, g.col, g.w, g.source)
    n_r, m_r = oracle.reached(g.row_ptr, ref)
    cfg = {"workload": a.workload, "description": desc, "n": g.n, "m": g.m, "m_reached": m_r, "source": g.source,
           "threshold": 64, "row_per_thread_cta": 256, "timing": "CUDA events around each call's iteration loop"}
    if a.impl == "reference":
        if rank == 0:
            cfg["parallelism"] = "host cores"
            print(json.dumps(run_reference(a, nps, g, m_r, n_r, cfg)))
        return 0
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    at = importlib.import_module("nested-parallelism_b200.autotune")
    pol = importlib.import_module("nested-parallelism_b200.policy")
    dg = at.to_device(g, device=dev)
    reps = max(1, min(a.steps, 3))
    rows = {}

    def run_solution(sol):
        stats = []
        for i in range(1 + reps):  # one untimed call first (workspace, device runtime set-up)
            d_cost = torch.full((g.n,), nps.INF, dtype=torch.int32, device=dev)
            d_upd = torch.zeros(g.n, dtype=torch.uint8, device=dev)
            d_cost[g.source] = 0
            d_upd[g.source] = 1
            st, info = nps.sssp_solution_state(sol, dg.row_ptr, dg.col, dg.w, d_cost, d_upd, g.n, g.m,
                                               nps.Params(device=local, threshold=64, block_size=256))
            if i:
                stats.append((st, info))
        exact = bool((d_cost.cpu().numpy().view(np.uint32) == ref).all())
        return stats, exact

    for sol in range(6):
        stats, exact = run_solution(sol)
        ms = statistics.median(s.kernel_ms for s, _ in stats)
        st, info = stats[-1]
        rows[nps.SOLUTION_NAMES[sol]] = {
            "solution": sol, "ms": ms, "gteps": m_r / ms / 1e6, "exact": exact, "iterations": st.iterations,
            "edges_scanned_per_m_r": st.edges_scanned / max(m_r, 1), "deferred_rows": info.deferred,
            "child_launches": info.child_launches, "launch_fallbacks": info.launch_fallbacks,
            "host_reads": info.host_reads}
    wpath = os.path.join(ROOT, "nested-parallelism_b200", "policy_weights.npz")
    arms = [("plain", nps.Params(device=local, **DEFAULT_PARAMS["rmat"]))]
    if os.path.exists(wpath):
        pol.load_into_kernel(pol.MLPWeights.load(wpath), local)
        arms.append(("learned", nps.Params(device=local, policy=nps.POLICY_LEARNED, light_heavy=False,
                                           **DEFAULT_PARAMS["rmat"])))
    for name, p in arms:
        ms_l = []
        for i in range(3 + reps):
            st = nps.sssp_device(dg.row_ptr, dg.col, dg.w, g.n, g.m, g.source, dg.dist, p)
            if i >= 3:
                ms_l.append(st.kernel_ms)
        exact = bool((dg.dist.cpu().numpy().view(np.uint32) == ref).all())
        ms = statistics.median(ms_l)
        rows[f"sssp_np_consolidate_gpu ({name})"] = {
            "solution": 6, "ms": ms, "gteps": m_r / ms / 1e6, "exact": exact, "iterations": st.iterations,
            "edges_scanned_per_m_r": st.edges_scanned / max(m_r, 1)}
    head = rows[f"sssp_np_consolidate_gpu ({arms[-1][0]})"]
    if rank == 0:
        print(json.dumps({"metric": "SSSP GTEPS per SSSP_GPU solution (ablation)", "value": head["gteps"],
                          "unit": "GTEPS", "n_gpus": ws, "steps": reps, "warmup": 1, "ms_per_step": head["ms"],
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
                          "data": "synthetic", "config": cfg, "ablation": rows,
                          "all_exact": all(r["exact"] for r in rows.values())}))
    return 0


def bench_bfs(a, nps, ws, rank, local, desc):
    """Breadth-first levels on the SSSP engine (nps_bfs): the unordered frontier
    (the default, headline arm) and one-level buckets, both checked against the oracle.
    value = reached out-edges per second of device time; B_alg = 8 m_r + 12 n_r +
    4 n (column index and level per reached edge; row offsets, level read and
    write per reached vertex; the level array once)."""
    _, args, _ = WORKLOADS[a.workload]
    g = nps.gen_rmat(args["scale"], args["edge_factor"], seed=args["seed"])
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    want = oracle.bfs_levels(g.row_ptr, g.col, g.source)
    reached = want != oracle.BFS_UNDEFINED
    n_r, m_r = int(reached.sum()), int(np.diff(g.row_ptr)[reached].sum())
    cfg = {"workload": a.workload, "description": desc, "n": g.n, "m": g.m, "m_reached": m_r, "n_reached": n_r,
           "source": g.source}
    if a.impl == "reference":
        if rank == 0:
            use_ref = oracle.have_reference_bfs()
            fn = (lambda: oracle.ref_bfs_cpu(g.row_ptr, g.col, g.source)[1]) if use_ref else \
                (lambda: oracle.timed(oracle.bfs_levels, g.row_ptr, g.col, g.source)[1])
            for _ in range(min(a.warmup, 1)):
                fn()
            secs = [fn() for _ in range(a.steps)]
            value = m_r * a.steps / sum(secs) / 1e9
            kind = "reference" if use_ref else "port"
            cpu = {"value": value, "unit": "GTEPS", "cores": 1, "kind": kind,
                   "sample": ("the reference's bfs_cpu (apps/bfs-rec/src/gpu/bfs_rec.cpp:100-119, built from its "
                              "sources), one full BFS per step, 1 thread") if use_ref else
                             "the oracle's numpy level-synchronous BFS, one full BFS per step"}
            print(json.dumps({"impl": "reference", "metric": "BFS GTEPS", "value": value, "unit": "GTEPS",
                              "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
                              "ms_per_step": 1e3 * sum(secs) / a.steps, "higher_is_better": True,
                              "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
                              "config": dict(cfg, parallelism="host cores"), "cpu_baseline": cpu,
                              "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}))
        return 0
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    row = torch.from_numpy(g.row_ptr.view(np.int32)).to(dev)
    col = torch.from_numpy(g.col.view(np.int32)).to(dev)
    level = torch.empty(g.n, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    arms = {"unordered": nps.bfs_params(device=local),
            "levels": nps.bfs_params(device=local, delta=1)}

    def timed(p, clk=None):
        with torch.cuda.stream(stream):
            for _ in range(a.warmup):
                nps.bfs_device(row, col, g.n, g.m, g.source, level, p, stream=stream.cuda_stream)
        torch.cuda.synchronize(dev)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
        st = None
        with (clk if clk is not None else contextlib.nullcontext()):
            with torch.cuda.stream(stream):
                for i in range(a.steps):
                    flush.fill_(i & 0x7F)
                    evs[i][0].record(stream)
                    st = nps.bfs_device(row, col, g.n, g.m, g.source, level, p, stream=stream.cuda_stream)
                    evs[i][1].record(stream)
            torch.cuda.synchronize(dev)
        exact = bool((level.cpu().numpy() == want).all())
        return [s_.elapsed_time(e_) for s_, e_ in evs], st, exact

    lv_ms, lv_st, lv_exact = timed(arms["levels"])
    clk = ClockSampler(local)
    ms, st, exact = timed(arms["unordered"], clk)
    per = sum(ms) / a.steps
    value = ws * m_r / (per * 1e-3) / 1e9

    def pinned(x):
        return torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).pin_memory().numpy()
    hg = nps.Graph(pinned(g.row_ptr), pinned(g.col), np.zeros(0, np.uint32), g.source)
    nps.bfs(hg, g.source, arms["unordered"])
    t0 = time.perf_counter()
    e2e_steps = a.e2e_steps or a.steps
    for _ in range(e2e_steps):
        lv, _ = nps.bfs(hg, g.source, arms["unordered"])
    e2e_ms = (time.perf_counter() - t0) / e2e_steps * 1e3
    e2e_ok = bool((lv == want).all())
    peak, peak_src = load_peaks()
    b_alg = 8 * m_r + 12 * n_r + 4 * g.n
    achieved = b_alg / (per * 1e-3) / 1e9
    cpu = None
    if rank == 0 and not a.no_cpu_baseline and oracle.have_reference_bfs():
        lref, tcpu = oracle.ref_bfs_cpu(g.row_ptr, g.col, g.source)
        cpu = {"value": m_r / tcpu / 1e9, "unit": "GTEPS", "cores": 1, "kind": "reference", "seconds": tcpu,
               "sample": "one full BFS by the reference's bfs_cpu (bfs_rec.cpp:100-119), 1 thread",
               "exact_vs_gpu": bool((lref == want).all())}
    if rank == 0:
        print(json.dumps({
            "metric": "BFS GTEPS", "value": value, "unit": "GTEPS", "n_gpus": ws, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": per, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": dict(cfg, params=dataclasses.asdict(arms["unordered"]), iterations=st.iterations,
                           edges_scanned=st.edges_scanned, exact_vs_oracle=exact,
                           l2="flushed between steps (256 MB write)"),
            "one_level_buckets": {"value": ws * m_r / (sum(lv_ms) / a.steps * 1e-3) / 1e9, "unit": "GTEPS",
                                  "ms_per_step": sum(lv_ms) / a.steps, "edges_scanned": lv_st.edges_scanned,
                                  "iterations": lv_st.iterations, "buckets": lv_st.buckets,
                                  "exact_vs_oracle": lv_exact},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": _traffic("bfs22"), "peak_source": peak_src, "b_alg_bytes": b_alg,
                         "b_alg_formula": "8*m_r + 12*n_r + 4*n"},
            "e2e": {"value": ws * m_r / (e2e_ms * 1e-3) / 1e9, "unit": "GTEPS", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": 4 * (g.n + 1) + 4 * g.m, "d2h_bytes_per_step": 4 * g.n,
                    "exact_vs_oracle": e2e_ok, "call": "nps.bfs(host Graph, pinned)"},
            "gpu_launches": 2 * a.steps, "clocks": clk.summary(), "cpu_baseline": cpu}))
    return 0


def bench_spmv(a, nps, ws, rank, local, desc):
    """SpMV on the R-MAT scale-22 matrix at the three consolidation levels (GRID is
    the headline), device arrays resident, L2 flushed between steps, every y
    compared bit for bit with the reference's spmv_omp (exact for its data).
    value = algorithmic bytes / device time, B_alg = 12 m + 20 n + 4: column index
    and value per nonzero, x read once, y written once, row offsets."""
    _, args, _ = WORKLOADS[a.workload]
    g = nps.gen_rmat(args["scale"], args["edge_factor"], seed=args["seed"])
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    val, x = oracle.spmv_data(g.n, g.m)
    b_alg = 12 * g.m + 20 * g.n + 4
    cfg = {"workload": a.workload, "description": desc, "n": g.n, "m": g.m, "threshold": 64}
    if a.impl == "reference":
        if rank == 0:
            use_ref = oracle.have_reference_spmv()
            cores = os.cpu_count() or 1
            fn = (lambda: oracle.ref_spmv_cpu(g.row_ptr, g.col, cores)[3]) if use_ref else \
                (lambda: oracle.timed(oracle.spmv, g.row_ptr, g.col, val, x)[1])
            fn()
            secs = [fn() for _ in range(a.steps)]
            value = b_alg * a.steps / sum(secs) / 1e9
            cpu = {"value": value, "unit": "GB/s", "cores": cores if use_ref else 1,
                   "kind": "reference" if use_ref else "port",
                   "sample": "one full y = A x per step by the reference's spmv_omp (apps/SpMV/src/cpu/"
                             "SpMV_kernel.cpp:26-42, built from its sources) on all host threads" if use_ref else
                             "one full y = A x per step by the oracle's numpy restatement"}
            print(json.dumps({"impl": "reference", "metric": "SpMV GB/s", "value": value, "unit": "GB/s",
                              "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
                              "ms_per_step": 1e3 * sum(secs) / a.steps, "higher_is_better": True,
                              "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                              "config": dict(cfg, parallelism="host cores"), "cpu_baseline": cpu,
                              "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}))
        return 0
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    row = torch.from_numpy(g.row_ptr.view(np.int32)).to(dev)
    col = torch.from_numpy(g.col.view(np.int32)).to(dev)
    dv, dx = torch.from_numpy(val).to(dev), torch.from_numpy(x).to(dev)
    dy = torch.empty(g.n, dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    want = oracle.spmv(g.row_ptr, g.col, val, x)

    def timed(p, clk=None):
        with torch.cuda.stream(stream):
            for _ in range(a.warmup):
                nps.spmv_device(row, col, dv, dx, dy, g.n, g.m, p, stream=stream.cuda_stream)
        torch.cuda.synchronize(dev)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
        with (clk if clk is not None else contextlib.nullcontext()):
            with torch.cuda.stream(stream):
                for i in range(a.steps):
                    flush.fill_(i & 0x7F)
                    evs[i][0].record(stream)
                    nps.spmv_device(row, col, dv, dx, dy, g.n, g.m, p, stream=stream.cuda_stream)
                    evs[i][1].record(stream)
            torch.cuda.synchronize(dev)
        return sum(s_.elapsed_time(e_) for s_, e_ in evs) / a.steps, bool(np.array_equal(dy.cpu().numpy(), want))

    levels = {}
    for lv in (0, 1):
        ms_, ok = timed(nps.Params(device=local, level=lv))
        levels[["warp", "block"][lv]] = {"ms": ms_, "gbs": b_alg / (ms_ * 1e-3) / 1e9, "exact": ok}
    clk = ClockSampler(local)
    head = nps.Params(device=local, level=2)
    ms, exact = timed(head, clk)
    levels["grid"] = {"ms": ms, "gbs": b_alg / (ms * 1e-3) / 1e9, "exact": exact}
    peak, peak_src = load_peaks()
    achieved = b_alg / (ms * 1e-3) / 1e9
    hg = nps.Graph(g.row_ptr, g.col, np.zeros(0, np.uint32), g.source)
    pv = torch.from_numpy(val).pin_memory().numpy()
    px = torch.from_numpy(x).pin_memory().numpy()
    nps.spmv(hg, pv, px, head)
    e2e_steps = a.e2e_steps or a.steps
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        y, _ = nps.spmv(hg, pv, px, head)
    e2e_ms = (time.perf_counter() - t0) / e2e_steps * 1e3
    cpu = None
    if rank == 0 and not a.no_cpu_baseline and oracle.have_reference_spmv():
        yref, _, _, tcpu = oracle.ref_spmv_cpu(g.row_ptr, g.col, 1)
        cpu = {"value": b_alg / tcpu / 1e9, "unit": "GB/s", "cores": 1, "kind": "reference", "seconds": tcpu,
               "sample": "one full y = A x by the reference's spmv_omp (SpMV_kernel.cpp:26-42), 1 thread",
               "exact_vs_gpu": bool(np.array_equal(yref, want) and exact)}
    if rank == 0:
        print(json.dumps({
            "metric": "SpMV GB/s", "value": achieved, "unit": "GB/s", "n_gpus": ws, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(cfg, level="grid", gflops=2 * g.m / (ms * 1e-3) / 1e9, exact_vs_reference=exact,
                           l2="flushed between steps (256 MB write)", levels=levels),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_source": peak_src, "b_alg_bytes": b_alg,
                         "b_alg_formula": "12*m + 20*n + 4"},
            "e2e": {"value": b_alg / (e2e_ms * 1e-3) / 1e9, "unit": "GB/s", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": 4 * (g.n + 1) + 12 * g.m + 8 * g.n, "d2h_bytes_per_step": 8 * g.n,
                    "exact": bool(np.array_equal(y, want)), "call": "nps.spmv(host arrays, pinned values and x)"},
            "gpu_launches": 2 * a.steps, "clocks": clk.summary(), "cpu_baseline": cpu}))
    return 0


def bench_bc(a, nps, ws, rank, local, desc):
    """Betweenness centrality over every source of the R-MAT scale-14 graph in one
    nps_bc call per step.  value = source-edges per second (sources x m / device
    time): each source's forward and backward passes walk the reached rows once
    each.  Exactness: the first 512 sources against the oracle, bit for bit."""
    _, args, _ = WORKLOADS[a.workload]
    g = nps.gen_rmat(args["scale"], args["edge_factor"], seed=args["seed"])
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    cfg = {"workload": a.workload, "description": desc, "n": g.n, "m": g.m, "sources": g.n}
    sample = np.arange(min(512, g.n))
    if a.impl == "reference":
        if rank == 0:
            # bounded sample: the reference's bc_cpu clears an n x n matrix per source and
            # takes hours at this size, so the oracle's restatement runs a 512-source sample
            secs = []
            for _ in range(a.steps):
                _, t = oracle.timed(oracle.bc, g.row_ptr, g.col, sample)
                secs.append(t)
            value = sample.shape[0] * g.m * a.steps / sum(secs) / 1e9
            cpu = {"value": value, "unit": "GTEPS", "cores": 1, "kind": "port",
                   "sample": "the oracle's C restatement of bc_cpu over the first 512 sources per step "
                             "(the reference's bc_cpu clears an n x n byte matrix per source: hours here)"}
            print(json.dumps({"impl": "reference", "metric": "BC GTEPS (source-edges/s)", "value": value,
                              "unit": "GTEPS", "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
                              "ms_per_step": 1e3 * sum(secs) / a.steps, "higher_is_better": True,
                              "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                              "config": dict(cfg, parallelism="host cores", sources=int(sample.shape[0])),
                              "cpu_baseline": cpu,
                              "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}))
        return 0
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    row = torch.from_numpy(g.row_ptr.view(np.int32)).to(dev)
    col = torch.from_numpy(g.col.view(np.int32)).to(dev)
    out = torch.empty(g.n, dtype=torch.float32, device=dev)
    p = nps.Params(device=local)
    b_sample, _ = nps.bc(g, sample, p)
    exact = bool(np.array_equal(b_sample.view(np.uint32), oracle.bc(g.row_ptr, g.col, sample).view(np.uint32)))
    with torch.cuda.stream(stream):
        for _ in range(a.warmup):
            nps.bc_device(row, col, g.n, g.m, out, params=p, stream=stream.cuda_stream)
    torch.cuda.synchronize(dev)
    clk = ClockSampler(local)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    with clk:
        with torch.cuda.stream(stream):
            for i in range(a.steps):
                evs[i][0].record(stream)
                st = nps.bc_device(row, col, g.n, g.m, out, params=p, stream=stream.cuda_stream)
                evs[i][1].record(stream)
        torch.cuda.synchronize(dev)
    ms = sum(s_.elapsed_time(e_) for s_, e_ in evs) / a.steps
    value = g.n * g.m / (ms * 1e-3) / 1e9
    t0 = time.perf_counter()
    bh, _ = nps.bc(g, None, p)
    e2e_ms = (time.perf_counter() - t0) * 1e3
    repeat = bool(np.array_equal(bh.view(np.uint32), out.cpu().numpy().view(np.uint32)))
    if rank == 0:
        cpu = None
        if not a.no_cpu_baseline:
            _, tcpu = oracle.timed(oracle.bc, g.row_ptr, g.col, sample)
            cpu = {"value": sample.shape[0] * g.m / tcpu / 1e9, "unit": "GTEPS", "cores": 1, "kind": "port",
                   "sample": "the oracle's C restatement of bc_cpu over the first 512 sources", "seconds": tcpu}
        print(json.dumps({
            "metric": "BC GTEPS (source-edges/s)", "value": value, "unit": "GTEPS", "n_gpus": ws, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(cfg, grid_ctas=st.grid_ctas, exact_first_512_sources=exact,
                           host_call_matches_device_call=repeat,
                           l2="the graph (5 MB) stays in L2 across sources; the per-source work is the product"),
            "roofline": None,
            "e2e": {"value": g.n * g.m / (e2e_ms * 1e-3) / 1e9, "unit": "GTEPS", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": 4 * (g.n + 1) + 4 * g.m, "d2h_bytes_per_step": 4 * g.n,
                    "call": "nps.bc(host Graph)"},
            "gpu_launches": 3 * a.steps, "clocks": clk.summary(), "cpu_baseline": cpu}))
    return 0


def bench_color(a, nps, ws, rank, local, desc):
    """Graph coloring of the R-MAT scale-22 graph, device arrays resident, colors
    compared exactly with the oracle.  value = edges / device time (each edge is
    read about once by the resumable scan)."""
    _, args, _ = WORKLOADS[a.workload]
    g = nps.gen_rmat(args["scale"], args["edge_factor"], seed=args["seed"])
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    cfg = {"workload": a.workload, "description": desc, "n": g.n, "m": g.m}
    if a.impl == "reference":
        if rank == 0:
            secs = [oracle.timed(oracle.color, g.row_ptr, g.col)[1] for _ in range(a.steps)]
            value = g.m * a.steps / sum(secs) / 1e9
            cpu = {"value": value, "unit": "GTEPS", "cores": 1, "kind": "port",
                   "sample": "the oracle's closed form in id order (C), one full coloring per step; the "
                             "reference has no CPU coloring and its iterations would take n x colors steps"}
            print(json.dumps({"impl": "reference", "metric": "coloring GTEPS", "value": value, "unit": "GTEPS",
                              "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
                              "ms_per_step": 1e3 * sum(secs) / a.steps, "higher_is_better": True,
                              "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
                              "config": dict(cfg, parallelism="host cores"), "cpu_baseline": cpu,
                              "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}))
        return 0
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    row = torch.from_numpy(g.row_ptr.view(np.int32)).to(dev)
    col = torch.from_numpy(g.col.view(np.int32)).to(dev)
    out = torch.empty(g.n, dtype=torch.int32, device=dev)
    want, iters = oracle.color(g.row_ptr, g.col)
    p = nps.Params(device=local)
    with torch.cuda.stream(stream):
        for _ in range(a.warmup):
            nps.color_device(row, col, g.n, g.m, out, p, stream=stream.cuda_stream)
    torch.cuda.synchronize(dev)
    clk = ClockSampler(local)
    ms_l = []
    with clk:
        for _ in range(a.steps):
            st = nps.color_device(row, col, g.n, g.m, out, p, stream=stream.cuda_stream)
            ms_l.append(st.kernel_ms)
    exact = bool(np.array_equal(out.cpu().numpy(), want))
    ms = sum(ms_l) / a.steps
    t0 = time.perf_counter()
    got, _ = nps.color(g, p)
    e2e_ms = (time.perf_counter() - t0) * 1e3
    if rank == 0:
        cpu = None
        if not a.no_cpu_baseline:
            _, tcpu = oracle.timed(oracle.color, g.row_ptr, g.col)
            cpu = {"value": g.m / tcpu / 1e9, "unit": "GTEPS", "cores": 1, "kind": "port", "seconds": tcpu,
                   "sample": "the oracle's closed form in id order (C), one full coloring"}
        print(json.dumps({
            "metric": "coloring GTEPS", "value": g.m / (ms * 1e-3) / 1e9, "unit": "GTEPS", "n_gpus": ws,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": dict(cfg, colors=iters, rounds=st.buckets, edges_scanned=st.edges_scanned,
                           exact_vs_oracle=exact, iterations_match=st.iterations == iters,
                           timing="CUDA events around the call's rounds (host reads the list once per chunk)"),
            "roofline": None,
            "e2e": {"value": g.m / (e2e_ms * 1e-3) / 1e9, "unit": "GTEPS", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": 4 * (g.n + 1) + 4 * g.m, "d2h_bytes_per_step": 4 * g.n,
                    "exact": bool(np.array_equal(got, want)), "call": "nps.color(host Graph)"},
            "gpu_launches": 1 + st.buckets, "clocks": clk.summary(), "cpu_baseline": cpu}))
    return 0


# ---------------------------------------------------------------------------
# The default workload: R-MAT scale 22 on the learned policy's ten held-out
# evaluation seeds.  CPU work runs in spawned processes that build each graph
# with the oracle's restatement of the generator (identical arrays, checked by
# tests/test_oracle_cpu.py), so no CPU process ever loads the library.

def _rmat_cpu_worker(scale, ef, seeds, use_ref, q, go, timeout_s):
    """One host process: build the R-MAT (scale, ef) graphs of `seeds` (each distinct
    seed once), report ready, wait for `go`, then run one single-source search per entry
    of `seeds`, in order, by the reference's SSSP_CPU (oracle/_ref) or, without it, the
    oracle's restatement; report each search's distance hash and time."""
    os.environ["OMP_NUM_THREADS"] = "1"  # one core per process
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    try:
        graphs = {sd: oracle.gen_rmat(scale, ef, sd) for sd in dict.fromkeys(seeds)}
        q.put(("ready", seeds[0]))
        if not go.wait(timeout_s):
            q.put(("error", seeds[0], "start signal never came"))
            return
        for sd in seeds:
            row, col, w, src = graphs[sd]
            if use_ref:
                d, t = oracle.ref_sssp_cpu(row, col, w, src)
            else:
                d, t = oracle.timed(oracle.sssp_heap, row, col, w, src)
            n_r, m_r = oracle.reached(row, d)
            q.put(("done", sd, oracle.fnv1a(d), t, n_r, m_r, src, int(row.shape[0] - 1), int(col.shape[0])))
    except Exception as e:  # reported to the parent, which fails loudly
        q.put(("error", seeds[0], repr(e)))


class CpuSearches:
    """Spawned processes, each with a list of seeds: every process builds its graphs,
    then all start their searches together once every graph is built (synchronized)
    or as soon as their own are (not synchronized).  `runs` lists every search's
    result; `results` keeps the first per seed."""

    def __init__(self, scale, ef, seed_lists, use_ref, synchronized, timeout_s=1800):
        import multiprocessing as mp
        ctx = mp.get_context("spawn")
        self.q, self.go = ctx.Queue(), ctx.Event()
        self.synchronized = synchronized
        if not synchronized:
            self.go.set()
        self.procs = [ctx.Process(target=_rmat_cpu_worker,
                                  args=(scale, ef, list(sl), use_ref, self.q, self.go, timeout_s), daemon=True)
                      for sl in seed_lists if sl]
        self.expected = sum(len(sl) for sl in seed_lists)
        for pr in self.procs:
            pr.start()
        self.timeout_s = timeout_s
        self.wall = None
        self.runs = []
        self.results = {}

    def _get(self):
        """Next message; fails loudly when a process died without answering or the
        whole set ran past its time bound."""
        import queue
        t_end = time.perf_counter() + self.timeout_s
        while True:
            try:
                msg = self.q.get(timeout=5)
                break
            except queue.Empty:
                dead = [pr for pr in self.procs if pr.exitcode not in (None, 0)]
                if dead:
                    raise RuntimeError(f"a CPU search process exited with code {dead[0].exitcode}")
                if time.perf_counter() > t_end:
                    raise RuntimeError("CPU search processes did not answer in time")
        if msg[0] == "error":
            raise RuntimeError(f"CPU search for seed {msg[1]} failed: {msg[2]}")
        return msg

    def start(self):
        """Wait until every graph is built, then start all searches; returns when they end."""
        ready = 0
        while ready < len(self.procs):
            if self._get()[0] == "ready":
                ready += 1
        t0 = time.perf_counter()
        self.go.set()
        self.collect()
        self.wall = time.perf_counter() - t0
        return self.results

    def collect(self):
        while len(self.runs) < self.expected:
            msg = self._get()
            if msg[0] == "done":
                _, seed, h, t, n_r, m_r, src, n, m = msg
                r = dict(seed=seed, fnv=h, seconds=t, n_r=n_r, m_r=m_r, source=src, n=n, m=m)
                self.runs.append(r)
                self.results.setdefault(seed, r)
        for pr in self.procs:
            pr.join(timeout=60)
        return self.results


def _cpu_processes(scale, ef, wanted):
    """Processes to run at once: at most `wanted`, the host's cores, and what 60 % of
    the available memory holds at the generator's peak (about 40 bytes per edge)."""
    cores = os.cpu_count() or 1
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = 64 << 30
    per_proc = (ef << scale) * 40 + (256 << 20)
    return max(1, min(wanted, cores, int(avail * 0.6 // per_proc)))


def _cpu_use_ref():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle.have_reference()


def rmat_eval_config(wl, desc, seeds, per_seed):
    """The config block both arms print for the evaluation workload."""
    return {"workload": wl, "description": desc, "scale": WORKLOADS[wl][1]["scale"],
            "edge_factor": WORKLOADS[wl][1]["edge_factor"], "seeds": list(seeds),
            "n": per_seed[seeds[0]]["n"], "m_per_seed": [per_seed[sd]["m"] for sd in seeds],
            "m_reached_per_seed": [per_seed[sd]["m_r"] for sd in seeds],
            "step": f"one SSSP from the source of each of the {len(seeds)} graphs",
            "l2": "flushed before every SSSP (256 MB write); the 12 B/edge CSR also exceeds L2"}


def reference_rmat_eval(a, wl, desc):
    """--impl reference on the evaluation workload: the reference's SSSP_CPU on the host
    cores.  Each of the K steps is one full SSSP of one evaluation graph (seeds in turn);
    the steps run in parallel processes, one core each, all started together after every
    graph is built, and the value is the reached edges of all K searches over the wall time."""
    _, w, _ = WORKLOADS[wl]
    seeds = list(a.seeds or w["seeds"])
    use_ref = _cpu_use_ref()
    steps = [seeds[i % len(seeds)] for i in range(a.steps)]
    procs = _cpu_processes(w["scale"], w["edge_factor"], len(steps))
    lists = [steps[j::procs] for j in range(procs)]
    cs = CpuSearches(w["scale"], w["edge_factor"], lists, use_ref, synchronized=True)
    res = cs.start()
    wall = cs.wall
    total_edges = sum(r["m_r"] for r in cs.runs)
    value = total_edges / wall / 1e9
    used = sorted(res)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * wall / a.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic", "config": rmat_eval_config(wl, desc, used, res),
        "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": procs,
                         "kind": "reference" if use_ref else "port",
                         "sample": f"{a.steps} full SSSPs, one per step, the evaluation graphs in turn, {procs} "
                                   "processes (one core each) started together; "
                                   + ("the reference's SSSP_CPU (apps/sssp/src/cpu/sssp.cpp) built from its "
                                      "sources" if use_ref else "the oracle's restatement of SSSP_CPU")},
        "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "seconds_per_search": [round(r["seconds"], 3) for r in cs.runs],
        "warmup_note": "warm-up = every process builds its graphs and loads the reference code before the "
                       "timed searches start",
    }
    if use_ref:
        # the reference's other CPU path, usssp_cpu (apps/sssp/src/cpu/sssp_kernel.cpp): an OpenMP frontier
        # sweep on every host thread, on the first graph; its concurrent updates race, so it is reported with
        # whether it matched Dijkstra (distance hash) and never used as a result
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        cores = os.cpu_count() or 1
        sd = used[0]
        row, col, wt, src = oracle.gen_rmat(w["scale"], w["edge_factor"], sd)
        du, tu = oracle.ref_usssp_cpu(row, col, wt, src, threads=cores)
        line["usssp_cpu"] = {"value": res[sd]["m_r"] / tu / 1e9, "unit": "GTEPS", "threads": cores,
                             "seconds": tu, "seed": sd, "equal_to_dijkstra": oracle.fnv1a(du) == res[sd]["fnv"],
                             "exact": False, "note": "racy: concurrent unsynchronised updates (non-exact by design)"}
    return line


def bench_rmat_eval(a, ws, rank, local, wl, desc):
    """Our arm on the evaluation workload: the plain autotuned kernel and the learned
    policy on every evaluation graph, each SSSP checked against the reference's CPU
    Dijkstra run in spawned processes while the GPU works."""
    _, w, _ = WORKLOADS[wl]
    seeds = list(a.seeds or w["seeds"])
    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu_baseline:
        # started before the first CUDA call (spawned processes, no library loaded)
        procs = _cpu_processes(w["scale"], w["edge_factor"], len(seeds))
        cpu = CpuSearches(w["scale"], w["edge_factor"], [seeds[j::procs] for j in range(procs)], _cpu_use_ref(),
                          synchronized=False)
    nps = importlib.import_module("nested-parallelism_b200")
    import torch
    import torch.distributed as dist
    if ws > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    at = importlib.import_module("nested-parallelism_b200.autotune")
    pol = importlib.import_module("nested-parallelism_b200.policy")

    # ---- configuration: the autotuner runs on a graph of the same shape that is not an
    # evaluation graph (seed tune_seed), outside any timed region
    prm = dict(DEFAULT_PARAMS["rmat"])
    if a.delta is not None:
        prm["delta"] = a.delta
    if a.level is not None:
        prm["level"] = a.level
    wpath = os.path.join(ROOT, "nested-parallelism_b200", "policy_weights.npz")
    use_learned = a.policy == "learned" and os.path.exists(wpath)
    if use_learned:
        pol.load_into_kernel(pol.MLPWeights.load(wpath), local)
    tune_log = []
    sched = nps.SCHEDULE_ASYNC if a.schedule == "async" else nps.SCHEDULE_ITERATIONS
    if sched == nps.SCHEDULE_ASYNC:
        prm["light_heavy"] = False
    plain = nps.Params(device=local, schedule=sched, **prm)
    learned = dataclasses.replace(plain, policy=nps.POLICY_LEARNED, light_heavy=False, order_degree=0,
                                  delta_schedule=0) if use_learned else None
    if a.tune_budget > 0 and a.delta is None and a.level is None:
        gt = nps.gen_rmat(w["scale"], w["edge_factor"], seed=w["tune_seed"])
        dgt = at.to_device(gt, device=dev)
        plain, _, tune_log = at.autotune([dgt], repeats=3, budget=a.tune_budget, seed=plain)
        plain.device = local
        if use_learned:
            learned = dataclasses.replace(plain, policy=nps.POLICY_LEARNED, light_heavy=False, order_degree=0,
                                          delta_schedule=0)
            learned, _, ltune = at.autotune([dgt], repeats=3, budget=LEARNED_TUNE_BUDGET, seed=learned,
                                            axes=LEARNED_AXES)
            learned.device = local
            tune_log = tune_log + ltune
        del dgt, gt
    params = learned if use_learned else plain

    # ---- the evaluation graphs, resident on the device
    graphs = []
    for sd in seeds:
        g = nps.gen_rmat(w["scale"], w["edge_factor"], seed=sd)
        graphs.append((sd, g, at.to_device(g, device=dev)))
    flush = torch.empty(256 << 20, dtype=torch.int8, device=dev)  # > 126 MB L2
    stream = torch.cuda.Stream(dev)
    sptr = stream.cuda_stream

    def timed(p, clk=None):
        """W warm-up SSSPs per graph, then K steps of one SSSP per graph, the L2 flushed
        before each; CUDA events on the launch stream around every SSSP."""
        with torch.cuda.stream(stream):
            for _ in range(a.warmup):
                for _, g, dg in graphs:
                    nps.sssp_device(dg.row_ptr, dg.col, dg.w, g.n, g.m, g.source, dg.dist, p, stream=sptr)
        torch.cuda.synchronize(dev)
        evs = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                for _ in graphs] for _ in range(a.steps)]
        stats = [None] * len(graphs)
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        ctx = clk if clk is not None else contextlib.nullcontext()
        with ctx:
            with torch.cuda.stream(stream):
                for i in range(a.steps):
                    for j, (_, g, dg) in enumerate(graphs):
                        flush.fill_((i * len(graphs) + j) & 0x7F)
                        evs[i][j][0].record(stream)
                        stats[j] = nps.sssp_device(dg.row_ptr, dg.col, dg.w, g.n, g.m, g.source, dg.dist, p,
                                                   stream=sptr)
                        evs[i][j][1].record(stream)
                torch.cuda.synchronize(dev)
        if ws > 1:
            dist.barrier()
        ms = [[evs[i][j][0].elapsed_time(evs[i][j][1]) for i in range(a.steps)] for j in range(len(graphs))]
        return ms, stats

    def distances(p):
        out = []
        for _, g, dg in graphs:
            nps.sssp_device(dg.row_ptr, dg.col, dg.w, g.n, g.m, g.source, dg.dist, p)
            out.append(dg.dist.cpu().numpy().view(np.uint32).copy())
        return out

    plain_ms, plain_stats = timed(plain)
    d_plain = distances(plain)
    per = {}
    for j, (sd, g, _) in enumerate(graphs):
        reached = d_plain[j] < nps.INF
        n_r = int(reached.sum())
        m_r = int(np.diff(g.row_ptr)[reached].sum())
        per[sd] = dict(n=g.n, m=g.m, m_r=m_r, n_r=n_r, source=g.source, b_alg=12 * m_r + 12 * n_r + 4 * g.n,
                       wmax=int(g.w.max()) if g.m else 0)
    clk = ClockSampler(local)
    step_ms, stats = timed(params, clk)
    clocks = clk.summary()
    d_head = distances(params)
    exact_vs_plain = all(np.array_equal(x, y) for x, y in zip(d_head, d_plain))

    # ---- e2e: the public host-buffer call, pinned host CSR in, distances out, every SSSP
    def pinned(x):
        return torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).pin_memory().numpy()
    hosts = [(nps.Graph(pinned(g.row_ptr), pinned(g.col), pinned(g.w).view(np.uint32), g.source),
              torch.empty(g.n, dtype=torch.int32).pin_memory().numpy().view(np.uint32)) for _, g, _ in graphs]
    e2e_steps = a.e2e_steps or 1
    nps.sssp(hosts[0][0], None, params, out=hosts[0][1])
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for hg, hout in hosts:
            nps.sssp(hg, None, params, out=hout)  # synchronous: H2D + kernel + D2H
    e2e_wall = time.perf_counter() - t0
    e2e_ok = all(np.array_equal(hout, d) for (_, hout), d in zip(hosts, d_head))
    del hosts

    seed_ms = [sum(x) for x in step_ms]             # per graph, over K steps
    plain_seed_ms = [sum(x) for x in plain_ms]
    kern_ms = sum(seed_ms)
    tot_t = torch.tensor([kern_ms, e2e_wall * 1e3, sum(plain_seed_ms)], dtype=torch.float64, device=dev)
    if ws > 1:
        dist.all_reduce(tot_t, op=dist.ReduceOp.MAX)
    kern_ms_max, e2e_ms_max, plain_ms_max = float(tot_t[0]), float(tot_t[1]), float(tot_t[2])
    mr = [per[sd]["m_r"] for sd in seeds]
    gteps = [a.steps * m / (t * 1e-3) / 1e9 for m, t in zip(mr, seed_ms)]
    plain_gteps = [a.steps * m / (t * 1e-3) / 1e9 for m, t in zip(mr, plain_seed_ms)]
    geo = float(np.exp(np.mean(np.log(gteps))))
    plain_geo = float(np.exp(np.mean(np.log(plain_gteps))))
    # aggregate over ranks (replicas): every rank solved every graph K times
    value = ws * geo * kern_ms / kern_ms_max
    aggregate = ws * a.steps * sum(mr) / (kern_ms_max * 1e-3) / 1e9
    e2e_value = ws * e2e_steps * sum(mr) / (e2e_ms_max * 1e-3) / 1e9

    peak, peak_src = load_peaks()
    b_alg = [per[sd]["b_alg"] for sd in seeds]
    achieved = a.steps * sum(b_alg) / (kern_ms * 1e-3) / 1e9
    traffic = _traffic(wl + ("_learned" if use_learned else ""))

    cpu_line = None
    if cpu is not None:
        res = cpu.collect()
        fn = nps.fnv1a
        exact = {str(sd): bool(res[sd]["fnv"] == fn(d_head[j]) and res[sd]["fnv"] == fn(d_plain[j]))
                 for j, sd in enumerate(seeds)}
        secs = [res[sd]["seconds"] for sd in seeds]
        use_ref = _cpu_use_ref()
        cpu_line = {"value": float(np.mean([m / t / 1e9 for m, t in zip(mr, secs)])), "unit": "GTEPS", "cores": 1,
                    "kind": "reference" if use_ref else "port",
                    "sample": f"one full SSSP of each of the {len(seeds)} graphs, 1 thread each, "
                              + ("by the reference's SSSP_CPU (heap Dijkstra, apps/sssp/src/cpu/sssp.cpp, built "
                                 "from its sources), including its Heap() init" if use_ref else
                                 "by the oracle's restated heap Dijkstra")
                              + f"; the {len(seeds)} processes ran at once, beside the GPU timing",
                    "seconds_per_seed": {str(sd): t for sd, t in zip(seeds, secs)},
                    "bit_exact_vs_gpu": all(exact.values()), "bit_exact_per_seed": exact}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": ws, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": kern_ms_max / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": rmat_eval_config(wl, desc, seeds, per),
            "value_definition": "geometric mean over the graphs of m_r * K / (sum of the graph's K CUDA-event "
                                "SSSP times); aggregate_gteps = all reached edges / all SSSP time",
            "aggregate_gteps": aggregate,
            "ms_per_sssp": kern_ms_max / a.steps / len(seeds),
            "policy": "learned" if use_learned else "plain",
            "params": dataclasses.asdict(params),
            "parallelism": f"replicas x{ws}" if ws > 1 else "1 GPU",
            "tuning": {"graph": f"R-MAT scale {w['scale']} seed {w['tune_seed']} (not an evaluation graph)",
                       "autotune_evaluations": len(tune_log)},
            "per_seed": [{"seed": sd, "m_r": per[sd]["m_r"], "ms": seed_ms[j] / a.steps,
                          "gteps": gteps[j], "plain_ms": plain_seed_ms[j] / a.steps, "plain_gteps": plain_gteps[j],
                          "iterations": stats[j].iterations, "buckets": stats[j].buckets,
                          "edges_scanned": stats[j].edges_scanned,
                          "plain_iterations": plain_stats[j].iterations,
                          "plain_edges_scanned": plain_stats[j].edges_scanned,
                          "step_ms_min": min(step_ms[j]), "step_ms_max": max(step_ms[j])}
                         for j, sd in enumerate(seeds)],
            "plain": {"value": plain_geo, "unit": "GTEPS", "ms_per_step": plain_ms_max / a.steps,
                      "params": dataclasses.asdict(plain),
                      "note": "plain autotuned kernel (fixed parameters, no policy), same graphs, same timing"},
            "learned_over_plain": (geo / plain_geo) if use_learned else None,
            "bit_exact": {"learned_vs_plain": exact_vs_plain,
                          "vs_cpu_dijkstra": cpu_line["bit_exact_vs_gpu"] if cpu_line else None},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                         "traffic_note": "DRAM bytes of one launch on seed 1000 (profiles/traffic.json)",
                         "b_alg_bytes_per_seed": b_alg, "b_alg_formula": "12*m_r + 12*n_r + 4*n"},
            "e2e": {"value": e2e_value, "unit": "GTEPS",
                    "h2d_bytes_per_step": sum(host_call_h2d_bytes(per[sd]["n"], per[sd]["m"], per[sd]["wmax"])
                                              for sd in seeds),
                    "d2h_bytes_per_step": sum(4 * per[sd]["n"] for sd in seeds),
                    "ms_per_step": e2e_ms_max / e2e_steps, "steps": e2e_steps,
                    "bit_exact_vs_device_run": e2e_ok,
                    "call": "nps.sssp(host Graph, pinned) once per graph per step; weights in [1, 255] cross "
                            "PCIe as one byte each (packed on the host during the column copy, widened on the "
                            "device)"},
            "gpu_launches": a.steps * len(seeds),
            "clocks": clocks,
            "cpu_baseline": cpu_line,
        }
        print(json.dumps(line))
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rmat22", choices=sorted(WORKLOADS))
    ap.add_argument("--delta", type=int, default=None)
    ap.add_argument("--level", type=int, default=None)
    ap.add_argument("--policy", default=None, choices=["plain", "learned"],
                    help="arm reported as `value` (default: learned for rmat22, the learned-policy workload, "
                         "plain for the plain-SSSP workloads rmat20, grid4096 and uniform16k)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--tune-budget", type=int, default=24, help="autotuner evaluations before timing")
    ap.add_argument("--seeds", default=None, help="rmat22 only: comma-separated subset of the evaluation seeds")
    ap.add_argument("--schedule", default="iterations", choices=["iterations", "async"],
                    help="SSSP schedule of both arms: frontier iterations with a team barrier each, or asynchronous "
                         "buckets (NPS_SCHEDULE_ASYNC)")
    a = ap.parse_args()
    if a.policy is None:
        a.policy = "learned" if a.workload == "rmat22" else "plain"
    a.warmup = max(a.warmup, 3)
    a.seeds = tuple(int(x) for x in a.seeds.split(",")) if a.seeds else None

    ws, rank, local = dist_env()
    kind, _, desc = WORKLOADS[a.workload]
    if kind == "rmat_eval":
        if a.impl == "reference":
            if rank != 0:
                return 0
            print(json.dumps(reference_rmat_eval(a, a.workload, desc)))
            return 0
        return bench_rmat_eval(a, ws, rank, local, a.workload, desc)
    nps = importlib.import_module("nested-parallelism_b200")
    if kind == "batch":
        return bench_batch(a, nps, ws, rank, local, desc)
    if kind == "degree":
        return bench_degree(a, nps, ws, rank, local, desc)
    if kind == "solutions":
        return bench_solutions(a, nps, ws, rank, local, desc)
    if kind == "bfs":
        return bench_bfs(a, nps, ws, rank, local, desc)
    if kind == "spmv":
        return bench_spmv(a, nps, ws, rank, local, desc)
    if kind == "bc":
        return bench_bc(a, nps, ws, rank, local, desc)
    if kind == "color":
        return bench_color(a, nps, ws, rank, local, desc)
    prm = dict(DEFAULT_PARAMS[kind])
    if a.delta is not None:
        prm["delta"] = a.delta
    if a.level is not None:
        prm["level"] = a.level
    if a.schedule == "async":
        prm["schedule"] = 1  # NPS_SCHEDULE_ASYNC
        prm["light_heavy"] = False

    if a.impl == "reference":
        if rank != 0:
            return 0
        g = make_graph(nps, a.workload)
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        d0 = oracle.sssp_heap(g.row_ptr, g.col, g.w, g.source)
        n_r, m_r = oracle.reached(g.row_ptr, d0)
        cfg = {"workload": a.workload, "description": desc, "n": g.n, "m": g.m, "m_reached": m_r,
               "source": g.source, "parallelism": "host cores"}
        line = run_reference(a, nps, g, m_r, n_r, cfg)
        if oracle.have_reference():
            # the reference's other CPU path, usssp_cpu (apps/sssp/src/cpu/sssp_kernel.cpp): an OpenMP
            # frontier sweep on every host thread; its concurrent updates race, so it is reported
            # with its mismatch count and never used as a result
            threads = os.cpu_count() or 1
            du, tu = oracle.ref_usssp_cpu(g.row_ptr, g.col, g.w, g.source, threads=threads)
            line["usssp_cpu"] = {"value": m_r / tu / 1e9, "unit": "GTEPS", "threads": threads, "seconds": tu,
                                 "mismatches_vs_dijkstra": int((du != d0).sum()), "exact": False,
                                 "note": "racy: concurrent unsynchronised updates (non-exact by design)"}
        print(json.dumps(line))
        return 0

    import torch
    import torch.distributed as dist
    if ws > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    at = importlib.import_module("nested-parallelism_b200.autotune")
    pol = importlib.import_module("nested-parallelism_b200.policy")

    g = make_graph(nps, a.workload)
    dg = at.to_device(g, device=dev)
    row, col, w, dist_t = dg.row_ptr, dg.col, dg.w, dg.dist

    # plain autotuned configuration: the autotuner on this graph (outside the timed region),
    # unless --delta / --level pin it
    tune_log = []
    if a.tune_budget > 0 and a.delta is None and a.level is None:
        seed_p = nps.Params(device=local, **prm)
        plain, _, tune_log = at.autotune([dg], repeats=3, budget=a.tune_budget, seed=seed_p)
        plain.device = local
    else:
        plain = nps.Params(device=local, **prm)
    wpath = os.path.join(ROOT, "nested-parallelism_b200", "policy_weights.npz")
    use_learned = a.policy == "learned" and os.path.exists(wpath)
    learned = None
    if use_learned:
        pol.load_into_kernel(pol.MLPWeights.load(wpath), local)
        learned = dataclasses.replace(plain, policy=nps.POLICY_LEARNED, light_heavy=False, order_degree=0,
                                      delta_schedule=0)
        if tune_log:
            # the learned arm's static parameters (degree threshold, block shape) get their
            # own short autotune; the policy itself picks widths and levels
            learned, _, ltune = at.autotune([dg], repeats=3, budget=LEARNED_TUNE_BUDGET, seed=learned,
                                            axes=LEARNED_AXES)
            learned.device = local
            tune_log = tune_log + ltune
    params = learned if use_learned else plain

    flush = torch.empty(256 << 20, dtype=torch.int8, device=dev)  # > 126 MB L2
    stream = torch.cuda.Stream(dev)
    sptr = stream.cuda_stream

    def step(p):
        return nps.sssp_device(row, col, w, g.n, g.m, g.source, dist_t, p, stream=sptr)

    def timed(p, clk=None):
        """W warm-up steps, then K steps with an L2 flush before each; CUDA events
        on the launch stream around each SSSP.  Returns (per-step ms, stats, dist)."""
        with torch.cuda.stream(stream):
            for _ in range(a.warmup):
                step(p)
        torch.cuda.synchronize(dev)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(a.steps)]
        stats = []
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        ctx = clk if clk is not None else contextlib.nullcontext()
        with ctx:
            with torch.cuda.stream(stream):
                for i in range(a.steps):
                    flush.fill_(i & 0x7F)
                    evs[i][0].record(stream)
                    stats.append(step(p))
                    evs[i][1].record(stream)
            torch.cuda.synchronize(dev)
        if ws > 1:
            dist.barrier()
        return [s.elapsed_time(e) for s, e in evs], stats, dist_t.cpu().numpy().view(np.uint32).copy()

    # plain arm first (its distances define reached vertices), then the headline arm
    plain_ms, plain_stats, d_plain = timed(plain)
    reached = d_plain < nps.INF
    n_r = int(reached.sum())
    m_r = int(np.diff(g.row_ptr)[reached].sum())
    b_alg = 12 * m_r + 12 * n_r + 4 * g.n
    if use_learned:
        clk = ClockSampler(local)
        step_ms, stats, dh = timed(learned, clk)
    else:
        clk = ClockSampler(local)
        step_ms, stats, dh = timed(plain, clk)
    clocks = clk.summary()
    kern_ms = sum(step_ms)
    exact_vs_plain = bool(np.array_equal(dh, d_plain))

    # ---- e2e through the host-buffer public call (pinned host memory)
    def pinned(x):
        t = torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).pin_memory()
        return t.numpy()
    hg = nps.Graph(pinned(g.row_ptr), pinned(g.col), pinned(g.w).view(np.uint32), g.source)
    hout = torch.empty(g.n, dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    e2e_steps = a.e2e_steps or a.steps
    for _ in range(2):
        nps.sssp(hg, g.source, params, out=hout)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    e2e_dev_ms = []
    for _ in range(e2e_steps):
        _, st2 = nps.sssp(hg, g.source, params, out=hout)  # synchronous: H2D + kernel + D2H
        e2e_dev_ms.append(st2.total_ms)
    e2e_wall = (time.perf_counter() - t0) / e2e_steps
    e2e_ok = bool((hout == dh).all())

    tot_t = torch.tensor([kern_ms, e2e_wall * 1e3, sum(plain_ms)], dtype=torch.float64, device=dev)
    if ws > 1:
        dist.all_reduce(tot_t, op=dist.ReduceOp.MAX)
    kern_ms_max, e2e_ms_max, plain_ms_max = float(tot_t[0]), float(tot_t[1]), float(tot_t[2])
    value = ws * a.steps * m_r / (kern_ms_max * 1e-3) / 1e9
    plain_value = ws * a.steps * m_r / (plain_ms_max * 1e-3) / 1e9
    e2e_value = ws * m_r / (e2e_ms_max * 1e-3) / 1e9

    peak, peak_src = load_peaks()
    per_launch_s = kern_ms / a.steps * 1e-3
    achieved = b_alg / per_launch_s / 1e9
    traffic = None
    tr_path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tr_path):
        with open(tr_path) as f:
            tr = json.load(f)
        traffic = tr.get(a.workload + ("_learned" if use_learned else ""))

    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        if oracle.have_reference():
            dref, tcpu = oracle.ref_sssp_cpu(g.row_ptr, g.col, g.w, g.source)
            kind_cpu = "reference"
            sample = "one full SSSP of the workload by the reference's SSSP_CPU (heap Dijkstra, " \
                     "apps/sssp/src/cpu/sssp.cpp, built from its sources), 1 thread, including its Heap() init"
        else:
            dref, tcpu = oracle.timed(oracle.sssp_heap, g.row_ptr, g.col, g.w, g.source)
            kind_cpu = "port"
            sample = "one full SSSP of the workload by the oracle's restated heap Dijkstra, 1 thread"
        cpu = {"value": m_r / tcpu / 1e9, "unit": "GTEPS", "cores": 1, "kind": kind_cpu, "sample": sample,
               "seconds": tcpu, "bit_exact_vs_gpu": bool((dref == dh).all() and (dref == d_plain).all())}

    if rank == 0:
        st = stats[-1]
        line = {
            "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": ws, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": kern_ms_max / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": a.workload, "description": desc, "n": g.n, "m": g.m, "m_reached": m_r,
                       "n_reached": n_r, "source": g.source,
                       "policy": "learned" if use_learned else "plain",
                       "params": dataclasses.asdict(params),
                       "parallelism": f"replicas x{ws}" if ws > 1 else "1 GPU",
                       "l2": "flushed between steps (256 MB write); CSR 12 B/edge also exceeds L2",
                       "iterations": st.iterations, "buckets": st.buckets,
                       "edges_scanned": st.edges_scanned, "grid_ctas": st.grid_ctas,
                       "step_ms_min": min(step_ms), "step_ms_max": max(step_ms),
                       "autotune_evaluations": len(tune_log)},
            "plain": {"value": plain_value, "unit": "GTEPS", "ms_per_step": plain_ms_max / a.steps,
                      "params": dataclasses.asdict(plain), "iterations": plain_stats[-1].iterations,
                      "edges_scanned": plain_stats[-1].edges_scanned,
                      "note": "plain autotuned kernel (fixed parameters, no policy), same graph, same timing"},
            "learned_over_plain": (value / plain_value) if use_learned else None,
            "bit_exact": {"learned_vs_plain": exact_vs_plain,
                          "vs_cpu_dijkstra": cpu["bit_exact_vs_gpu"] if cpu else None},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                         "b_alg_bytes": b_alg, "b_alg_formula": "12*m_r + 12*n_r + 4*n"},
            "e2e": {"value": e2e_value, "unit": "GTEPS",
                    "h2d_bytes_per_step": host_call_h2d_bytes(g.n, g.m, int(g.w.max()) if g.m else 0),
                    "d2h_bytes_per_step": 4 * g.n,
                    "ms_per_step": e2e_ms_max, "device_ms_per_step": statistics.mean(e2e_dev_ms),
                    "bit_exact_vs_device_run": e2e_ok, "call": "nps.sssp(host Graph, pinned)"},
            "gpu_launches": a.steps,
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
