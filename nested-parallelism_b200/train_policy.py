#!/usr/bin/env python3
"""Train the SSSP policy MLP by imitating the best bucket schedules of the plain
kernel, and evaluate it against the plain autotuned kernel.

    python nested-parallelism_b200/train_policy.py --out nested-parallelism_b200/policy_weights.npz

1. Autotunes the plain kernel (fixed parameters) on R-MAT scale-20 graphs.
2. For R-MAT scales 16-20, seeds 0..S-1: a teacher search times the plain
   kernel under candidate per-bucket width schedules and levels (all seeds of
   the first --search-seeds get the full candidate set, later seeds the
   --topk schedules that won most often so far), runs the fastest traced, and
   labels its trace (policy.label_trace).
3. Trains the 12-32-14 MLP on the GPU with the library's bf16 kernels.
4. Evaluates learned vs plain on held-out R-MAT scale-22 graphs (seeds
   1000..), checking that both give the CPU Dijkstra oracle's distances.
"""
import argparse
import collections
import dataclasses
import importlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
nps = importlib.import_module("nested-parallelism_b200")
pol = importlib.import_module("nested-parallelism_b200.policy")
at = importlib.import_module("nested-parallelism_b200.autotune")


def median_ms(dg, p, reps=5):
    ts = []
    for _ in range(reps + 1):
        ts.append(nps.sssp_device(dg.row_ptr, dg.col, dg.w, dg.n, dg.m, dg.src, dg.dist, p).kernel_ms)
    return float(np.median(ts[1:]))


def learned_params(plain):
    """The learned configuration: the plain one with the policy deciding widths and
    levels (no light/heavy split and no degree ordering, as in the teacher runs), on
    graphs of every size (the library's minimum graph size for the policy is off)."""
    return dataclasses.replace(plain, policy=nps.POLICY_LEARNED, light_heavy=False, order_degree=0,
                               delta_schedule=0, policy_min_edges=-1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scales", type=int, nargs="+", default=[16, 17, 18, 19, 20])
    ap.add_argument("--seeds", type=int, default=100)
    ap.add_argument("--search-seeds", type=int, default=12)
    ap.add_argument("--topk", type=int, default=10)
    ap.add_argument("--eval-scale", type=int, default=22)
    ap.add_argument("--eval-seeds", type=int, default=10)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--tune-budget", type=int, default=40)
    ap.add_argument("--no-oracle", action="store_true", help="skip the CPU Dijkstra check of the evaluation")
    ap.add_argument("--out", default=os.path.join(HERE, "policy_weights.npz"))
    ap.add_argument("--report", default=None)
    a = ap.parse_args()
    import torch
    dev = torch.device("cuda", 0)
    t0 = time.time()
    report = {"scales": a.scales, "seeds": a.seeds, "search_seeds": a.search_seeds, "topk": a.topk}

    # 1. plain autotuned configuration (fixed parameters) on scale-20 training graphs
    tune_graphs = [at.to_device(nps.gen_rmat(max(a.scales), 16, seed=s)) for s in range(2)]
    plain, plain_ms, _ = at.autotune(tune_graphs, budget=a.tune_budget,
                                     seed=nps.Params(level=2, threshold=64, delta=0, block_size=512))
    report["plain"] = dataclasses.asdict(plain)
    report["plain_tune_ms"] = plain_ms
    print("plain", dataclasses.asdict(plain), f"{plain_ms:.3f} ms", flush=True)
    del tune_graphs

    # 2. teacher search, traces and labels
    base = dataclasses.replace(plain, light_heavy=False, order_degree=0)
    full = pol.candidate_schedules()
    wins = collections.Counter()
    Xs, yds, yls, wts, rows = [], [], [], [], []
    for scale in a.scales:
        for seed in range(a.seeds):
            g = nps.gen_rmat(scale, 16, seed=seed)
            dg = at.to_device(g)
            cands = full if seed < a.search_seeds or not wins else [s for s, _ in wins.most_common(a.topk)]
            best_ms, (lead, rest), level, times = pol.teacher_search(dg, base, cands)
            if seed < a.search_seeds:
                for s in sorted(times, key=times.get)[:3]:
                    wins[s] += 1
            p_ms = pol._time(dg, plain)
            recs = pol.trace_schedule(dg, base, lead, rest, level)
            X, yd, yl, wt = pol.label_trace(recs, g.n, lead, level,
                                            source_degree=int(g.row_ptr[g.source + 1] - g.row_ptr[g.source]))
            Xs.append(X); yds.append(yd); yls.append(yl); wts.append(wt)
            rows.append({"scale": scale, "seed": seed, "plain_ms": p_ms, "teacher_ms": best_ms,
                         "lead": list(lead), "rest": rest, "level": level, "records": int(len(X))})
            del dg
        sub = [r for r in rows if r["scale"] == scale]
        gain = float(np.exp(np.mean([np.log(r["plain_ms"] / r["teacher_ms"]) for r in sub])))
        print(f"scale {scale}: {len(sub)} graphs, teacher / plain speedup {gain:.3f} "
              f"({time.time() - t0:.0f} s)", flush=True)
    report["teacher"] = rows
    report["schedule_wins"] = {f"{list(k[0])}+{k[1]}": v for k, v in wins.most_common(20)}
    X, yd, yl, wt = (np.concatenate(v) for v in (Xs, yds, yls, wts))
    report["records"] = int(X.shape[0])
    report["delta_decisions"] = int((yd >= 0).sum())

    # 3. train on the GPU with the library's kernels
    w, losses = pol.train(X, yd, yl, wt, dev, steps=a.steps, log_every=100)
    report["losses"] = losses
    w.save(a.out)
    print(f"trained on {X.shape[0]} records ({report['delta_decisions']} width decisions), "
          f"loss {losses[0]:.3f} -> {losses[-1]:.3f}", flush=True)

    # 4. held-out evaluation against the plain autotuned kernel and the CPU oracle
    pol.load_into_kernel(w, 0)
    learned = learned_params(plain)
    oracle = None
    if not a.no_oracle:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
    ev = []
    for seed in range(1000, 1000 + a.eval_seeds):
        g = nps.gen_rmat(a.eval_scale, 16, seed=seed)
        dg = at.to_device(g)
        mp = median_ms(dg, plain)
        dp = dg.dist.cpu().numpy().view(np.uint32).copy()
        ml = median_ms(dg, learned)
        st = nps.sssp_device(dg.row_ptr, dg.col, dg.w, dg.n, dg.m, dg.src, dg.dist, learned)
        dl = dg.dist.cpu().numpy().view(np.uint32).copy()
        reached = dp < nps.INF
        m_r = int(np.diff(g.row_ptr)[reached].sum())
        row = {"seed": seed, "m_r": m_r, "plain_ms": mp, "learned_ms": ml, "plain_gteps": m_r / mp / 1e6,
               "learned_gteps": m_r / ml / 1e6, "learned_iterations": st.iterations,
               "learned_buckets": st.buckets, "learned_edges": st.edges_scanned,
               "identical": bool(np.array_equal(dp, dl))}
        if oracle is not None:
            ref = oracle.sssp_heap(g.row_ptr, g.col, g.w, g.source)
            row["oracle_exact"] = bool(np.array_equal(ref, dp) and np.array_equal(ref, dl))
        ev.append(row)
        print(json.dumps(row), flush=True)
        del dg
    report["eval"] = ev
    report["speedup_geomean"] = float(np.exp(np.mean([np.log(r["plain_ms"] / r["learned_ms"]) for r in ev])))
    report["wall_s"] = time.time() - t0
    print("speedup (geomean) learned / plain:", report["speedup_geomean"], flush=True)
    if a.report:
        with open(a.report, "w") as f:
            json.dump(summary(report), f, indent=1)


def summary(report):
    """The committed record of a training run (policy_training.json): the plain
    configuration, per-scale teacher gains, the winning schedules and the held-out
    evaluation, from the full report `main` builds."""
    by_scale = collections.defaultdict(list)
    for r in report["teacher"]:
        by_scale[r["scale"]].append(np.log(r["plain_ms"] / r["teacher_ms"]))
    rnd = lambda r: {k: (round(v, 4) if isinstance(v, float) else v) for k, v in r.items()}
    return {
        "what": "training and held-out evaluation of policy_weights.npz (nested-parallelism_b200/train_policy.py, "
                "default arguments, one B200)",
        "command": "python nested-parallelism_b200/train_policy.py --out nested-parallelism_b200/policy_weights.npz "
                   "--report <file>",
        "training_graphs": {"scales": report["scales"], "seeds_per_scale": report["seeds"],
                            "full_search_seeds": report["search_seeds"], "topk": report["topk"]},
        "plain_autotuned_on_scale20": report["plain"],
        "records": report["records"],
        "width_decisions": report["delta_decisions"],
        "loss_first_last": [report["losses"][0], report["losses"][-1]],
        "teacher_speedup_over_plain_by_scale": {str(k): float(np.exp(np.mean(v))) for k, v in sorted(by_scale.items())},
        "schedule_wins_top10": dict(list(report["schedule_wins"].items())[:10]),
        "eval_rmat22_seeds_1000_1009": [rnd(r) for r in report["eval"]],
        "speedup_geomean_learned_over_plain": report["speedup_geomean"],
        "wall_s": report["wall_s"],
    }


if __name__ == "__main__":
    main()
