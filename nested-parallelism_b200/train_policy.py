#!/usr/bin/env python3
"""Train the SSSP policy MLP on traces of plain autotuned runs and evaluate it.

    python nested-parallelism_b200/train_policy.py --out nested-parallelism_b200/policy_weights.npz

1. Autotunes the plain kernel on R-MAT scale-20 training graphs.
2. Collects traces on R-MAT scales 16-20 (seeds 0..S-1) for every fixed
   (delta, level) configuration around the plain one.
3. Labels every trace record with the configuration that is cheapest in its
   progress bin and trains the 12-32-14 MLP with the bf16 training kernels.
4. Evaluates learned vs plain on held-out R-MAT scale-22 graphs (seeds
   1000..), checking that distances are identical.
"""
import argparse
import dataclasses
import importlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
nps = importlib.import_module("nested-parallelism_b200")
pol = importlib.import_module("nested-parallelism_b200.policy")
at = importlib.import_module("nested-parallelism_b200.autotune")


def median_ms(dg, p, reps=5):
    ts = []
    for _ in range(reps + 1):
        ts.append(nps.sssp_device(dg.row_ptr, dg.col, dg.w, dg.n, dg.m, dg.src, dg.dist, p).kernel_ms)
    return float(np.median(ts[1:]))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scales", type=int, nargs="+", default=[16, 17, 18, 19, 20])
    ap.add_argument("--seeds", type=int, default=12)
    ap.add_argument("--eval-scale", type=int, default=22)
    ap.add_argument("--eval-seeds", type=int, default=10)
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--tune-budget", type=int, default=40)
    ap.add_argument("--out", default=os.path.join(HERE, "policy_weights.npz"))
    ap.add_argument("--report", default=None)
    a = ap.parse_args()
    import torch
    dev = torch.device("cuda", 0)
    t0 = time.time()
    report = {"scales": a.scales, "seeds": a.seeds}

    # 1. plain autotuned configuration on scale-20 training graphs
    tune_graphs = [at.to_device(nps.gen_rmat(max(a.scales), 16, seed=s)) for s in range(2)]
    plain, plain_ms, log = at.autotune(tune_graphs, budget=a.tune_budget,
                                       seed=nps.Params(level=2, threshold=64, delta=0, block_size=512))
    report["plain"] = dataclasses.asdict(plain)
    report["plain_tune_ms"] = plain_ms
    print("plain", dataclasses.asdict(plain), f"{plain_ms:.3f} ms", flush=True)
    del tune_graphs

    # 2-3. traces and labels
    base = dataclasses.replace(plain, light_heavy=False, local_rounds=0, level=2)
    Xs, yds, yls, wts = [], [], [], []
    for scale in a.scales:
        for seed in range(a.seeds):
            g = nps.gen_rmat(scale, 16, seed=seed)
            dg = at.to_device(g)
            runs = {}
            for di, d in enumerate(pol.DELTA_CHOICES):
                for li, lv in enumerate(pol.LEVEL_CHOICES):
                    runs[(di, li)] = pol.trace_run(dg, pol.config_params(base, d, lv))
            X, yd, yl, wt = pol.label_graph(runs)
            Xs.append(X); yds.append(yd); yls.append(yl); wts.append(wt)
            tot = {f"d{pol.DELTA_CHOICES[k[0]]}_l{k[1]}": v[0] for k, v in runs.items()}
            report.setdefault("run_ms", []).append({"scale": scale, "seed": seed, "ms": tot})
            del dg
        print(f"scale {scale} traced ({time.time() - t0:.0f} s)", flush=True)
    X, yd, yl, wt = (np.concatenate(v) for v in (Xs, yds, yls, wts))
    report["records"] = int(X.shape[0])
    w, losses = pol.train(X, yd, yl, wt, dev, steps=a.steps, log_every=100)
    report["losses"] = losses
    w.save(a.out)
    print(f"trained on {X.shape[0]} records, loss {losses[0]:.3f} -> {losses[-1]:.3f}", flush=True)

    # 4. held-out evaluation
    pol.load_into_kernel(w, 0)
    learned = dataclasses.replace(plain, policy=nps.POLICY_LEARNED)
    rows = []
    for seed in range(1000, 1000 + a.eval_seeds):
        g = nps.gen_rmat(a.eval_scale, 16, seed=seed)
        dg = at.to_device(g)
        mp = median_ms(dg, plain)
        dp = dg.dist.cpu().numpy().copy()
        ml = median_ms(dg, learned)
        dl = dg.dist.cpu().numpy().copy()
        reached = dp.view(np.uint32) < nps.INF
        m_r = int(np.diff(g.row_ptr)[reached].sum())
        rows.append({"seed": seed, "m_r": m_r, "plain_ms": mp, "learned_ms": ml, "plain_gteps": m_r / mp / 1e6,
                     "learned_gteps": m_r / ml / 1e6, "identical": bool(np.array_equal(dp, dl))})
        print(json.dumps(rows[-1]), flush=True)
        del dg
    report["eval"] = rows
    report["speedup_geomean"] = float(np.exp(np.mean([np.log(r["plain_ms"] / r["learned_ms"]) for r in rows])))
    print("speedup (geomean) learned / plain:", report["speedup_geomean"], flush=True)
    if a.report:
        with open(a.report, "w") as f:
            json.dump(report, f, indent=1)


if __name__ == "__main__":
    main()
