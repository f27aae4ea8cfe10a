#!/usr/bin/env python3
"""Golden colors from the reference's own graph-coloring program.

Runs oracle/_ref/gpu-graph-color -- the reference's gpu-graph-color built from its
sources (apps/graph-color/src/gpu) by oracle/Makefile -- with `-s 0` on the three
golden reader files and on generated graphs written as DIMACS9, and records every
vertex's color (gclr_nopruning_gpu(): one gclr_bitmap_kernel launch per color,
graph_color_wrapper.cu:113-130, graph_color_kernel.cu:14-35; written out by the hook
of oracle/ref_gclr_hook.cpp).  It needs a GPU; the output is committed as
tests/golden/color_reference.json and checked against the oracle on CPU by
tests/test_color_cpu.py.

    python tests/golden/make_color_golden.py --out tests/golden/color_reference.json
"""
import argparse
import importlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
BIN = os.path.join(ROOT, "oracle", "_ref", "gpu-graph-color")

READERS = [("reader_dimacs9.gr", 0), ("reader_dimacs10.graph", 1), ("reader_slndc.txt", 2)]
# generated graphs: name -> (generator, arguments); written as DIMACS9 and read back by the reference
GENERATED = {
    "rmat12_ef8_s3": ("gen_rmat", dict(scale=12, edge_factor=8, seed=3)),
    "rmat14_ef16_s5": ("gen_rmat", dict(scale=14, edge_factor=16, seed=5)),
    "uniform3000_s2": ("gen_uniform", dict(n=3000, m=20000, wmax=10, seed=2)),
    "grid40x40_s1": ("gen_grid", dict(rows=40, cols=40, drop=0.1, wmax=10, seed=1)),
}


def run_reference(path, fmt):
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "colors.bin")
        subprocess.run([BIN, "-s", "0", "-f", str(fmt), "-i", path], capture_output=True, text=True, timeout=600,
                       check=True, env=dict(os.environ, NPS_REF_COLORS=out))
        return np.fromfile(out, dtype=np.int32)


def fnv1a(a):
    h = 1469598103934665603
    for x in np.asarray(a, dtype=np.uint32).tolist():
        h = ((h ^ x) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    sys.path.insert(0, ROOT)
    nps = importlib.import_module("nested-parallelism_b200")
    res = {"generator": "tests/golden/make_color_golden.py", "program": "gpu-graph-color -s 0", "graphs": {}}
    for name, fmt in READERS:
        c = run_reference(os.path.join(HERE, name), fmt)
        res["graphs"][name] = {"format": fmt, "n": int(c.size), "max_color": int(c.max()), "colors": c.tolist()}
    with tempfile.TemporaryDirectory() as td:
        for name, (gen, kw) in GENERATED.items():
            g = getattr(nps, gen)(**kw)
            path = os.path.join(td, name + ".gr")
            nps.writeDIMACS9(path, g)
            c = run_reference(path, 0)
            res["graphs"][name] = {"format": 0, "generator": gen, "args": kw, "n": int(c.size),
                                   "max_color": int(c.max()), "fnv1a": str(fnv1a(c))}
    with open(a.out, "w") as f:
        json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
