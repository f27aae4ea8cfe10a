#!/usr/bin/env python3
"""Generate tests/golden/ fixtures by running the reference's own code.

For each case the graph comes from this repository's seeded generators, and the
expected distances come from the reference's SSSP_CPU() (apps/sssp/src/cpu/
sssp.cpp:13-47 with common/heap.cpp), compiled from its unmodified sources into
oracle/_ref/libref_sssp.so by oracle/Makefile.  The degree-statistics goldens
come from the reference's graph analyzer (utility/graph-analyzer/analyzer.cpp),
built into oracle/_ref/analyzer, run on the reader fixtures and on generated
graphs written as DIMACS9.  The BFS goldens come from the reference's bfs_cpu
(apps/bfs-rec/src/gpu/bfs_rec.cpp:100-119), built into oracle/_ref/libref_bfs.so,
on the same generated graphs and edge cases, and the SpMV goldens from the
reference's SpMV_CPU path (prepare_cpu + spmv_omp, apps/SpMV/src/cpu/
SpMV_kernel.cpp), built into oracle/_ref/libref_spmv.so, and the betweenness
centrality goldens from the reference's bc_cpu (apps/bc/src/cpu/bc.cpp), built
into oracle/_ref/libref_bc.so, on small graphs (it keeps an n x n matrix).  The
reader fixtures are small
synthetic DIMACS9 / DIMACS10 / SNAP files written here; their expected CSR comes
from the reference's readInputDIMACS9/10/SLNDC() + convertCSR() (common/
global.cpp:29-235) on the same files.

Run from the repository root in a tree where oracle/_ref exists:
    python tests/golden/make_golden.py
Writes golden.json, golden_dist.npz and the reader fixture files.
"""
import importlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402

nps = importlib.import_module("nested-parallelism_b200")

# (name, generator, args, source or None for the generator's pick)
CASES = [
    ("uniform16k_s1", "uniform", dict(n=16384, m=131072, wmax=100, seed=1), 0),
    ("uniform16k_s2", "uniform", dict(n=16384, m=131072, wmax=100, seed=2), 0),
    ("uniform16k_s3_src77", "uniform", dict(n=16384, m=131072, wmax=100, seed=3), 77),
    ("rmat14_ef16_s1", "rmat", dict(scale=14, edge_factor=16, seed=1), None),
    ("rmat12_ef8_s9", "rmat", dict(scale=12, edge_factor=8, seed=9), None),
    ("rmat13_ef32_s4_src5", "rmat", dict(scale=13, edge_factor=32, seed=4), 5),
    ("rmat16_ef4_s7", "rmat", dict(scale=16, edge_factor=4, seed=7), None),
    ("grid64_s1", "grid", dict(rows=64, cols=64, drop=0.05, wmax=1000, seed=1), None),
    ("grid128x32_s2", "grid", dict(rows=128, cols=32, drop=0.05, wmax=1000, seed=2), None),
    ("grid256_nodrop_s3", "grid", dict(rows=256, cols=256, drop=0.0, wmax=1000, seed=3), None),
]

# tiny hand-made edge cases: (name, n, src, dst, w, source)
EDGE_CASES = [
    ("single_vertex", 1, [], [], [], 0),
    ("isolated_source", 5, [1, 2], [2, 3], [4, 5], 0),
    ("chain_to_inf", 4, [0, 1, 0], [1, 2, 3], [1 << 29, 1 << 29, 7], 0),
    ("zero_weights", 6, [0, 1, 2, 3, 4, 0], [1, 2, 3, 4, 5, 5], [0, 0, 0, 0, 0, 9], 0),
    ("multi_edges_self_loops", 5, [0, 0, 0, 1, 1, 2, 3], [1, 1, 0, 1, 2, 3, 4], [5, 3, 1, 2, 2, 2, 2], 0),
    ("star_hub", 2001, [0] * 2000, list(range(1, 2001)), [(i * 37) % 97 + 1 for i in range(2000)], 0),
]


def gen(kind, a):
    if kind == "uniform":
        return nps.gen_uniform(a["n"], a["m"], a["wmax"], a["seed"])
    if kind == "rmat":
        return nps.gen_rmat(a["scale"], a["edge_factor"], seed=a["seed"])
    return nps.gen_grid(a["rows"], a["cols"], a["drop"], a["wmax"], a["seed"])


def csr_hash(g):
    return {"row": nps.fnv1a(g.row_ptr.view(np.uint32)), "col": nps.fnv1a(g.col.view(np.uint32)),
            "w": nps.fnv1a(g.w)}


def write_reader_fixtures():
    """Small synthetic input files in the three formats the reference reads."""
    rng = np.random.default_rng(2024)
    # DIMACS9: a random graph written by this library's writer, with an 's' line
    g = nps.gen_rmat(9, 8, seed=11)
    nps.writeDIMACS9(os.path.join(HERE, "reader_dimacs9.gr"), g, source=3)
    # DIMACS10 (METIS-like adjacency, undirected: each edge listed from both ends)
    n10 = 300
    adj = [set() for _ in range(n10)]
    for _ in range(900):
        u, v = rng.integers(0, n10, 2)
        if u != v:
            adj[u].add(int(v))
            adj[v].add(int(u))
    m_und = sum(len(a) for a in adj) // 2
    with open(os.path.join(HERE, "reader_dimacs10.graph"), "w") as f:
        f.write("% synthetic DIMACS10 fixture\n")
        f.write(f"{n10} {m_und}\n")
        for a in adj:
            f.write(" ".join(str(x + 1) for x in sorted(a)) + "\n")
    # SNAP edge list (SLNDC): sparse ids, two comment lines, a Nodes/Edges line, one more comment
    ids = rng.choice(np.arange(5, 300), size=150, replace=False)  # the reference requires ids < 2 * Nodes
    with open(os.path.join(HERE, "reader_slndc.txt"), "w") as f:
        f.write("# Directed graph (each unordered pair of nodes is saved once)\n")
        f.write("# synthetic SNAP fixture\n")
        f.write(f"# Nodes: {len(ids)} Edges: 600\n")
        f.write("# FromNodeId\tToNodeId\n")
        for _ in range(600):
            a, b = rng.choice(ids, 2)
            f.write(f"{a}\t{b}\n")


# graphs for the degree analyzer: the reader fixtures, and generated graphs written
# as DIMACS9 for the reference's analyzer to read
ANALYZER_GRAPHS = [("rmat12_ef8_s9", "rmat", dict(scale=12, edge_factor=8, seed=9)),
                   ("uniform16k_s1", "uniform", dict(n=16384, m=131072, wmax=100, seed=1)),
                   ("grid64_s1", "grid", dict(rows=64, cols=64, drop=0.05, wmax=1000, seed=1))]


def analyzer_goldens():
    """The reference's graph analyzer (utility/graph-analyzer/analyzer.cpp, built by
    oracle/Makefile into oracle/_ref/analyzer) run with -d on each file: its printed
    statistics and degree distribution."""
    import tempfile
    if not oracle.have_analyzer():
        sys.exit("oracle/_ref/analyzer missing: build it with `make -C oracle NPS_REFERENCE=<reference checkout>`")
    res = {}
    for fname, fmt in (("reader_dimacs9.gr", 0), ("reader_dimacs10.graph", 1), ("reader_slndc.txt", 2)):
        r = oracle.ref_analyzer(os.path.join(HERE, fname), fmt)
        r["dist"] = sorted([int(k), int(v)] for k, v in r["dist"].items())
        res[fname] = dict(r, file=fname, format=fmt)
    with tempfile.TemporaryDirectory() as td:
        for name, kind, args in ANALYZER_GRAPHS:
            g = gen(kind, args)
            path = os.path.join(td, name + ".gr")
            nps.writeDIMACS9(path, g)
            r = oracle.ref_analyzer(path, 0)
            r["dist"] = sorted([int(k), int(v)] for k, v in r["dist"].items())
            res[name] = dict(r, kind=kind, args=args)
    return res


def bfs_goldens():
    """Levels from the reference's bfs_cpu on every case graph (FNV-1a of the int32
    levels viewed as uint32) and on the edge cases (the levels themselves)."""
    if not oracle.have_reference_bfs():
        sys.exit("oracle/_ref/libref_bfs.so missing: build it with `make -C oracle NPS_REFERENCE=<reference checkout>`")
    res = {"cases": {}, "edge_cases": {}}
    for name, kind, args, src in CASES:
        g = gen(kind, args)
        s = g.source if src is None else src
        lv, _ = oracle.ref_bfs_cpu(g.row_ptr, g.col, s)
        fin = lv[lv != oracle.BFS_UNDEFINED]
        res["cases"][name] = {"source": int(s), "levels_fnv1a": oracle.fnv1a(lv.view(np.uint32)),
                              "n_reached": int(fin.size), "max_level": int(fin.max())}
    for name, n, s, t, w, src in EDGE_CASES:
        g = nps.convertCSR(n, s, t, w)
        lv, _ = oracle.ref_bfs_cpu(g.row_ptr, g.col, src)
        res["edge_cases"][name] = [int(x) for x in lv]
    return res


def spmv_goldens():
    """y from the reference's spmv_omp on its own data for every case graph (FNV-1a
    of the float64 bits) and on the edge cases (the values themselves)."""
    if not oracle.have_reference_spmv():
        sys.exit("oracle/_ref/libref_spmv.so missing: build it with `make -C oracle NPS_REFERENCE=<reference checkout>`")
    res = {"cases": {}, "edge_cases": {}}
    for name, kind, args, _ in CASES:
        g = gen(kind, args)
        y, _, _, _ = oracle.ref_spmv_cpu(g.row_ptr, g.col, 1)
        res["cases"][name] = {"y_fnv1a": oracle.fnv1a(y.view(np.uint32)), "y_sum": float(y.sum()),
                              "y_max": float(y.max())}
    for name, n, s, t, w, _ in EDGE_CASES:
        g = nps.convertCSR(n, s, t, w)
        y, _, _, _ = oracle.ref_spmv_cpu(g.row_ptr, g.col, 1)
        res["edge_cases"][name] = [float(v) for v in y]
    return res


# graphs small enough for the reference's bc_cpu, which clears an n x n byte matrix per source
BC_GRAPHS = [("rmat10_ef8_s3", "rmat", dict(scale=10, edge_factor=8, seed=3)),
             ("rmat11_ef16_s7", "rmat", dict(scale=11, edge_factor=16, seed=7)),
             ("grid30_s1", "grid", dict(rows=30, cols=30, drop=0.1, wmax=10, seed=1)),
             ("uniform1500_s2", "uniform", dict(n=1500, m=6000, wmax=10, seed=2))]


def bc_goldens():
    """Centralities from the reference's bc_cpu (every vertex a source, one thread):
    FNV-1a of the float32 bits per graph, and the values for the edge cases."""
    if not oracle.have_reference_bc():
        sys.exit("oracle/_ref/libref_bc.so missing: build it with `make -C oracle NPS_REFERENCE=<reference checkout>`")
    res = {"cases": {}, "edge_cases": {}}
    for name, kind, args in BC_GRAPHS:
        g = gen(kind, args)
        b, _ = oracle.ref_bc_cpu(g.row_ptr, g.col)
        res["cases"][name] = {"kind": kind, "args": args, "bc_fnv1a": oracle.fnv1a(b.view(np.uint32)),
                              "bc_max": float(b.max()), "bc_sum": float(b.astype(np.float64).sum())}
    for name, n, s, t, w, _ in EDGE_CASES:
        g = nps.convertCSR(n, s, t, w)
        b, _ = oracle.ref_bc_cpu(g.row_ptr, g.col)
        res["edge_cases"][name] = [float(v) for v in b]
    return res


def main():
    if not oracle.have_reference():
        sys.exit("oracle/_ref/libref_sssp.so missing: build it with `make -C oracle NPS_REFERENCE=<reference checkout>`")
    out = {"generator": "nested-parallelism_b200 seeded generators (splitmix64 counter streams)",
           "expected_by": "reference SSSP_CPU (apps/sssp/src/cpu/sssp.cpp) built from its sources",
           "cases": {}, "edge_cases": {}, "readers": {}}
    dists = {}
    for name, kind, args, src in CASES:
        g = gen(kind, args)
        s = g.source if src is None else src
        d, _ = oracle.ref_sssp_cpu(g.row_ptr, g.col, g.w, s)
        n_r, m_r = oracle.reached(g.row_ptr, d)
        out["cases"][name] = {"kind": kind, "args": args, "source": int(s), "n": g.n, "m": g.m,
                              "csr_fnv1a": csr_hash(g), "dist_fnv1a": oracle.fnv1a(d), "n_reached": n_r,
                              "m_reached": m_r, "max_dist": int(d[d < oracle.INF].max())}
        if g.n <= 16384:
            dists[name] = d
        print(name, g.n, g.m, hex(oracle.fnv1a(d)))
    for name, n, s, t, w, src in EDGE_CASES:
        g = nps.convertCSR(n, s, t, w)
        d, _ = oracle.ref_sssp_cpu(g.row_ptr, g.col, g.w, src)
        out["edge_cases"][name] = {"n": n, "src": s, "dst": t, "w": w, "source": src,
                                   "dist": [int(x) for x in d]}
    write_reader_fixtures()
    for fname, fmt in (("reader_dimacs9.gr", 0), ("reader_dimacs10.graph", 1), ("reader_slndc.txt", 2)):
        row, col, w, src = oracle.ref_read_graph(os.path.join(HERE, fname), fmt)
        out["readers"][fname] = {"format": fmt, "n": int(row.shape[0] - 1), "m": int(col.shape[0]), "source": src,
                                 "row_fnv1a": nps.fnv1a(row.view(np.uint32)),
                                 "col_fnv1a": nps.fnv1a(col.view(np.uint32)), "w_fnv1a": nps.fnv1a(w)}
    out["analyzer"] = analyzer_goldens()
    out["bfs"] = bfs_goldens()
    out["spmv"] = spmv_goldens()
    out["bc"] = bc_goldens()
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    np.savez_compressed(os.path.join(HERE, "golden_dist.npz"), **dists)


if __name__ == "__main__":
    main()
