#!/usr/bin/env python3
"""Sector-granular byte model of one SSSP pass over an R-MAT graph.

    python nested-parallelism_b200/traffic_model.py --scale 22 --seed 1000

Counts, on the host, what one walk of every reached row moves at the 32-byte
sector granularity of DRAM and L2, against the bytes the algorithm needs
(B_alg = 12 m_r + 12 n_r + 4 n: column and weight per reached edge, the two row
offsets, a distance read and write per reached vertex, the distance
initialisation):

- column and weight arrays: the sectors of [row_ptr[v], row_ptr[v+1]) in each;
- row offsets: the one or two sectors holding row_ptr[v] and row_ptr[v+1].

Reached vertices come from a breadth-first search from the source (scipy), so no
GPU is needed.  The kernel's measured DRAM bytes per launch (ncu) are compared
with this model in the profiles; the difference is re-scans, the random
per-vertex arrays and their misses.
"""
import argparse
import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
nps = importlib.import_module("nested-parallelism_b200")


def reached_mask(row_ptr, col, src):
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import breadth_first_order
    n = row_ptr.size - 1
    a = csr_matrix((np.ones(col.size, np.int8), col, row_ptr), shape=(n, n))
    order = breadth_first_order(a, src, directed=True, return_predecessors=False)
    r = np.zeros(n, bool)
    r[order] = True
    return r


def model(row_ptr, col, src):
    """Dictionary of the byte counts described in the module docstring."""
    n = row_ptr.size - 1
    r = reached_mask(row_ptr, col, src)
    s = row_ptr[:-1].astype(np.int64)
    e = row_ptr[1:].astype(np.int64)
    deg = e - s
    nr = int(r.sum())
    mr = int(deg[r].sum())
    sect = np.where(deg > 0, ((e - 1) * 4) // 32 - (s * 4) // 32 + 1, 0)
    out = {
        "n": n, "m": int(col.size), "n_r": nr, "m_r": mr,
        "b_alg": 12 * mr + 12 * nr + 4 * n,
        "csr_useful": 8 * mr,
        "csr_sectors": int(2 * 32 * sect[r].sum()),
        "row_ptr_useful": 8 * nr,
        "row_ptr_sectors": int(32 * np.where((s * 4) // 32 == (e * 4) // 32, 1, 2)[r].sum()),
        "by_degree": [],
    }
    for lo, hi in [(1, 4), (4, 32), (32, 256), (256, 1 << 31)]:
        mm = r & (deg >= lo) & (deg < hi)
        out["by_degree"].append({"degree": [lo, hi], "rows": int(mm.sum()), "edges": int(deg[mm].sum()),
                                 "csr_sectors": int(2 * 32 * sect[mm].sum()), "csr_useful": int(8 * deg[mm].sum())})
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--seed", type=int, default=1000)
    a = ap.parse_args()
    g = nps.gen_rmat(a.scale, a.edge_factor, seed=a.seed)
    t = model(np.asarray(g.row_ptr), np.asarray(g.col), g.source)
    print(f"n={t['n']} m={t['m']} n_r={t['n_r']} m_r={t['m_r']} B_alg={t['b_alg'] / 1e6:.1f} MB")
    print(f"columns + weights: useful {t['csr_useful'] / 1e6:.1f} MB, at 32-byte sectors "
          f"{t['csr_sectors'] / 1e6:.1f} MB ({t['csr_sectors'] / t['csr_useful']:.3f}x)")
    print(f"row offsets: useful {t['row_ptr_useful'] / 1e6:.1f} MB, at sectors {t['row_ptr_sectors'] / 1e6:.1f} MB")
    for b in t["by_degree"]:
        lo, hi = b["degree"]
        print(f"  rows of degree [{lo}, {hi}): {b['rows']} rows, {b['edges']} edges, "
              f"{b['csr_sectors'] / 1e6:.1f} MB at sectors for {b['csr_useful'] / 1e6:.1f} MB useful")


if __name__ == "__main__":
    main()
