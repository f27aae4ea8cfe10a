"""Python loader of the SSSP oracle -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and the cpu_baseline / reference
legs of bench.py, always as the checker or the timed CPU baseline.  The library
in nested-parallelism_b200/ never imports it.

  liboracle.so          C restatement (sssp_oracle.c): heap Dijkstra, d-heap
                        Dijkstra, state fixpoint
  _ref/libref_sssp.so   the reference's own SSSP_CPU / usssp_cpu / dheap built
                        from its sources by oracle/Makefile (absent if the
                        reference tree was not available when it was built)
  _ref/libref_bfs.so    the reference's own CPU BFS (bfs-rec's bfs_cpu), likewise
  _ref/libref_spmv.so   the reference's own CPU SpMV (spmv_omp with its data), likewise
  _ref/libref_bc.so     the reference's own CPU betweenness centrality (bc_cpu), likewise
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref_sssp.so")
REF_BFS_SO = os.path.join(HERE, "_ref", "libref_bfs.so")
REF_SPMV_SO = os.path.join(HERE, "_ref", "libref_spmv.so")
REF_BC_SO = os.path.join(HERE, "_ref", "libref_bc.so")
INF = 0x40000000
BFS_UNDEFINED = 0x7FFFFFFF  # apps/bfs-rec/src/gpu/bfs_rec.h:13

_P, _I32, _I64, _D = C.c_void_p, C.c_int32, C.c_int64, C.c_double

_orc = None
_ref = None


def _load_oracle():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_SO):
            raise ImportError(f"{ORACLE_SO} missing: run `make -C {HERE}`")
        lib = C.CDLL(ORACLE_SO)
        lib.oracle_sssp_heap.argtypes = [_I32, _P, _P, _P, _I32, _P]
        lib.oracle_sssp_heap.restype = C.c_int
        lib.oracle_sssp_dheap.argtypes = [_I32, _P, _P, _P, _I32, C.c_int, _P]
        lib.oracle_sssp_dheap.restype = C.c_int
        lib.oracle_sssp_state.argtypes = [_I32, _P, _P, _P, _P, _P]
        lib.oracle_sssp_state.restype = C.c_int
        lib.oracle_reached.argtypes = [_I32, _P, _P, C.POINTER(_I64), C.POINTER(_I64)]
        lib.oracle_reached.restype = None
        lib.oracle_fnv1a_u32.argtypes = [_P, _I64]
        lib.oracle_fnv1a_u32.restype = C.c_uint64
        lib.oracle_bc.argtypes = [_I32, _P, _P, _I32, _P, _P]
        lib.oracle_bc.restype = C.c_int
        lib.oracle_color.argtypes = [_I32, _P, _P, _P]
        lib.oracle_color.restype = _I32
        lib.oracle_color_iterations.argtypes = [_I32, _P, _P, _P]
        lib.oracle_color_iterations.restype = _I32
        lib.oracle_gen_rmat.argtypes = [_I32, _I32, _D, _D, _D, C.c_uint32, C.c_uint64, _P, _P, _P,
                                        C.POINTER(_I32)]
        lib.oracle_gen_rmat.restype = _I64
        _orc = lib
    return _orc


def gen_rmat(scale: int, edge_factor: int = 16, seed: int = 1, a: float = 0.57, b: float = 0.19,
             c: float = 0.19, wmax: int = 255):
    """The benchmark's seeded R-MAT graph (deduplicated, no self-loops, rows in reverse
    edge order), identical to the library's gen_rmat.  Returns (row_ptr int32[n+1],
    col int32[m], w uint32[m], source)."""
    lib = _load_oracle()
    n, m = 1 << scale, edge_factor << scale
    row = np.empty(n + 1, dtype=np.int32)
    col = np.empty(m, dtype=np.int32)
    w = np.empty(m, dtype=np.uint32)
    src = _I32(0)
    k = lib.oracle_gen_rmat(scale, edge_factor, a, b, c, wmax, seed, row.ctypes.data, col.ctypes.data,
                            w.ctypes.data, C.byref(src))
    if k < 0:
        raise ValueError("gen_rmat: bad parameters")
    return row, col[:k].copy(), w[:k].copy(), int(src.value)


def have_reference() -> bool:
    return os.path.exists(REF_SO)


def _load_ref():
    global _ref
    if _ref is None:
        if not have_reference():
            raise ImportError(f"{REF_SO} missing: the reference CPU code was not built")
        lib = C.CDLL(REF_SO)
        lib.nps_ref_sssp_cpu.argtypes = [_I32, _I32, _P, _P, _P, _I32, _P]
        lib.nps_ref_sssp_cpu.restype = _D
        lib.nps_ref_heap_init_seconds.argtypes = []
        lib.nps_ref_heap_init_seconds.restype = _D
        lib.nps_ref_usssp_cpu.argtypes = [_I32, _I32, _P, _P, _P, _I32, _I32, _P]
        lib.nps_ref_usssp_cpu.restype = _D
        lib.nps_ref_dijkstra_dheap.argtypes = [_I32, _P, _P, _P, _I32, _I32, _P]
        lib.nps_ref_dijkstra_dheap.restype = _D
        _ref = lib
    return _ref


def _arrs(row, col, w):
    return (np.ascontiguousarray(row, dtype=np.int32), np.ascontiguousarray(col, dtype=np.int32),
            np.ascontiguousarray(w, dtype=np.uint32))


def sssp_heap(row, col, w, src):
    """Restated SSSP_CPU (lazy binary-heap Dijkstra)."""
    row, col, w = _arrs(row, col, w)
    n = row.shape[0] - 1
    d = np.empty(n, dtype=np.uint32)
    rc = _load_oracle().oracle_sssp_heap(n, row.ctypes.data, col.ctypes.data, w.ctypes.data, int(src),
                                         d.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"oracle_sssp_heap failed ({rc})")
    return d


def sssp_dheap(row, col, w, src, d=4):
    """Restated d-ary-heap Dijkstra with decrease-key (dheap API)."""
    row, col, w = _arrs(row, col, w)
    n = row.shape[0] - 1
    out = np.empty(n, dtype=np.uint32)
    rc = _load_oracle().oracle_sssp_dheap(n, row.ctypes.data, col.ctypes.data, w.ctypes.data, int(src), int(d),
                                          out.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"oracle_sssp_dheap failed ({rc})")
    return out


def sssp_state(row, col, w, cost, update):
    """Label-correcting fixpoint from a cost / update state (returns new arrays)."""
    row, col, w = _arrs(row, col, w)
    n = row.shape[0] - 1
    c = np.array(cost, dtype=np.uint32, copy=True)
    u = np.array(update, dtype=np.uint8, copy=True)
    rc = _load_oracle().oracle_sssp_state(n, row.ctypes.data, col.ctypes.data, w.ctypes.data, c.ctypes.data,
                                          u.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"oracle_sssp_state failed ({rc})")
    return c, u


def reached(row, dist):
    row = np.ascontiguousarray(row, dtype=np.int32)
    dist = np.ascontiguousarray(dist, dtype=np.uint32)
    a, b = _I64(0), _I64(0)
    _load_oracle().oracle_reached(row.shape[0] - 1, row.ctypes.data, dist.ctypes.data, C.byref(a), C.byref(b))
    return int(a.value), int(b.value)


def fnv1a(dist) -> int:
    a = np.ascontiguousarray(dist, dtype=np.uint32)
    return int(_load_oracle().oracle_fnv1a_u32(a.ctypes.data, a.shape[0]))


# ---- the reference's own code --------------------------------------------

def ref_sssp_cpu(row, col, w, src):
    """The reference's SSSP_CPU() on these arrays; returns (dist uint32, seconds)."""
    row, col, w = _arrs(row, col, w)
    n, m = row.shape[0] - 1, col.shape[0]
    cost = np.empty(n, dtype=np.int32)
    t = _load_ref().nps_ref_sssp_cpu(n, m, row.ctypes.data, col.ctypes.data, w.ctypes.data, int(src),
                                     cost.ctypes.data)
    return cost.view(np.uint32), float(t)


def ref_heap_init_seconds() -> float:
    return float(_load_ref().nps_ref_heap_init_seconds())


def ref_usssp_cpu(row, col, w, src, threads=0):
    """The reference's OpenMP frontier sweep (racy, not exact with >1 thread)."""
    row, col, w = _arrs(row, col, w)
    n, m = row.shape[0] - 1, col.shape[0]
    cost = np.empty(n, dtype=np.int32)
    t = _load_ref().nps_ref_usssp_cpu(n, m, row.ctypes.data, col.ctypes.data, w.ctypes.data, int(src),
                                      int(threads), cost.ctypes.data)
    return cost.view(np.uint32), float(t)


def ref_dijkstra_dheap(row, col, w, src, d=2):
    """Dijkstra with decrease-key on the reference's dheap class."""
    row, col, w = _arrs(row, col, w)
    n = row.shape[0] - 1
    cost = np.empty(n, dtype=np.int32)
    t = _load_ref().nps_ref_dijkstra_dheap(n, row.ctypes.data, col.ctypes.data, w.ctypes.data, int(src), int(d),
                                           cost.ctypes.data)
    return cost.view(np.uint32), float(t)


def bfs_levels(row, col, src):
    """Restated bfs_cpu of the bfs-rec application (apps/bfs-rec/src/gpu/bfs_rec.cpp:100-119):
    the hop count from src, BFS_UNDEFINED for unreachable vertices.  The reference
    walks a FIFO queue and re-queues a vertex whose level drops; in FIFO order a
    vertex is first reached at its least hop count, so the levels are those of a
    level-synchronous sweep, which this restatement runs one frontier at a time
    in numpy."""
    row = np.ascontiguousarray(row, dtype=np.int64)
    col = np.ascontiguousarray(col, dtype=np.int64)
    n = row.shape[0] - 1
    level = np.full(n, BFS_UNDEFINED, dtype=np.int32)
    level[src] = 0
    frontier = np.array([src], dtype=np.int64)
    depth = 0
    while frontier.size:
        depth += 1
        starts, ends = row[frontier], row[frontier + 1]
        lens = ends - starts
        total = int(lens.sum())
        if total == 0:
            break
        # edge indices of every frontier row, concatenated
        offs = np.repeat(starts - np.concatenate(([0], np.cumsum(lens)[:-1])), lens)
        nbr = col[np.arange(total, dtype=np.int64) + offs]
        nbr = np.unique(nbr[level[nbr] == BFS_UNDEFINED])
        level[nbr] = depth
        frontier = nbr
    return level


def have_reference_bfs() -> bool:
    return os.path.exists(REF_BFS_SO)


_ref_bfs = None


def ref_bfs_cpu(row, col, src):
    """The reference's bfs_cpu() on these arrays; returns (levels int32, seconds)."""
    global _ref_bfs
    if _ref_bfs is None:
        if not have_reference_bfs():
            raise ImportError(f"{REF_BFS_SO} missing: the reference CPU code was not built")
        lib = C.CDLL(REF_BFS_SO)
        lib.nps_ref_bfs_cpu.argtypes = [_I32, _I32, _P, _P, _I32, _P]
        lib.nps_ref_bfs_cpu.restype = _D
        _ref_bfs = lib
    row = np.ascontiguousarray(row, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    n, m = row.shape[0] - 1, col.shape[0]
    level = np.empty(n, dtype=np.int32)
    t = _ref_bfs.nps_ref_bfs_cpu(n, m, row.ctypes.data, col.ctypes.data, int(src), level.ctypes.data)
    return level, float(t)


def spmv_data(n, m):
    """The values and x the reference's SpMV multiplies (prepare_cpu,
    apps/SpMV/src/cpu/SpMV_kernel.cpp:11-16; the GPU build's prepare_gpu,
    apps/SpMV/src/gpu/SpMV_wrapper.cu:105-113): val[i] = i % 13 + 0.5 and
    x[i] = i % 17 + 0.5, in double."""
    return (np.arange(m) % 13 + 0.5).astype(np.float64), (np.arange(n) % 17 + 0.5).astype(np.float64)


def spmv(row, col, val, x):
    """Restated spmv_omp (apps/SpMV/src/cpu/SpMV_kernel.cpp:26-42): y[r] = sum over
    row r of val[k] * x[col[k]], accumulated from 0 in k order (bincount adds its
    weights in index order, the reference's loop order)."""
    row = np.ascontiguousarray(row, dtype=np.int64)
    n = row.shape[0] - 1
    deg = np.diff(row)
    prod = np.asarray(val, dtype=np.float64) * np.asarray(x, dtype=np.float64)[np.asarray(col, dtype=np.int64)]
    owner = np.repeat(np.arange(n, dtype=np.int64), deg)
    return np.bincount(owner, weights=prod, minlength=n).astype(np.float64)


def have_reference_spmv() -> bool:
    return os.path.exists(REF_SPMV_SO)


_ref_spmv = None


def ref_spmv_cpu(row, col, threads=1):
    """The reference's SpMV_CPU path on this matrix: its own prepare_cpu() data and
    spmv_omp() with `threads` OpenMP threads.  Returns (y, x, val, seconds)."""
    global _ref_spmv
    if _ref_spmv is None:
        if not have_reference_spmv():
            raise ImportError(f"{REF_SPMV_SO} missing: the reference CPU code was not built")
        lib = C.CDLL(REF_SPMV_SO)
        lib.nps_ref_spmv_cpu.argtypes = [_I32, _I32, _P, _P, _I32, _P, _P, _P]
        lib.nps_ref_spmv_cpu.restype = _D
        _ref_spmv = lib
    row = np.ascontiguousarray(row, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    n, m = row.shape[0] - 1, col.shape[0]
    y, x, val = np.empty(n), np.empty(n), np.empty(max(m, 1))
    t = _ref_spmv.nps_ref_spmv_cpu(n, m, row.ctypes.data, col.ctypes.data, int(threads), y.ctypes.data,
                                   x.ctypes.data, val.ctypes.data)
    return y, x, val[:m], float(t)


def bc(row, col, sources=None):
    """Restated bc_cpu (apps/bc/src/cpu/bc.cpp:152-186, bc_kernel.cpp:3-106):
    float32 betweenness centrality over `sources` in the given order (every
    vertex in id order when None), with the reference's float / double rounding
    step by step (see oracle_bc in sssp_oracle.c)."""
    row = np.ascontiguousarray(row, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    n = row.shape[0] - 1
    out = np.empty(n, dtype=np.float32)
    if sources is None:
        rc = _load_oracle().oracle_bc(n, row.ctypes.data, col.ctypes.data, 0, None, out.ctypes.data)
    else:
        src = np.ascontiguousarray(sources, dtype=np.int32)
        rc = _load_oracle().oracle_bc(n, row.ctypes.data, col.ctypes.data, src.shape[0], src.ctypes.data,
                                      out.ctypes.data)
    if rc != 0:
        raise RuntimeError("oracle_bc: out of memory")
    return out


def color(row, col, literal=False):
    """The graph-color application's colors (gclr_bitmap_kernel,
    apps/graph-color/src/gpu/graph_color_kernel.cu:14-35): (int32 colors, the
    iteration count).  literal=True simulates the reference's iterations one by
    one (O(n x iterations)); the default is the closed form in id order."""
    row = np.ascontiguousarray(row, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    n = row.shape[0] - 1
    out = np.zeros(n, dtype=np.int32)
    fn = _load_oracle().oracle_color_iterations if literal else _load_oracle().oracle_color
    it = fn(n, row.ctypes.data, col.ctypes.data, out.ctypes.data)
    return out, int(it)


def have_reference_bc() -> bool:
    return os.path.exists(REF_BC_SO)


_ref_bc = None


def ref_bc_cpu(row, col):
    """The reference's bc_cpu() over every source (one OpenMP thread; it holds an
    n x n byte matrix, so only small graphs).  Returns (bc float32, seconds)."""
    global _ref_bc
    if _ref_bc is None:
        if not have_reference_bc():
            raise ImportError(f"{REF_BC_SO} missing: the reference CPU code was not built")
        lib = C.CDLL(REF_BC_SO)
        lib.nps_ref_bc_cpu.argtypes = [_I32, _I32, _P, _P, _P]
        lib.nps_ref_bc_cpu.restype = _D
        _ref_bc = lib
    row = np.ascontiguousarray(row, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    n = row.shape[0] - 1
    out = np.empty(n, dtype=np.float32)
    t = _ref_bc.nps_ref_bc_cpu(n, col.shape[0], row.ctypes.data, col.ctypes.data, out.ctypes.data)
    return out, float(t)


def degree_stats(row):
    """Restated getStatInfo() of the reference's graph analyzer
    (utility/graph-analyzer/analyzer.cpp:75-138) on CSR row offsets: degrees are the
    row lengths; the maximum and minimum keep the first (lowest) vertex id that
    attains them, and the minimum starts from 999999 (analyzer.cpp:85-86, strict
    comparisons at :101-108); the average is float(total) / n (:110); "Edge by
    degree" is total / 2 (:112).  Also the 8-bin histogram [4^k - 1, 4^(k+1) - 1)
    and the distribution (vertices per degree, 0..max)."""
    row = np.ascontiguousarray(row, dtype=np.int64)
    deg = np.diff(row)
    n = deg.shape[0]
    total = int(deg.sum())
    mx = int(deg.max()) if n else 0
    below = deg < 999999
    mn = int(deg[below].min()) if below.any() else 999999
    lb = np.floor(np.log2(deg.astype(np.float64) + 1.0)).astype(np.int64) >> 1
    bins = np.bincount(np.minimum(lb, 7), minlength=8)[:8]
    return {"n": n, "m": int(row[-1]), "total_degree": total, "edges_by_degree": total // 2,
            "avg_degree": float(np.float32(total) / np.float32(n)), "max_degree": mx, "min_degree": mn,
            "max_degree_node": int(np.argmax(deg == mx)) if n else -1,
            "min_degree_node": int(np.argmax(deg == mn)) if below.any() else -1,
            "bins": [int(x) for x in bins], "dist": np.bincount(deg, minlength=mx + 1).astype(np.int64)}


ANALYZER = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "analyzer")


def ref_analyzer(path, fmt=0):
    """Run the reference's graph analyzer (built from utility/graph-analyzer/ by
    this directory's Makefile into _ref/analyzer) on a graph file with -d; returns
    its printed statistics and distribution."""
    import subprocess
    r = subprocess.run([ANALYZER, "-i", str(path), "-f", str(int(fmt)), "-d"], capture_output=True, text=True,
                       timeout=600)
    if r.returncode != 0:
        raise RuntimeError(f"reference analyzer failed ({r.returncode}): {r.stderr[-200:]}")
    out = {"dist": {}}
    keys = {"Node": "n", "Edge by degree": "edges_by_degree", "Edge": "m", "Avg": "avg_degree",
            "Max": "max_degree", "Min": "min_degree", "Node ID with max degree": "max_degree_node",
            "Node ID with min degree": "min_degree_node"}
    for line in r.stdout.splitlines():
        if ":" in line:
            k, v = line.split(":", 1)
            if k.strip() in keys:
                out[keys[k.strip()]] = float(v) if k.strip() == "Avg" else int(v)
        elif line.strip():
            d, c = line.split()
            out["dist"][int(d)] = int(c)
    return out


def have_analyzer() -> bool:
    return os.path.exists(ANALYZER)


def timed(fn, *a, **k):
    t0 = time.perf_counter()
    r = fn(*a, **k)
    return r, time.perf_counter() - t0


def ref_read_graph(path, fmt):
    """The reference's readInputDIMACS9/10/SLNDC (fmt 0/1/2) + convertCSR on a file.
    Returns (row int32[n+1], col int32[m], w uint32[m], source)."""
    lib = _load_ref()
    if not hasattr(lib, "_rg_typed"):
        lib.nps_ref_read_graph.argtypes = [C.c_char_p, _I32] + [C.POINTER(_I32)] * 3 + [_P, _P, _P, _I32, _I32]
        lib.nps_ref_read_graph.restype = C.c_int
        lib._rg_typed = True
    n, m, s = _I32(0), _I32(0), _I32(0)
    p = str(path).encode()
    rc = lib.nps_ref_read_graph(p, int(fmt), C.byref(n), C.byref(m), C.byref(s), None, None, None, 0, 0)
    if rc != 0:
        raise RuntimeError(f"reference reader failed ({rc})")
    row = np.empty(n.value + 1, np.int32)
    col = np.empty(max(m.value, 1), np.int32)
    w = np.empty(max(m.value, 1), np.int32)
    rc = lib.nps_ref_read_graph(p, int(fmt), C.byref(n), C.byref(m), C.byref(s), row.ctypes.data, col.ctypes.data,
                                w.ctypes.data, n.value, m.value)
    if rc != 0:
        raise RuntimeError(f"reference reader failed ({rc})")
    return row, col[: m.value], w[: m.value].view(np.uint32), int(s.value)
