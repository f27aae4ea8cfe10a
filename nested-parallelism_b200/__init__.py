"""B200-native single-source shortest paths with warp / block / grid workload
consolidation -- the Python face of libnps.so.

The names mirror the reference's SSSP path (dadaism/nested-parallelism):

  readInputDIMACS9 / readInputDIMACS10 / readInputSLNDC   common/global.cpp:29-190
  convertCSR                                              common/global.cpp:192-235
  SSSP_GPU                                                apps/sssp/src/gpu/sssp_wrapper.cu:548-583
  sssp_np_consolidate_gpu                                 apps/sssp/src/gpu/sssp_wrapper.cu:475-546
  CONSOLIDATE_WARP/BLOCK/GRID (CONSOLIDATE_LEVEL 0/1/2)   apps/sssp/src/gpu/sssp_wrapper.cu:503-531
  THRESHOLD = 64                                          apps/sssp/src/gpu/sssp_kernel.cu:7
  INF = 2^30                                              apps/sssp/src/gpu/sssp_wrapper.cu:7

Where the reference calls exit() on an error this module raises NpsError.
Every compute call runs the CUDA kernels of libnps.so; there is no CPU path.
Import it as importlib.import_module("nested-parallelism_b200").
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Iterable, List, Optional, Sequence

import numpy as np

from ._native import (NPS_INF, NPS_MLP_HID, NPS_MLP_IN, NPS_MLP_OUT, NpsError, check, lib,
                      nps_degree_info, nps_graph, nps_instance, nps_params, nps_solution_info, nps_stats,
                      nps_trace_rec)

INF = NPS_INF
THRESHOLD = 64
CONSOLIDATE_WARP, CONSOLIDATE_BLOCK, CONSOLIDATE_GRID, CONSOLIDATE_HYBRID = 0, 1, 2, 3
POLICY_PLAIN, POLICY_LEARNED = 0, 1
SCHEDULE_ITERATIONS, SCHEDULE_ASYNC = 0, 1
# `-s <solution>` of the reference CLI (apps/sssp/src/gpu/sssp.cpp:38), the cases of
# SSSP_GPU()'s switch (apps/sssp/src/gpu/sssp_wrapper.cu:554-566)
(SOLUTION_TQUEUE, SOLUTION_DUAL_QUEUE, SOLUTION_SHARED_DELAYED, SOLUTION_GLOBAL_DELAYED,
 SOLUTION_NP_NAIVE, SOLUTION_NP_OPT, SOLUTION_CONSOLIDATE) = range(7)
SOLUTION_NAMES = ("sssp_tqueue_gpu", "sssp_dual_queue_gpu", "sssp_shared_delayed_buffer_gpu",
                  "sssp_global_delayed_buffer_gpu", "sssp_np_naive_gpu", "sssp_np_opt_gpu",
                  "sssp_np_consolidate_gpu")

__all__ = [
    "INF", "THRESHOLD", "CONSOLIDATE_WARP", "CONSOLIDATE_BLOCK", "CONSOLIDATE_GRID",
    "CONSOLIDATE_HYBRID", "POLICY_PLAIN", "POLICY_LEARNED", "SCHEDULE_ITERATIONS", "SCHEDULE_ASYNC", "Graph", "Params", "Stats",
    "NpsError", "gen_uniform", "gen_rmat", "gen_grid", "convertCSR", "readInputDIMACS9",
    "readInputDIMACS10", "readInputSLNDC", "writeDIMACS9", "sssp", "sssp_device", "SSSP_GPU",
    "sssp_np_consolidate_gpu", "sssp_solution", "sssp_solution_state", "SolutionInfo",
    "SOLUTION_TQUEUE", "SOLUTION_DUAL_QUEUE", "SOLUTION_SHARED_DELAYED", "SOLUTION_GLOBAL_DELAYED",
    "SOLUTION_NP_NAIVE", "SOLUTION_NP_OPT", "SOLUTION_CONSOLIDATE", "SOLUTION_NAMES", "sssp_batch",
    "bfs", "bfs_device", "bfs_params", "BFS_UNDEFINED", "spmv", "spmv_device", "bc", "bc_device", "color", "color_device", "trace_read", "fnv1a", "delta_schedule", "degree_stats", "abi_version", "lib",
]


def abi_version() -> int:
    return int(lib.nps_abi_version())


# ---------------------------------------------------------------------------
# graphs

@dataclass
class Graph:
    """CSR graph: the struct _GRAPH_ members and noNodeTotal / noEdgeTotal /
    source globals of common/global.h:28-58."""
    vertexArray: np.ndarray  # int32 [n+1]
    edgeArray: np.ndarray    # int32 [m]
    weightArray: np.ndarray  # uint32 [m]
    source: int = 0

    @property
    def noNodeTotal(self) -> int:
        return int(self.vertexArray.shape[0] - 1)

    @property
    def noEdgeTotal(self) -> int:
        return int(self.edgeArray.shape[0])

    n = noNodeTotal
    m = noEdgeTotal

    @property
    def row_ptr(self) -> np.ndarray:
        return self.vertexArray

    @property
    def col(self) -> np.ndarray:
        return self.edgeArray

    @property
    def w(self) -> np.ndarray:
        return self.weightArray

    def degrees(self) -> np.ndarray:
        return np.diff(self.vertexArray)


def _take(g: nps_graph) -> Graph:
    try:
        n, m = int(g.n), int(g.m)
        row = np.ctypeslib.as_array(g.row_ptr, shape=(n + 1,)).copy()
        col = np.ctypeslib.as_array(g.col, shape=(max(m, 1),))[:m].copy()
        w = np.ctypeslib.as_array(g.w, shape=(max(m, 1),))[:m].copy()
        return Graph(row, col, w, int(g.source))
    finally:
        lib.nps_graph_free(C.byref(g))


def gen_uniform(n: int, m: int, wmax: int = 100, seed: int = 1) -> Graph:
    """Uniform random directed graph: each edge picks src and dst uniformly
    (self-loops redrawn), weight uniform in [1, wmax]; source 0."""
    g = nps_graph()
    check(lib.nps_gen_uniform(n, m, wmax, seed, C.byref(g)), "gen_uniform")
    return _take(g)


def gen_rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
             wmax: int = 255, seed: int = 1) -> Graph:
    """R-MAT graph (no noise), duplicates and self-loops removed; source is the
    highest-out-degree vertex (lowest id on ties)."""
    g = nps_graph()
    check(lib.nps_gen_rmat(scale, edge_factor, a, b, c, wmax, seed, C.byref(g)), "gen_rmat")
    return _take(g)


def gen_grid(rows: int, cols: int, drop: float = 0.05, wmax: int = 1000, seed: int = 1) -> Graph:
    """4-neighbour grid, each undirected pair dropped with probability `drop`,
    independent weights per direction in [1, wmax]; source (0, 0)."""
    g = nps_graph()
    check(lib.nps_gen_grid(rows, cols, drop, wmax, seed, C.byref(g)), "gen_grid")
    return _take(g)


def convertCSR(n: int, src, dst, w, dedupe: bool = False, drop_self_loops: bool = False) -> Graph:
    """Edge list (in insertion order) to CSR with every row in reverse insertion
    order, as convertCSR() lays out the adjacency lists (global.cpp:211-225)."""
    s = np.ascontiguousarray(src, dtype=np.int32)
    d = np.ascontiguousarray(dst, dtype=np.int32)
    ww = np.ascontiguousarray(w, dtype=np.uint32)
    if not (s.shape == d.shape == ww.shape):
        raise ValueError("src, dst and w must have the same length")
    g = nps_graph()
    check(lib.nps_csr_from_edges(n, s.shape[0], s.ctypes.data, d.ctypes.data, ww.ctypes.data,
                                 int(dedupe), int(drop_self_loops), C.byref(g)), "convertCSR")
    return _take(g)


def _read(fn, path: str, where: str) -> Graph:
    g = nps_graph()
    check(fn(str(path).encode(), C.byref(g)), where)
    return _take(g)


def readInputDIMACS9(path: str) -> Graph:
    return _read(lib.nps_read_dimacs9, path, "readInputDIMACS9")


def readInputDIMACS10(path: str) -> Graph:
    return _read(lib.nps_read_dimacs10, path, "readInputDIMACS10")


def readInputSLNDC(path: str) -> Graph:
    return _read(lib.nps_read_slndc, path, "readInputSLNDC")


def _as_nps_graph(g: Graph) -> nps_graph:
    row = np.ascontiguousarray(g.vertexArray, dtype=np.int32)
    col = np.ascontiguousarray(g.edgeArray, dtype=np.int32)
    w = np.ascontiguousarray(g.weightArray, dtype=np.uint32)
    ng = nps_graph()
    ng.n, ng.m, ng.source = row.shape[0] - 1, col.shape[0], int(g.source)
    ng.row_ptr = row.ctypes.data_as(C.POINTER(C.c_int32))
    ng.col = col.ctypes.data_as(C.POINTER(C.c_int32))
    ng.w = w.ctypes.data_as(C.POINTER(C.c_uint32))
    ng._keep = (row, col, w)  # keep the buffers alive with the struct
    return ng


def writeDIMACS9(path: str, g: Graph, source: Optional[int] = None) -> None:
    ng = _as_nps_graph(g)
    check(lib.nps_write_dimacs9(str(path).encode(), C.byref(ng), g.source if source is None else source),
          "writeDIMACS9")


def delta_schedule(first, rest: int) -> int:
    """Params.delta_schedule word: bucket b < len(first) is 2**first[b] wide (at most
    7 entries), every later bucket 2**rest.  Exponents are 0..15."""
    ks = list(first)
    if len(ks) > 7 or not all(0 <= k <= 15 for k in ks + [rest]):
        raise ValueError("at most 7 leading exponents, each in 0..15")
    ks = ks + [rest] * (7 - len(ks))
    word = 0
    for b, k in enumerate(ks + [rest]):
        word |= int(k) << (4 * b)
    return word


def fnv1a(dist: np.ndarray) -> int:
    a = np.ascontiguousarray(dist, dtype=np.uint32)
    return int(lib.nps_fnv1a_u32(a.ctypes.data, a.shape[0]))


# ---------------------------------------------------------------------------
# parameters and statistics

@dataclass
class Params:
    level: int = CONSOLIDATE_BLOCK      # CONSOLIDATE_LEVEL (Makefile default 1)
    threshold: int = THRESHOLD
    block_threshold: int = 256
    grid_threshold: int = 4096
    block_size: int = 256
    ctas_per_sm: int = 0
    delta: int = 0                      # 0 = the reference's unordered frontier
    policy: int = POLICY_PLAIN
    device: int = 0
    timeout_s: float = 10.0
    trace: bool = False
    light_heavy: bool = True            # delta > 0: heavy edges (w >= delta) relaxed once per bucket
    local_rounds: int = 0               # warp-local rounds on just-improved vertices per work item
    order_degree: int = 0               # delta > 0: rows below this degree ignore the bucket bound
    delta_schedule: int = 0             # per-bucket log2 widths, 4 bits each (see delta_schedule())
    fault_inject_wait: bool = False     # test hook: the first barrier can never complete
    fault_inject_disagree: bool = False  # test hook: CTA 1 reports another decision hash (NPS_ERR_INTERNAL)
    bc_block_sources: int = 0           # bc: sources per block of dependency rows (0 = as memory allows)
    schedule: int = 0                   # SCHEDULE_ITERATIONS or SCHEDULE_ASYNC (see include/nps.h)
    policy_min_edges: int = 0           # learned policy only from this many edges (0: library default, <0: none)
    sort_at_push: int = 0               # grid-tier rows sorted at push: 1 on, -1 off, 0 by the grid threshold

    def to_c(self, device_ptrs: bool, stream: Optional[int] = None) -> nps_params:
        p = nps_params()
        lib.nps_params_default(C.byref(p))
        p.level, p.threshold = self.level, self.threshold
        p.block_threshold, p.grid_threshold = self.block_threshold, self.grid_threshold
        p.block_size, p.ctas_per_sm, p.delta = self.block_size, self.ctas_per_sm, self.delta
        p.policy, p.device, p.timeout_s = self.policy, self.device, float(self.timeout_s)
        p.trace = int(bool(self.trace))
        p.light_heavy = int(bool(self.light_heavy))
        p.local_rounds = int(self.local_rounds)
        p.order_degree = int(self.order_degree)
        p.delta_schedule = int(self.delta_schedule) & 0xFFFFFFFF
        p.device_ptrs = int(bool(device_ptrs))
        p.stream = stream
        p.reserved[0] = 2 if self.fault_inject_disagree else int(bool(self.fault_inject_wait))
        p.reserved[1] = int(self.bc_block_sources)
        p.schedule = int(self.schedule)
        p.policy_min_edges = int(self.policy_min_edges)
        p.sort_at_push = int(self.sort_at_push)
        return p


@dataclass
class Stats:
    iterations: int = 0
    buckets: int = 0
    edges_scanned: int = 0
    improvements: int = 0
    vertices_processed: int = 0
    reached: int = 0
    kernel_ms: float = 0.0
    total_ms: float = 0.0
    status: int = 0
    grid_ctas: int = 0
    phase_cycles: tuple = ()
    policy_used: int = 0

    @staticmethod
    def from_c(s: nps_stats) -> "Stats":
        return Stats(int(s.iterations), int(s.buckets), int(s.edges_scanned), int(s.improvements),
                     int(s.vertices_processed), int(s.reached), float(s.kernel_ms), float(s.total_ms),
                     int(s.status), int(s.grid_ctas), tuple(int(x) for x in s.phase_cycles),
                     int(s.policy_used))


def _ptr(x) -> int:
    """Device pointer of a tensor-like object (data_ptr()) or a raw int."""
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return int(x.data_ptr())
    raise TypeError(f"expected a device pointer or an object with data_ptr(), got {type(x)!r}")


# ---------------------------------------------------------------------------
# SSSP

def sssp(g: Graph, source: Optional[int] = None, params: Optional[Params] = None,
         out: Optional[np.ndarray] = None):
    """Shortest distances from `source` on host CSR arrays.  The call copies the
    graph to the device, runs one persistent launch and copies distances back.
    Returns (dist uint32[n], Stats); unreachable vertices hold INF."""
    p = params or Params()
    src = g.source if source is None else int(source)
    row = np.ascontiguousarray(g.vertexArray, dtype=np.int32)
    col = np.ascontiguousarray(g.edgeArray, dtype=np.int32)
    w = np.ascontiguousarray(g.weightArray, dtype=np.uint32)
    n = row.shape[0] - 1
    dist = out if out is not None else np.empty(n, dtype=np.uint32)
    if dist.dtype != np.uint32 or dist.shape[0] != n or not dist.flags.c_contiguous:
        raise ValueError("out must be a contiguous uint32 array of n entries")
    st = nps_stats()
    cp = p.to_c(device_ptrs=False)
    check(lib.nps_sssp(row.ctypes.data, col.ctypes.data, w.ctypes.data, n, col.shape[0], src,
                       C.byref(cp), dist.ctypes.data, C.byref(st)), "sssp")
    return dist, Stats.from_c(st)


def sssp_device(row_ptr, col, w, n: int, m: int, src: int, dist_out,
                params: Optional[Params] = None, stream: Optional[int] = None) -> Stats:
    """Same on device-resident arrays (tensors or raw pointers); launches on
    `stream` (a cudaStream_t as int) when given, else on the library's stream."""
    p = params or Params()
    st = nps_stats()
    cp = p.to_c(device_ptrs=True, stream=stream)
    check(lib.nps_sssp(_ptr(row_ptr), _ptr(col), _ptr(w), n, m, src, C.byref(cp), _ptr(dist_out),
                       C.byref(st)), "sssp_device")
    return Stats.from_c(st)


BFS_UNDEFINED = 0x7FFFFFFF  # apps/bfs-rec/src/gpu/bfs_rec.h:13


def bfs_params(**kw) -> Params:
    """Default BFS configuration: the unordered frontier (delta 0) at the grid
    consolidation level, threshold 32, 512-thread CTAs.  With unit weights each
    frontier is already one BFS level, so every reached row is walked once
    without buckets.  On R-MAT scale 22 a sweep of level x threshold x CTA size
    gave 0.60 ms for this configuration (0.77 ms with 256-thread CTAs and
    threshold 64, 1.17 ms with one-level buckets)."""
    kw.setdefault("level", CONSOLIDATE_GRID)
    kw.setdefault("delta", 0)
    kw.setdefault("threshold", 32)
    kw.setdefault("block_size", 512)
    return Params(**kw)


def bfs(g: Graph, source: Optional[int] = None, params: Optional[Params] = None) -> tuple:
    """Breadth-first levels from `source` on host arrays -- the bfs-rec application's
    bfs_rec_dp_cons_gpu() (apps/bfs-rec/src/gpu/bfs_rec_wrapper.cu:170-229) on the
    SSSP engine with every edge weighing 1.  Returns (int32 levels with
    BFS_UNDEFINED for unreachable vertices, Stats)."""
    p = params or bfs_params()
    src = g.source if source is None else source
    row = np.ascontiguousarray(g.vertexArray, dtype=np.int32)
    col = np.ascontiguousarray(g.edgeArray, dtype=np.int32)
    level = np.empty(g.noNodeTotal, dtype=np.int32)
    st = nps_stats()
    cp = p.to_c(device_ptrs=False)
    check(lib.nps_bfs(row.ctypes.data, col.ctypes.data, g.noNodeTotal, col.shape[0], src, C.byref(cp),
                      level.ctypes.data, C.byref(st)), "bfs")
    return level, Stats.from_c(st)


def bfs_device(row_ptr, col, n: int, m: int, src: int, level_out, params: Optional[Params] = None,
               stream: Optional[int] = None) -> Stats:
    """bfs() on device-resident arrays (tensors or raw pointers): level_out (int32[n])
    receives the levels, as bfs_rec_dp_cons_gpu() leaves d_levelArray."""
    p = params or bfs_params()
    st = nps_stats()
    cp = p.to_c(device_ptrs=True, stream=stream)
    check(lib.nps_bfs(_ptr(row_ptr), _ptr(col), n, m, src, C.byref(cp), _ptr(level_out), C.byref(st)),
          "bfs_device")
    return Stats.from_c(st)


def spmv(g: Graph, val, x, params: Optional[Params] = None) -> tuple:
    """y = A x for the CSR matrix of `g` (row offsets and columns) with values
    `val` (float64[m]) and x (float64[n]) on host arrays -- the SpMV application's
    spmv_np_consolidate_gpu() (apps/SpMV/src/gpu/SpMV_wrapper.cu:285-311).  Returns
    (y float64[n], Stats).  params.level (WARP, BLOCK or GRID, default GRID) and
    params.threshold select the consolidation of long rows."""
    p = params or Params(level=CONSOLIDATE_GRID)
    row = np.ascontiguousarray(g.vertexArray, dtype=np.int32)
    col = np.ascontiguousarray(g.edgeArray, dtype=np.int32)
    val = np.ascontiguousarray(val, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = g.noNodeTotal
    if val.shape[0] != col.shape[0] or x.shape[0] != n:
        raise ValueError("spmv: val needs m entries and x n entries")
    y = np.empty(n, dtype=np.float64)
    st = nps_stats()
    cp = p.to_c(device_ptrs=False)
    check(lib.nps_spmv(row.ctypes.data, col.ctypes.data, val.ctypes.data, x.ctypes.data, y.ctypes.data, n,
                       col.shape[0], C.byref(cp), C.byref(st)), "spmv")
    return y, Stats.from_c(st)


def spmv_device(row_ptr, col, val, x, y, n: int, m: int, params: Optional[Params] = None,
                stream: Optional[int] = None) -> Stats:
    """spmv() on device-resident arrays (tensors or raw pointers)."""
    p = params or Params(level=CONSOLIDATE_GRID)
    st = nps_stats()
    cp = p.to_c(device_ptrs=True, stream=stream)
    check(lib.nps_spmv(_ptr(row_ptr), _ptr(col), _ptr(val), _ptr(x), _ptr(y), n, m, C.byref(cp), C.byref(st)),
          "spmv_device")
    return Stats.from_c(st)


def color(g: Graph, params: Optional[Params] = None) -> tuple:
    """Graph coloring on host arrays -- the graph-color application's
    gclr_np_consolidate_gpu() (apps/graph-color/src/gpu/graph_color_wrapper.cu:368-412).
    Returns (int32 colors, Stats); Stats.iterations is the reference's iteration
    count (the largest color)."""
    p = params or Params()
    row = np.ascontiguousarray(g.vertexArray, dtype=np.int32)
    col = np.ascontiguousarray(g.edgeArray, dtype=np.int32)
    out = np.empty(g.noNodeTotal, dtype=np.int32)
    st = nps_stats()
    cp = p.to_c(device_ptrs=False)
    check(lib.nps_color(row.ctypes.data, col.ctypes.data, g.noNodeTotal, col.shape[0], C.byref(cp), out.ctypes.data,
                        C.byref(st)), "color")
    return out, Stats.from_c(st)


def color_device(row_ptr, col, n: int, m: int, color_out, params: Optional[Params] = None,
                 stream: Optional[int] = None) -> Stats:
    """color() on device-resident arrays, as the reference leaves d_colorArray."""
    p = params or Params()
    st = nps_stats()
    cp = p.to_c(device_ptrs=True, stream=stream)
    check(lib.nps_color(_ptr(row_ptr), _ptr(col), n, m, C.byref(cp), _ptr(color_out), C.byref(st)), "color_device")
    return Stats.from_c(st)


def bc(g: Graph, sources=None, params: Optional[Params] = None) -> tuple:
    """Betweenness centrality on host arrays -- the bc application's
    bc_np_consolidate_gpu() (apps/bc/src/gpu/bc_wrapper.cu:678-741) with the
    exact result of its bc_cpu (apps/bc/src/cpu/bc.cpp:152-186).  `sources` (ints)
    are taken in the given order; None means every vertex in id order, as the
    reference does.  Returns (float32 bc, Stats)."""
    p = params or Params()
    row = np.ascontiguousarray(g.vertexArray, dtype=np.int32)
    col = np.ascontiguousarray(g.edgeArray, dtype=np.int32)
    out = np.empty(g.noNodeTotal, dtype=np.float32)
    st = nps_stats()
    cp = p.to_c(device_ptrs=False)
    if sources is None:
        srcp, ns = None, 0
    else:
        src = np.ascontiguousarray(sources, dtype=np.int32)
        srcp, ns = src.ctypes.data, src.shape[0]
    check(lib.nps_bc(row.ctypes.data, col.ctypes.data, g.noNodeTotal, col.shape[0], srcp, ns, C.byref(cp),
                     out.ctypes.data, C.byref(st)), "bc")
    return out, Stats.from_c(st)


def bc_device(row_ptr, col, n: int, m: int, bc_out, sources=None, nsrc: int = 0,
              params: Optional[Params] = None, stream: Optional[int] = None) -> Stats:
    """bc() on device-resident arrays; `sources` is a device array of nsrc ints or None."""
    p = params or Params()
    st = nps_stats()
    cp = p.to_c(device_ptrs=True, stream=stream)
    check(lib.nps_bc(_ptr(row_ptr), _ptr(col), n, m, None if sources is None else _ptr(sources), nsrc,
                     C.byref(cp), _ptr(bc_out), C.byref(st)), "bc_device")
    return Stats.from_c(st)


@dataclass
class SolutionInfo:
    """How solutions 0-5 handled large rows (nps_solution_info)."""
    deferred: int = 0
    child_launches: int = 0
    launch_fallbacks: int = 0
    host_reads: int = 0

    @staticmethod
    def from_c(s: nps_solution_info) -> "SolutionInfo":
        return SolutionInfo(int(s.deferred), int(s.child_launches), int(s.launch_fallbacks), int(s.host_reads))


def sssp_solution(g: Graph, solution: int, src: Optional[int] = None,
                  params: Optional[Params] = None) -> tuple:
    """One run of SSSP_GPU()'s solution `solution` (0-6, sssp_wrapper.cu:548-583)
    on host arrays: (uint32 distances, Stats, SolutionInfo).  Solutions 0-5 use
    params.threshold (the large-row degree, THRESHOLD = 64 in the reference) and
    params.block_size (threads of the row-per-thread CTAs); 6 is sssp()."""
    p = params or Params()
    src = g.source if src is None else src
    n = g.noNodeTotal
    row = np.ascontiguousarray(g.vertexArray, dtype=np.int32)
    col = np.ascontiguousarray(g.edgeArray, dtype=np.int32)
    w = np.ascontiguousarray(g.weightArray, dtype=np.uint32)
    dist = np.empty(n, dtype=np.uint32)
    st, info = nps_stats(), nps_solution_info()
    cp = p.to_c(device_ptrs=False)
    check(lib.nps_sssp_solution(solution, row.ctypes.data, col.ctypes.data, w.ctypes.data, n, col.shape[0], src,
                                C.byref(cp), dist.ctypes.data, C.byref(st), C.byref(info)),
          f"sssp_solution({solution})")
    return dist, Stats.from_c(st), SolutionInfo.from_c(info)


def sssp_solution_state(solution: int, d_vertexArray, d_edgeArray, d_weightArray, d_costArray, d_update,
                        noNodeTotal: int, noEdgeTotal: int, params: Optional[Params] = None,
                        stream: Optional[int] = None) -> tuple:
    """The state form of solution `solution` (device arrays as prepare_gpu()
    leaves them, as sssp_np_consolidate_gpu): costs updated in place, d_update
    cleared.  Returns (Stats, SolutionInfo)."""
    p = params or Params()
    st, info = nps_stats(), nps_solution_info()
    cp = p.to_c(device_ptrs=True, stream=stream)
    check(lib.nps_sssp_solution_state(solution, _ptr(d_vertexArray), _ptr(d_edgeArray), _ptr(d_weightArray),
                                      noNodeTotal, noEdgeTotal, _ptr(d_costArray), _ptr(d_update), C.byref(cp),
                                      C.byref(st), C.byref(info)), f"sssp_solution_state({solution})")
    return Stats.from_c(st), SolutionInfo.from_c(info)


def SSSP_GPU(g: Graph, solution: int = SOLUTION_CONSOLIDATE, level: int = CONSOLIDATE_BLOCK,
             params: Optional[Params] = None) -> np.ndarray:
    """graph.costArray after one SSSP_GPU() run (sssp_wrapper.cu:548-583): int32
    costs with INF = 2^30 for unreachable vertices.  `solution` selects the case
    of the reference's switch: 0-5 the earlier load-balancing schemes
    (sssp_solution), 6 workload consolidation at `level`."""
    if solution < 0 or solution > SOLUTION_CONSOLIDATE:
        raise NpsError(1, f"SSSP_GPU: solution must be 0..6, got {solution}")
    if solution != SOLUTION_CONSOLIDATE:
        dist, _, _ = sssp_solution(g, solution, g.source, params)
        return dist.view(np.int32)
    p = params or Params(level=level)
    dist, _ = sssp(g, g.source, p)
    return dist.view(np.int32)


def sssp_np_consolidate_gpu(d_vertexArray, d_edgeArray, d_weightArray, d_costArray, d_update,
                            noNodeTotal: int, noEdgeTotal: int, level: int = CONSOLIDATE_BLOCK,
                            params: Optional[Params] = None, stream: Optional[int] = None) -> Stats:
    """The state form of sssp_np_consolidate_gpu() (sssp_wrapper.cu:475-546):
    device arrays as prepare_gpu() leaves them -- d_costArray int32 (INF except
    the source), d_update uint8 flags (the source set).  Costs are updated in
    place and d_update is cleared.  Returns Stats (Stats.iterations is the
    reference's `iteration` counter)."""
    p = params or Params(level=level)
    st = nps_stats()
    cp = p.to_c(device_ptrs=True, stream=stream)
    check(lib.nps_sssp_state(_ptr(d_vertexArray), _ptr(d_edgeArray), _ptr(d_weightArray), noNodeTotal,
                             noEdgeTotal, _ptr(d_costArray), _ptr(d_update), C.byref(cp), C.byref(st)),
          "sssp_np_consolidate_gpu")
    return Stats.from_c(st)


@dataclass
class Instance:
    """One batched SSSP instance on device-resident arrays."""
    row_ptr: object
    col: object
    w: object
    dist: object
    n: int
    m: int
    src: int


def sssp_batch(instances: Sequence[Instance], params: Optional[Params] = None, use_graph: bool = True,
               stream: Optional[int] = None):
    """Run many independent instances in one persistent cooperative launch
    (captured into a CUDA graph and replayed when use_graph).  Returns
    (list[Stats], kernel_ms)."""
    p = params or Params()
    k = len(instances)
    arr = (nps_instance * k)()
    for i, x in enumerate(instances):
        arr[i].row_ptr, arr[i].col, arr[i].w, arr[i].dist = _ptr(x.row_ptr), _ptr(x.col), _ptr(x.w), _ptr(x.dist)
        arr[i].n, arr[i].m, arr[i].src = int(x.n), int(x.m), int(x.src)
    stats = (nps_stats * k)()
    ms = C.c_float(0.0)
    cp = p.to_c(device_ptrs=True, stream=stream)
    check(lib.nps_sssp_batch(arr, k, C.byref(cp), int(bool(use_graph)), stats, C.byref(ms)), "sssp_batch")
    return [Stats.from_c(s) for s in stats], float(ms.value)


def degree_stats(g, distribution: bool = True, device: int = 0) -> dict:
    """Degree statistics of a graph on the GPU: what the reference's graph analyzer
    prints (utility/graph-analyzer/analyzer.cpp:75-138): Node, Edge, Edge by degree
    (total / 2), Avg, Max, Min and the lowest node ids with the maximum / minimum
    degree, plus `bins` (the 8-bin histogram [4^k - 1, 4^(k+1) - 1)) and, with
    `distribution`, `dist` (vertices per degree, 0..max).  `g` is a Graph or a row
    offset array (numpy host array, or a device tensor with `data_ptr`)."""
    if isinstance(g, Graph):
        row, dev_ptr = np.ascontiguousarray(g.row_ptr, np.int32), False
    elif hasattr(g, "data_ptr"):
        row, dev_ptr = g, True
    else:
        row, dev_ptr = np.ascontiguousarray(g, np.int32), False
    n = (int(row.numel()) if dev_ptr else int(row.shape[0])) - 1
    ptr = row.data_ptr() if dev_ptr else row.ctypes.data
    info = nps_degree_info()
    check(lib.nps_degree_stats(ptr, n, int(dev_ptr), device, C.byref(info), None, 0), "degree_stats")
    out = {"n": info.n, "m": int(info.m), "total_degree": int(info.total_degree),
           "edges_by_degree": int(info.edges_by_degree), "avg_degree": float(info.avg_degree),
           "max_degree": info.max_degree, "min_degree": info.min_degree,
           "max_degree_node": info.max_degree_node, "min_degree_node": info.min_degree_node,
           "bins": [int(x) for x in info.bins]}
    if distribution:
        if dev_ptr:
            import torch
            d = torch.empty(info.max_degree + 1, dtype=torch.int64, device=row.device)
            check(lib.nps_degree_stats(ptr, n, 1, device, C.byref(info), d.data_ptr(), d.numel()), "degree_stats")
            out["dist"] = d.cpu().numpy()
        else:
            d = np.zeros(info.max_degree + 1, np.int64)
            check(lib.nps_degree_stats(ptr, n, 0, device, C.byref(info), d.ctypes.data, d.shape[0]), "degree_stats")
            out["dist"] = d
    return out


def trace_read(device: int = 0, cap: int = 1 << 16) -> List[dict]:
    """Per-iteration records of the last call made with Params(trace=True)."""
    buf = (nps_trace_rec * cap)()
    cnt = C.c_int32(0)
    check(lib.nps_trace_read(device, buf, cap, C.byref(cnt)), "trace_read")
    out = []
    for r in buf[: cnt.value]:
        out.append(dict(iteration=r.iteration, frontier=r.frontier, far_len=r.far_len,
                        bucket_hi=r.bucket_hi, delta=r.delta, level=r.level, hist=list(r.hist),
                        edges=int(r.edges), improvements=int(r.improvements), reached=r.reached,
                        heavy=r.heavy, t_us=r.t_ns / 1e3, feat=list(r.feat)))
    return out
