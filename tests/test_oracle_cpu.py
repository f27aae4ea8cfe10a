"""The oracle and the generators against the golden fixtures (CPU only).

tests/golden/golden.json was produced by tests/golden/make_golden.py, which ran
the reference's own SSSP_CPU() (apps/sssp/src/cpu/sssp.cpp:13-47, built from its
sources) on graphs from this repository's seeded generators.  These tests pin:
  * the generators (CSR fingerprints must not drift),
  * the oracle's restated heap Dijkstra and d-heap Dijkstra (distance fingerprints),
  * when oracle/_ref is present, the restatement against the reference itself on
    further random graphs.
"""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "golden.json")))
DISTS = np.load(os.path.join(HERE, "golden", "golden_dist.npz"))


def _gen(nps, case):
    a = case["args"]
    if case["kind"] == "uniform":
        return nps.gen_uniform(a["n"], a["m"], a["wmax"], a["seed"])
    if case["kind"] == "rmat":
        return nps.gen_rmat(a["scale"], a["edge_factor"], seed=a["seed"])
    return nps.gen_grid(a["rows"], a["cols"], a["drop"], a["wmax"], a["seed"])


@pytest.mark.parametrize("name", sorted(GOLD["cases"]))
def test_generators_reproduce_golden_csr(nps, name):
    case = GOLD["cases"][name]
    g = _gen(nps, case)
    assert (g.n, g.m) == (case["n"], case["m"])
    h = case["csr_fnv1a"]
    assert nps.fnv1a(g.row_ptr.view(np.uint32)) == h["row"]
    assert nps.fnv1a(g.col.view(np.uint32)) == h["col"]
    assert nps.fnv1a(g.w) == h["w"]


@pytest.mark.parametrize("name", sorted(GOLD["cases"]))
def test_oracle_heap_and_dheap_match_reference_goldens(nps, oracle, name):
    case = GOLD["cases"][name]
    g = _gen(nps, case)
    d = oracle.sssp_heap(g.row_ptr, g.col, g.w, case["source"])
    assert oracle.fnv1a(d) == case["dist_fnv1a"]
    assert oracle.reached(g.row_ptr, d) == (case["n_reached"], case["m_reached"])
    if name in DISTS.files:
        assert np.array_equal(d, DISTS[name])
    for arity in (2, 4, 8):
        assert oracle.fnv1a(oracle.sssp_dheap(g.row_ptr, g.col, g.w, case["source"], arity)) == case["dist_fnv1a"]


@pytest.mark.parametrize("name", sorted(GOLD["edge_cases"]))
def test_oracle_edge_cases(nps, oracle, name):
    c = GOLD["edge_cases"][name]
    g = nps.convertCSR(c["n"], c["src"], c["dst"], c["w"])
    assert oracle.sssp_heap(g.row_ptr, g.col, g.w, c["source"]).tolist() == c["dist"]
    assert oracle.sssp_dheap(g.row_ptr, g.col, g.w, c["source"]).tolist() == c["dist"]


def test_state_oracle_reduces_to_dijkstra_from_the_standard_state(nps, oracle):
    """From prepare_gpu()'s state (INF except the source, update[source] = 1) the
    fixpoint is ordinary SSSP."""
    g = nps.gen_rmat(12, 8, seed=3)
    cost = np.full(g.n, oracle.INF, np.uint32)
    upd = np.zeros(g.n, np.uint8)
    cost[g.source] = 0
    upd[g.source] = 1
    c, u = oracle.sssp_state(g.row_ptr, g.col, g.w, cost, upd)
    assert np.array_equal(c, oracle.sssp_heap(g.row_ptr, g.col, g.w, g.source))
    assert u.sum() == 0


def test_state_oracle_keeps_unflagged_values_that_are_never_improved(nps, oracle):
    # 0 -> 1 (w 10), 1 -> 2 (w 1); vertex 1 starts at 2 (not flagged): 0's path does not
    # improve it, so 1 never propagates and 2 stays INF (the label-correcting fixpoint)
    g = nps.convertCSR(3, [0, 1], [1, 2], [10, 1])
    c, _ = oracle.sssp_state(g.row_ptr, g.col, g.w, np.array([0, 2, oracle.INF], np.uint32),
                             np.array([1, 0, 0], np.uint8))
    assert c.tolist() == [0, 2, oracle.INF]


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libref_sssp.so")),
                    reason="reference CPU code not built")
@pytest.mark.parametrize("seed", range(6))
def test_restatement_against_the_reference_itself(nps, oracle, seed):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(50, 3000))
    m = int(rng.integers(0, 20 * n))
    s = rng.integers(0, n, m)
    t = rng.integers(0, n, m)
    w = rng.integers(0, 300 if seed % 2 else 5, m)
    g = nps.convertCSR(n, s, t, w)
    src = int(rng.integers(0, n))
    ref, _ = oracle.ref_sssp_cpu(g.row_ptr, g.col, g.w, src)
    assert np.array_equal(oracle.sssp_heap(g.row_ptr, g.col, g.w, src), ref)
    assert np.array_equal(oracle.sssp_dheap(g.row_ptr, g.col, g.w, src), ref)
    rd, _ = oracle.ref_dijkstra_dheap(g.row_ptr, g.col, g.w, src)
    assert np.array_equal(rd, ref)
    u1, _ = oracle.ref_usssp_cpu(g.row_ptr, g.col, g.w, src, threads=1)  # exact with one thread
    assert np.array_equal(u1, ref)


@pytest.mark.parametrize("scale,ef,seed,probs", [(8, 4, 1, (0.57, 0.19, 0.19)), (12, 16, 1000, (0.57, 0.19, 0.19)),
                                                  (14, 8, 7, (0.45, 0.15, 0.15)), (17, 16, 3, (0.57, 0.19, 0.19))])
def test_oracle_rmat_input_equals_the_library_generator(nps, oracle, scale, ef, seed, probs):
    """The benchmark's reference arm builds its input with the oracle's generator (so it
    never loads the library); it must be the same graph, source included."""
    a, b, c = probs
    row, col, w, src = oracle.gen_rmat(scale, ef, seed, a, b, c, 255)
    g = nps.gen_rmat(scale, ef, a, b, c, seed=seed)
    assert np.array_equal(row, g.row_ptr) and np.array_equal(col, g.col) and np.array_equal(w, g.w)
    assert src == g.source
