"""Graph construction and the file front-ends (CPU only).

The readers replace readInputDIMACS9/10/SLNDC() + convertCSR() (common/
global.cpp:29-235); their output on the fixture files must equal what the
reference's own readers produced (fingerprints in tests/golden/golden.json).
"""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
GOLD = json.load(open(os.path.join(GOLDEN, "golden.json")))
READERS = {0: "readInputDIMACS9", 1: "readInputDIMACS10", 2: "readInputSLNDC"}


@pytest.mark.parametrize("fname", sorted(GOLD["readers"]))
def test_readers_match_the_reference_readers(nps, fname):
    exp = GOLD["readers"][fname]
    g = getattr(nps, READERS[exp["format"]])(os.path.join(GOLDEN, fname))
    assert (g.n, g.m, g.source) == (exp["n"], exp["m"], exp["source"])
    assert nps.fnv1a(g.row_ptr.view(np.uint32)) == exp["row_fnv1a"]
    assert nps.fnv1a(g.col.view(np.uint32)) == exp["col_fnv1a"]
    assert nps.fnv1a(g.w) == exp["w_fnv1a"]


def test_convertcsr_keeps_reverse_insertion_order(nps):
    # convertCSR pops adjacency lists from the back (global.cpp:216-220)
    g = nps.convertCSR(3, [0, 0, 1, 0], [1, 2, 2, 0], [5, 6, 7, 8])
    assert g.row_ptr.tolist() == [0, 3, 4, 4]
    assert g.col.tolist() == [0, 2, 1, 2]
    assert g.w.tolist() == [8, 6, 5, 7]


def test_dedupe_keeps_first_and_drops_self_loops(nps):
    g = nps.convertCSR(3, [0, 0, 0, 1, 1], [1, 1, 0, 2, 2], [9, 3, 4, 5, 6], dedupe=True, drop_self_loops=True)
    assert g.row_ptr.tolist() == [0, 1, 2, 2]
    assert g.col.tolist() == [1, 2] and g.w.tolist() == [9, 5]


def test_dimacs9_round_trip(nps, tmp_path):
    for g in (nps.gen_rmat(10, 8, seed=2), nps.gen_grid(20, 30, 0.1, 1000, 4), nps.gen_uniform(300, 2000, 7, 5)):
        p = tmp_path / "g.gr"
        nps.writeDIMACS9(str(p), g, source=min(5, g.n - 1))
        h = nps.readInputDIMACS9(str(p))
        assert h.source == min(5, g.n - 1)
        for a, b in ((g.row_ptr, h.row_ptr), (g.col, h.col), (g.w, h.w)):
            assert np.array_equal(a, b)


def test_dimacs9_round_trip_through_the_reference_reader(nps, oracle, tmp_path):
    if not oracle.have_reference():
        pytest.skip("reference CPU code not built")
    g = nps.gen_rmat(11, 16, seed=8)
    p = tmp_path / "g.gr"
    nps.writeDIMACS9(str(p), g)
    row, col, w, src = oracle.ref_read_graph(str(p), 0)
    assert np.array_equal(row, g.row_ptr) and np.array_equal(col, g.col) and np.array_equal(w, g.w)
    assert src == g.source


def test_generators_are_seeded_and_thread_independent(nps):
    a, b = nps.gen_rmat(12, 16, seed=4), nps.gen_rmat(12, 16, seed=4)
    assert np.array_equal(a.col, b.col) and np.array_equal(a.w, b.w)
    c = nps.gen_rmat(12, 16, seed=5)
    assert not np.array_equal(a.col[: min(a.m, c.m)], c.col[: min(a.m, c.m)])
    assert a.source == int(np.argmax(np.diff(a.row_ptr)))


def test_rmat_has_no_duplicates_or_self_loops(nps):
    g = nps.gen_rmat(11, 16, seed=3)
    for v in range(g.n):
        row = g.col[g.row_ptr[v]: g.row_ptr[v + 1]]
        assert v not in row
        assert len(set(row.tolist())) == len(row)
    assert g.w.min() >= 1 and g.w.max() <= 255


def test_uniform_has_no_self_loops_and_exact_edge_count(nps):
    g = nps.gen_uniform(16384, 131072, 100, 1)
    assert g.m == 131072
    src = np.repeat(np.arange(g.n), np.diff(g.row_ptr))
    assert not np.any(src == g.col)
    assert g.w.min() >= 1 and g.w.max() <= 100


def test_grid_shape_and_drop_rate(nps):
    g = nps.gen_grid(64, 64, 0.05, 1000, 1)
    pairs = 64 * 63 * 2
    kept = g.m // 2
    assert 0.9 * pairs <= kept <= pairs
    src = np.repeat(np.arange(g.n), np.diff(g.row_ptr))
    dr, dc = np.abs(src // 64 - g.col // 64), np.abs(src % 64 - g.col % 64)
    assert np.all(dr + dc == 1)


@pytest.mark.parametrize("content,fn", [
    ("p sp 3\n", "readInputDIMACS9"),
    ("p sp 2 1\na 1 5 3\n", "readInputDIMACS9"),
    ("2 5\n2\n1\n", "readInputDIMACS10"),
    ("# a\n# b\n# Nodes: 2 Edges: 1\n# c\n0 9\n", "readInputSLNDC"),
])
def test_malformed_files_raise(nps, tmp_path, content, fn):
    p = tmp_path / "bad.txt"
    p.write_text(content)
    with pytest.raises(nps.NpsError) as ei:
        getattr(nps, fn)(str(p))
    assert ei.value.status == 7  # NPS_ERR_FORMAT


def test_missing_file_raises_io(nps, tmp_path):
    with pytest.raises(nps.NpsError) as ei:
        nps.readInputDIMACS9(str(tmp_path / "nope.gr"))
    assert ei.value.status == 6


@pytest.mark.parametrize("call", [
    lambda nps: nps.gen_uniform(1, 10),
    lambda nps: nps.gen_rmat(0, 16),
    lambda nps: nps.gen_rmat(10, 16, a=0.9, b=0.2, c=0.2),
    lambda nps: nps.gen_grid(0, 5),
    lambda nps: nps.convertCSR(3, [0, 5], [1, 1], [1, 1]),
])
def test_invalid_generator_arguments(nps, call):
    with pytest.raises(nps.NpsError):
        call(nps)
