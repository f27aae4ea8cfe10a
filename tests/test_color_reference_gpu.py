"""Graph coloring against the reference's own program, run on the GPU.

oracle/_ref/gpu-graph-color is the reference's gpu-graph-color built from its
sources (apps/graph-color/src/gpu) by oracle/Makefile.  `-s 0` colors the graph
with gclr_nopruning_gpu() -- one gclr_bitmap_kernel launch per color
(graph_color_wrapper.cu:113-130, graph_color_kernel.cu:14-35) -- and the hook of
oracle/ref_gclr_hook.cpp writes every vertex's color to a file.  The library's nps_color and the oracle's closed form must both
equal it, vertex for vertex.
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "gpu-graph-color")
GOLDEN = os.path.join(ROOT, "tests", "golden")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(BIN), reason="the reference's gpu-graph-color was not built")]


def _reference_colors(path, fmt, tmp):
    out = os.path.join(tmp, "colors.bin")
    r = subprocess.run([BIN, "-s", "0", "-f", str(fmt), "-i", path], capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, NPS_REF_COLORS=out))
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return np.fromfile(out, dtype=np.int32)


@pytest.mark.parametrize("name,fmt,reader", [("reader_dimacs9.gr", 0, "readInputDIMACS9"),
                                             ("reader_dimacs10.graph", 1, "readInputDIMACS10"),
                                             ("reader_slndc.txt", 2, "readInputSLNDC")])
def test_colors_equal_the_reference_program_on_golden_files(nps, oracle, cuda_device, tmp_path, name, fmt, reader):
    path = os.path.join(GOLDEN, name)
    g = getattr(nps, reader)(path)
    want = _reference_colors(path, fmt, str(tmp_path))
    got, st = nps.color(g)
    assert np.array_equal(got, want)
    assert st.iterations == int(want.max())
    assert np.array_equal(oracle.color(g.row_ptr, g.col)[0], want)


@pytest.mark.parametrize("kind", ["rmat", "uniform", "grid"])
def test_colors_equal_the_reference_program_on_generated_graphs(nps, oracle, cuda_device, tmp_path, kind):
    g = {"rmat": lambda: nps.gen_rmat(15, 16, seed=9), "uniform": lambda: nps.gen_uniform(20000, 160000, 10, 4),
         "grid": lambda: nps.gen_grid(150, 150, 0.05, 10, 3)}[kind]()
    path = str(tmp_path / f"{kind}.gr")
    nps.writeDIMACS9(path, g)
    h = nps.readInputDIMACS9(path)
    want = _reference_colors(path, 0, str(tmp_path))
    got, _ = nps.color(h)
    assert np.array_equal(got, want)
    assert np.array_equal(oracle.color(h.row_ptr, h.col)[0], want)
