"""The drop-in shim inside the reference's own SSSP program.

oracle/Makefile builds the reference's command-line program gpu-sssp from its
sources where they lie: main() in apps/sssp/src/gpu/sssp.cpp:102-156, prepare_gpu()
/ SSSP_GPU() / clean_gpu() in sssp_wrapper.cu:58-149 and :548-583, the readers and
convertCSR() in common/global.cpp:29-235.  Its own sssp_np_consolidate_gpu() is
replaced at link time by compat/sssp_np_consolidate_gpu.cpp on libnps, one binary
per CONSOLIDATE_LEVEL.  `-s 6 -f <format> -i <file>` then takes the reference's
path end to end: the file is read and converted, and SSSP_GPU() runs ten times,
each run after a cudaDeviceReset() in prepare_gpu(), with case 6 reaching the
shim.  The costs of the last run (written by the clear() hook of
oracle/ref_gpu_host_hook.cpp) must equal the CPU oracle's Dijkstra on the same
file, bit for bit.
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
GOLDEN = os.path.join(ROOT, "tests", "golden")
BINS = {lv: os.path.join(REF, f"gpu-sssp-nps-l{lv}") for lv in (0, 1, 2)}
built = pytest.mark.skipif(not all(os.path.exists(b) for b in BINS.values()),
                           reason="the reference's gpu-sssp was not built (needs the reference sources)")


@built
def test_reference_program_links_the_shim():
    """One definition of sssp_np_consolidate_gpu(), the shim's, which calls into libnps."""
    for b in BINS.values():
        syms = subprocess.run(["nm", "-C", b], capture_output=True, text=True, check=True).stdout.splitlines()
        defs = [s for s in syms if s.endswith(" sssp_np_consolidate_gpu()") and " T " in s]
        assert len(defs) == 1
        assert any(s.strip() == "U nps_sssp_state" for s in syms)


def _run(binary, fmt, path, tmp_path):
    out = tmp_path / "costs.bin"
    env = dict(os.environ, NPS_REF_COSTS=str(out))
    r = subprocess.run([binary, "-s", "6", "-f", str(fmt), "-i", path], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "sssp_np_consolidate_gpu:" not in r.stderr, r.stderr[-2000:]  # the shim reports failures there
    return np.fromfile(out, dtype=np.int32).view(np.uint32)


@built
@pytest.mark.gpu
@pytest.mark.parametrize("level", [0, 1, 2])
@pytest.mark.parametrize("name,fmt,reader", [("reader_dimacs9.gr", 0, "readInputDIMACS9"),
                                             ("reader_dimacs10.graph", 1, "readInputDIMACS10"),
                                             ("reader_slndc.txt", 2, "readInputSLNDC")])
def test_reference_program_on_the_golden_files(nps, oracle, cuda_device, tmp_path, level, name, fmt, reader):
    path = os.path.join(GOLDEN, name)
    g = getattr(nps, reader)(path)
    got = _run(BINS[level], fmt, path, tmp_path)
    assert np.array_equal(got, oracle.sssp_heap(g.row_ptr, g.col, g.w, g.source))


@built
@pytest.mark.gpu
@pytest.mark.parametrize("level", [0, 1, 2])
def test_reference_program_on_a_power_law_graph(nps, oracle, cuda_device, tmp_path, level):
    """R-MAT scale 16 written as DIMACS9 and read back by the reference's reader."""
    g = nps.gen_rmat(16, 16, seed=8)
    path = str(tmp_path / "rmat16.gr")
    nps.writeDIMACS9(path, g)
    h = nps.readInputDIMACS9(path)
    got = _run(BINS[level], 0, path, tmp_path)
    assert np.array_equal(got, oracle.sssp_heap(h.row_ptr, h.col, h.w, h.source))


OWN = {lv: os.path.join(REF, f"gpu-sssp-ref-l{lv}") for lv in (0, 1, 2)}


@pytest.mark.gpu
@pytest.mark.skipif(not all(os.path.exists(b) for b in OWN.values()),
                    reason="the reference's gpu-sssp was not built (needs the reference sources)")
@pytest.mark.parametrize("level", [0, 1, 2])
def test_library_equals_the_reference_gpu_kernels_on_the_uniform_graph(nps, oracle, cuda_device, tmp_path, level):
    """The reference's own consolidation kernels (consolidate_{warp,block,grid}_dp_kernel with their
    dynamic-parallelism children, sssp_kernel.cu:330-541, driven by sssp_np_consolidate_gpu(),
    sssp_wrapper.cu:475-546) on the CPU-runnable configuration: 16,384 vertices, 131,072 uniform
    edges, weights in [1, 100], source 0.  At this size every per-warp (256-slot) and per-block
    (2048-slot) slice of the reference's 10.24 M-entry buffer lies inside it (at most 86 blocks of
    192 threads), so the kernels stay in bounds.  The library's distances, the reference kernels'
    and the CPU oracle's must all agree."""
    g = nps.gen_uniform(16384, 131072, 100, 1)
    path = str(tmp_path / "uniform16k.gr")
    nps.writeDIMACS9(path, g)
    h = nps.readInputDIMACS9(path)
    want = oracle.sssp_heap(h.row_ptr, h.col, h.w, h.source)
    ref = _run(OWN[level], 0, path, tmp_path)
    mine, _ = nps.sssp(h, h.source, nps.Params(level=level))
    assert np.array_equal(mine, want)
    assert np.array_equal(ref, want), f"reference kernels: {(ref != want).sum()} mismatches against the oracle"
