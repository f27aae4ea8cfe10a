"""The drop-in shims linked the way a reference build would link them: a harness
owns the reference's globals and fills them as prepare_gpu() does.
  - `sssp_np_consolidate_gpu()` and the other six cases of SSSP_GPU()'s switch
    (tests/compat/harness.cpp);
  - bfs-rec's `bfs_rec_dp_cons_gpu()` (tests/compat/harness_bfs.cpp);
  - SpMV's, bc's and graph-color's `*_np_consolidate_gpu()` (tests/compat/harness_apps.cpp).
On CPU the shims and harnesses compile and link against libnps for every
CONSOLIDATE_LEVEL; on the GPU the harnesses run and their outputs hash to the
oracle's."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "nested-parallelism_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _build(out, level):
    cmd = ["g++", "-O2", "-std=c++17", f"-DCONSOLIDATE_LEVEL={level}", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "compat", "harness.cpp"),
           os.path.join(PKG, "compat", "sssp_np_consolidate_gpu.cpp"),
           os.path.join(PKG, "compat", "sssp_solutions_gpu.cpp"), "-o", str(out), "-L", PKG, "-lnps",
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{PKG}:{os.path.join(CUDA, 'lib64')}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return str(out)


@pytest.fixture(scope="module")
def harnesses(tmp_path_factory):
    d = tmp_path_factory.mktemp("compat")
    return {lv: _build(d / f"harness_l{lv}", lv) for lv in (0, 1, 2)}


def test_shim_builds_against_reference_globals(harnesses):
    for path in harnesses.values():
        assert os.access(path, os.X_OK)


@pytest.mark.gpu
@pytest.mark.parametrize("level", [0, 1, 2])
@pytest.mark.parametrize("kind,size,seed", [("uniform", 16384, 1), ("rmat", 14, 5)])
def test_shim_matches_the_oracle(nps, oracle, cuda_device, harnesses, level, kind, size, seed):
    r = subprocess.run([harnesses[level], kind, str(size), str(seed)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    f = dict(zip(r.stdout.split()[0::2], r.stdout.split()[1::2]))
    g = nps.gen_rmat(size, 16, seed=seed) if kind == "rmat" else nps.gen_uniform(size, 8 * size, 100, seed)
    ref = oracle.sssp_heap(g.row_ptr, g.col, g.w, g.source)
    assert int(f["status"]) == 0 and int(f["source"]) == g.source
    assert int(f["fnv1a"], 16) == nps.fnv1a(ref)
    assert int(f["update_left"]) == 0 and int(f["iterations"]) > 0


@pytest.mark.gpu
@pytest.mark.parametrize("solution", [0, 1, 2, 3, 4, 5])
def test_solution_shims_match_the_oracle(nps, oracle, cuda_device, harnesses, solution):
    """SSSP_GPU()'s cases 0-5 (sssp_wrapper.cu:554-564) through the drop-in shims."""
    r = subprocess.run([harnesses[1], "rmat", "14", "5", str(solution)], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    f = dict(zip(r.stdout.split()[0::2], r.stdout.split()[1::2]))
    g = nps.gen_rmat(14, 16, seed=5)
    ref = oracle.sssp_heap(g.row_ptr, g.col, g.w, g.source)
    assert int(f["status"]) == 0
    assert int(f["fnv1a"], 16) == nps.fnv1a(ref)
    assert int(f["update_left"]) == 0 and int(f["iterations"]) > 0


def _build_bfs(out, level):
    cmd = ["g++", "-O2", "-std=c++17", f"-DCONSOLIDATE_LEVEL={level}", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "compat", "harness_bfs.cpp"),
           os.path.join(PKG, "compat", "bfs_rec_dp_cons_gpu.cpp"), "-o", str(out), "-L", PKG, "-lnps",
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{PKG}:{os.path.join(CUDA, 'lib64')}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return str(out)


@pytest.fixture(scope="module")
def bfs_harnesses(tmp_path_factory):
    d = tmp_path_factory.mktemp("compat_bfs")
    return {lv: _build_bfs(d / f"harness_bfs_l{lv}", lv) for lv in (0, 1, 2)}


def test_bfs_shim_builds_against_reference_globals(bfs_harnesses):
    for path in bfs_harnesses.values():
        assert os.access(path, os.X_OK)


@pytest.mark.gpu
@pytest.mark.parametrize("level", [0, 1, 2])
@pytest.mark.parametrize("kind,size,seed", [("uniform", 16384, 1), ("rmat", 14, 5)])
def test_bfs_shim_matches_the_oracle(nps, oracle, cuda_device, bfs_harnesses, level, kind, size, seed):
    """bfs_rec_dp_cons_gpu() through the drop-in shim: levels hash to the oracle's."""
    r = subprocess.run([bfs_harnesses[level], kind, str(size), str(seed)], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    f = dict(zip(r.stdout.split()[0::2], r.stdout.split()[1::2]))
    g = nps.gen_rmat(size, 16, seed=seed) if kind == "rmat" else nps.gen_uniform(size, 8 * size, 100, seed)
    ref = oracle.bfs_levels(g.row_ptr, g.col, g.source)
    assert int(f["status"]) == 0 and int(f["source"]) == g.source
    assert int(f["fnv1a"], 16) == nps.fnv1a(ref.view(np.uint32))


@pytest.fixture(scope="module")
def apps_harness(tmp_path_factory):
    out = tmp_path_factory.mktemp("compat_apps") / "harness_apps"
    cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "compat", "harness_apps.cpp"),
           os.path.join(PKG, "compat", "spmv_np_consolidate_gpu.cpp"),
           os.path.join(PKG, "compat", "bc_np_consolidate_gpu.cpp"),
           os.path.join(PKG, "compat", "gclr_np_consolidate_gpu.cpp"), "-o", str(out), "-L", PKG, "-lnps",
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{PKG}:{os.path.join(CUDA, 'lib64')}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return str(out)


def test_app_shims_build_against_reference_globals(apps_harness):
    assert os.access(apps_harness, os.X_OK)


@pytest.mark.gpu
@pytest.mark.parametrize("app", ["spmv", "bc", "color"])
def test_app_shims_match_the_oracle(nps, oracle, cuda_device, apps_harness, app):
    scale = 10 if app == "bc" else 14
    r = subprocess.run([apps_harness, app, str(scale), "5"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    f = dict(zip(r.stdout.split()[0::2], r.stdout.split()[1::2]))
    g = nps.gen_rmat(scale, 16, seed=5)
    if app == "spmv":
        val, x = oracle.spmv_data(g.n, g.m)
        want = oracle.spmv(g.row_ptr, g.col, val, x).view(np.uint32)
    elif app == "bc":
        want = oracle.bc(g.row_ptr, g.col).view(np.uint32)
    else:
        colors, iters = oracle.color(g.row_ptr, g.col)
        want = colors.view(np.uint32)
        assert int(f["iterations"]) == iters
    assert int(f["status"]) == 0
    assert int(f["fnv1a"], 16) == nps.fnv1a(want)
