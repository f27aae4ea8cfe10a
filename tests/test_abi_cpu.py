"""The C ABI: libnps.so loads, exports every function include/nps.h declares, the
header compiles as C, and calls fail with status codes (never exit) -- CPU only,
no computation on a GPU."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "nps.h")
LIBDIR = os.path.join(ROOT, "nested-parallelism_b200")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nps_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_function_is_exported(nps):
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(nps.lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", os.path.join(LIBDIR, "libnps.so")], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (nps_[a-z0-9_]+)", out))
    assert set(names) <= exported


def test_header_compiles_as_c_and_links(tmp_path):
    src = tmp_path / "abi.c"
    src.write_text('#include "nps.h"\n#include <stdio.h>\n'
                   'int main(void) { nps_params p; nps_params_default(&p);\n'
                   '  printf("%d %d %d %u\\n", nps_abi_version(), p.level, p.threshold, (unsigned)NPS_INF);\n'
                   '  return 0; }\n')
    exe = tmp_path / "abi"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", f"-I{os.path.join(ROOT, 'include')}", str(src), "-o",
                    str(exe), f"-L{LIBDIR}", "-lnps", f"-Wl,-rpath,{LIBDIR}"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    assert out == ["3", "1", "64", str(0x40000000)]  # ABI 3: nps_params grew sort_at_push


def test_params_defaults_match_the_reference_build(nps):
    p = nps.Params().to_c(device_ptrs=False)
    assert p.level == 1       # Makefile: CONSOLIDATE_LEVEL=1 (apps/sssp/src/gpu/Makefile:28)
    assert p.threshold == 64  # THRESHOLD (apps/sssp/src/gpu/sssp_kernel.cu:7)
    assert p.light_heavy == 1 and p.timeout_s == 10.0
    assert nps.INF == 1 << 30


def test_fnv1a_is_the_documented_hash(nps):
    import numpy as np
    h = 1469598103934665603
    for v in (0, 1, 2**30, 7):
        h = ((h ^ v) * 1099511628211) % (1 << 64)
    assert nps.fnv1a(np.array([0, 1, 2**30, 7], np.uint32)) == h


def test_compute_calls_without_a_gpu_return_a_status(nps):
    import torch
    if torch.cuda.is_available():
        pytest.skip("this test is for machines without a GPU")
    g = nps.gen_uniform(100, 500, 10, 1)
    with pytest.raises(nps.NpsError) as ei:
        nps.sssp(g, 0)
    assert ei.value.status == 5  # NPS_ERR_NO_DEVICE: reported, not a crash or exit
    assert "CUDA" in str(ei.value) or "device" in str(ei.value)


def test_solution_arguments_are_checked_before_the_device(nps):
    """nps_sssp_solution rejects bad solutions and parameters with status 1
    before it touches a device."""
    g = nps.gen_uniform(100, 500, 10, 1)
    cases = ((7, {}), (-1, {}), (0, {"block_size": 100}), (1, {"block_size": 32}), (2, {"block_size": 2048}),
             (3, {"threshold": 0}), (4, {"timeout_s": 0.0}))
    for sol, kw in cases:
        with pytest.raises(nps.NpsError) as ei:
            nps.sssp_solution(g, sol, 0, nps.Params(**kw))
        assert ei.value.status == 1, (sol, kw)
    with pytest.raises(nps.NpsError) as ei:
        nps.sssp_solution(g, 0, g.n)  # source out of range
    assert ei.value.status == 1
    with pytest.raises(nps.NpsError):
        nps.SSSP_GPU(g, solution=9)
