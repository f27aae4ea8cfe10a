"""Host-side rules of bench.py that its JSON line depends on, checked without a GPU:
the bytes a host-pointer SSSP call moves to the device (the library packs weights
that fit in 8 or 16 bits on graphs of at least 2^20 edges, include/nps.h) and the
workload table the driver's configurations map to."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_host_call_h2d_bytes_follows_the_packing_rule():
    b = _bench()
    n, big, small = 1000, 1 << 20, (1 << 20) - 1
    base = 4 * (n + 1)
    assert b.host_call_h2d_bytes(n, small, 255) == base + 8 * small          # below the minimum: 4-byte weights
    assert b.host_call_h2d_bytes(n, big, 255) == base + 4 * big + big        # 1-byte weights
    assert b.host_call_h2d_bytes(n, big, 256) == base + 4 * big + 2 * big    # 2-byte weights
    assert b.host_call_h2d_bytes(n, big, 65535) == base + 4 * big + 2 * big
    assert b.host_call_h2d_bytes(n, big, 65536) == base + 8 * big            # no packing


def test_workloads_cover_the_configurations():
    b = _bench()
    w = b.WORKLOADS
    assert w["rmat22"][0] == "rmat_eval" and w["rmat22"][1]["seeds"] == tuple(range(1000, 1010))
    assert w["rmat20"][1]["scale"] == 20 and w["grid4096"][1]["rows"] == 4096 and w["uniform16k"][1]["n"] == 16384
    assert "batch64" in w
