"""ctypes binding of libnps.so (the C ABI declared in include/nps.h).

The shared library is built in-tree by `make -C nested-parallelism_b200`
(or `__graft_entry__.build()`).  There is no fallback implementation: if the
library is missing or cannot be loaded, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnps.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"libnps.so not found at {LIB_PATH}; build it with `make -C {_HERE}` "
        "(the SSSP path has no CPU fallback)")
lib = C.CDLL(LIB_PATH)

NPS_INF = 0x40000000
NPS_MLP_IN, NPS_MLP_HID, NPS_MLP_OUT = 12, 32, 14

STATUS_NAMES = {
    0: "NPS_OK", 1: "NPS_ERR_INVALID_ARG", 2: "NPS_ERR_CUDA", 3: "NPS_ERR_CAPACITY",
    4: "NPS_ERR_TIMEOUT", 5: "NPS_ERR_NO_DEVICE", 6: "NPS_ERR_IO", 7: "NPS_ERR_FORMAT",
    8: "NPS_ERR_OOM", 9: "NPS_ERR_INTERNAL",
}


class nps_params(C.Structure):
    _fields_ = [
        ("level", C.c_int32), ("threshold", C.c_int32), ("block_threshold", C.c_int32),
        ("grid_threshold", C.c_int32), ("block_size", C.c_int32), ("ctas_per_sm", C.c_int32),
        ("delta", C.c_uint32), ("policy", C.c_int32), ("device_ptrs", C.c_int32),
        ("device", C.c_int32), ("stream", C.c_void_p), ("timeout_s", C.c_double),
        ("trace", C.c_int32), ("light_heavy", C.c_int32), ("local_rounds", C.c_int32),
        ("order_degree", C.c_int32), ("delta_schedule", C.c_uint32), ("reserved", C.c_int32 * 2),
        ("schedule", C.c_int32), ("policy_min_edges", C.c_int64), ("sort_at_push", C.c_int32),
        ("reserved2", C.c_int32),
    ]


class nps_stats(C.Structure):
    _fields_ = [
        ("iterations", C.c_uint32), ("buckets", C.c_uint32), ("edges_scanned", C.c_uint64),
        ("improvements", C.c_uint64), ("vertices_processed", C.c_uint64), ("reached", C.c_uint32),
        ("policy_used", C.c_uint32), ("reached_edges", C.c_uint64), ("kernel_ms", C.c_float),
        ("total_ms", C.c_float), ("status", C.c_int32), ("grid_ctas", C.c_int32),
        ("phase_cycles", C.c_uint64 * 9),
    ]


class nps_trace_rec(C.Structure):
    _fields_ = [
        ("iteration", C.c_uint32), ("frontier", C.c_uint32), ("far_len", C.c_uint32),
        ("bucket_hi", C.c_uint32), ("delta", C.c_uint32), ("level", C.c_uint32),
        ("hist", C.c_uint32 * 8), ("edges", C.c_uint64), ("improvements", C.c_uint64),
        ("reached", C.c_uint32), ("heavy", C.c_uint32), ("t_ns", C.c_uint64),
        ("feat", C.c_float * 12),
    ]


class nps_graph(C.Structure):
    _fields_ = [
        ("n", C.c_int32), ("source", C.c_int32), ("m", C.c_int64),
        ("row_ptr", C.POINTER(C.c_int32)), ("col", C.POINTER(C.c_int32)),
        ("w", C.POINTER(C.c_uint32)),
    ]


class nps_instance(C.Structure):
    _fields_ = [
        ("row_ptr", C.c_void_p), ("col", C.c_void_p), ("w", C.c_void_p), ("dist", C.c_void_p),
        ("n", C.c_int32), ("src", C.c_int32), ("m", C.c_int64),
    ]


class nps_degree_info(C.Structure):
    _fields_ = [
        ("n", C.c_int32), ("max_degree", C.c_int32), ("m", C.c_int64), ("total_degree", C.c_int64),
        ("edges_by_degree", C.c_int64), ("min_degree", C.c_int32), ("max_degree_node", C.c_int32),
        ("min_degree_node", C.c_int32), ("avg_degree", C.c_float), ("bins", C.c_int64 * 8),
    ]


class nps_solution_info(C.Structure):
    _fields_ = [
        ("deferred", C.c_uint64), ("child_launches", C.c_uint64), ("launch_fallbacks", C.c_uint64),
        ("host_reads", C.c_uint32), ("pad", C.c_uint32),
    ]


_P = C.c_void_p
_I32, _I64, _U32, _U64, _F, _D = C.c_int32, C.c_int64, C.c_uint32, C.c_uint64, C.c_float, C.c_double

SIGNATURES = {
    "nps_abi_version": (_I32, []),
    "nps_last_error_string": (C.c_char_p, []),
    "nps_params_default": (None, [C.POINTER(nps_params)]),
    "nps_gen_uniform": (_I32, [_I32, _I64, _U32, _U64, C.POINTER(nps_graph)]),
    "nps_gen_rmat": (_I32, [_I32, _I32, _D, _D, _D, _U32, _U64, C.POINTER(nps_graph)]),
    "nps_gen_grid": (_I32, [_I32, _I32, _D, _U32, _U64, C.POINTER(nps_graph)]),
    "nps_csr_from_edges": (_I32, [_I32, _I64, _P, _P, _P, _I32, _I32, C.POINTER(nps_graph)]),
    "nps_graph_free": (None, [C.POINTER(nps_graph)]),
    "nps_fnv1a_u32": (_U64, [_P, _I64]),
    "nps_read_dimacs9": (_I32, [C.c_char_p, C.POINTER(nps_graph)]),
    "nps_read_dimacs10": (_I32, [C.c_char_p, C.POINTER(nps_graph)]),
    "nps_read_slndc": (_I32, [C.c_char_p, C.POINTER(nps_graph)]),
    "nps_write_dimacs9": (_I32, [C.c_char_p, C.POINTER(nps_graph), _I32]),
    "nps_sssp": (_I32, [_P, _P, _P, _I32, _I64, _I32, C.POINTER(nps_params), _P, C.POINTER(nps_stats)]),
    "nps_ctx_create": (_I32, [_I32, C.POINTER(_P)]),
    "nps_ctx_destroy": (_I32, [_P]),
    "nps_sssp_ctx": (_I32, [_P, _P, _P, _P, _I32, _I64, _I32, C.POINTER(nps_params), _P,
                            C.POINTER(nps_stats)]),
    "nps_sssp_state": (_I32, [_P, _P, _P, _I32, _I64, _P, _P, C.POINTER(nps_params),
                              C.POINTER(nps_stats)]),
    "nps_color": (_I32, [_P, _P, _I32, _I64, C.POINTER(nps_params), _P, C.POINTER(nps_stats)]),
    "nps_bc": (_I32, [_P, _P, _I32, _I64, _P, _I32, C.POINTER(nps_params), _P, C.POINTER(nps_stats)]),
    "nps_spmv": (_I32, [_P, _P, _P, _P, _P, _I32, _I64, C.POINTER(nps_params), C.POINTER(nps_stats)]),
    "nps_bfs": (_I32, [_P, _P, _I32, _I64, _I32, C.POINTER(nps_params), _P, C.POINTER(nps_stats)]),
    "nps_sssp_solution": (_I32, [_I32, _P, _P, _P, _I32, _I64, _I32, C.POINTER(nps_params), _P,
                                 C.POINTER(nps_stats), C.POINTER(nps_solution_info)]),
    "nps_sssp_solution_state": (_I32, [_I32, _P, _P, _P, _I32, _I64, _P, _P, C.POINTER(nps_params),
                                       C.POINTER(nps_stats), C.POINTER(nps_solution_info)]),
    "nps_trace_read": (_I32, [_I32, C.POINTER(nps_trace_rec), _I32, C.POINTER(_I32)]),
    "nps_sssp_noalloc": (_I32, [_P, _P, _P, _I32, _I64, _I32, _P, C.POINTER(nps_params), C.POINTER(nps_stats)]),
    "nps_sssp_batch": (_I32, [C.POINTER(nps_instance), _I32, C.POINTER(nps_params), _I32,
                              C.POINTER(nps_stats), C.POINTER(_F)]),
    "nps_degree_stats": (_I32, [_P, _I32, _I32, _I32, C.POINTER(nps_degree_info), _P, _I64]),
    "nps_policy_set_weights": (_I32, [_I32, _P, _P, _P, _P, _P, _P]),
    "nps_mlp_forward": (_I32, [_P, _P, _P, _P, _P, _I32, _P, _P]),
    "nps_mlp_loss_backward": (_I32, [_P, _P, _P, _P, _P, _P, _P, _P, _I32, _P, _P, _P, _P, _P, _P]),
    "nps_mlp_adam_step": (_I32, [_P, _P, _P, _P, _P, _I32, _F, _F, _F, _F, _I32, _P]),
}

for _name, (_res, _args) in SIGNATURES.items():
    _fn = getattr(lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args


class NpsError(RuntimeError):
    """A non-zero nps_status from the library (the reference would have exit()ed)."""

    def __init__(self, status: int, where: str):
        msg = lib.nps_last_error_string().decode(errors="replace")
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def check(status: int, where: str) -> None:
    if status != 0:
        raise NpsError(status, where)
