"""ctypes binding of the C ABI (include/usap.h, usap_b200/libusap_b200.so).

The library is built in-tree (``make -C usap_b200/csrc``); there is no CPU
fallback: loading fails loudly if the shared library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libusap_b200.so")

i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)

USAP_OK = 0
ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "out of memory", -4: "size limit",
          -5: "no sm_100 device", -6: "internal error", -7: "bad call order"}


class UsapError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"usap error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class Graph(C.Structure):
    _fields_ = [("n", C.c_int32), ("e", C.c_int64), ("src", i32p), ("dst", i32p),
                ("weight", i32p), ("one_based", C.c_int32)]


class Params(C.Structure):
    _fields_ = [("beta", C.c_int32), ("block_size", C.c_int32),
                ("num_agg_proposals_per_block", C.c_int32),
                ("num_block_reduction_rate", C.c_float), ("max_num_nodal_itr", C.c_int32),
                ("num_batch_nodal_update", C.c_int32), ("delta_entropy_threshold1", C.c_double),
                ("delta_entropy_threshold2", C.c_double),
                ("delta_entropy_moving_avg_window", C.c_int32), ("verbose", C.c_int32),
                ("dfs_depth", C.c_int32), ("t_block_num", C.c_int32), ("seed", C.c_uint64),
                ("init_mode", C.c_int32), ("dense_max", C.c_int32), ("device", C.c_int32),
                ("stats", C.c_int32), ("trace_kinds", C.c_int32), ("sweep_graphs", C.c_int32),
                ("persistent", C.c_int32), ("persistent_ctas", C.c_int32),
                ("precision", C.c_int32), ("fp64_shadow", C.c_int32)]


class Result(C.Structure):
    _fields_ = [("B", C.c_int32), ("stages", C.c_int32), ("S", C.c_double), ("S_q", C.c_int64),
                ("sweeps", C.c_int64), ("batches", C.c_int64), ("nodal_proposals", C.c_int64),
                ("nodal_moves", C.c_int64), ("near_threshold", C.c_int64),
                ("merge_shortfall", C.c_int64), ("edge_visits", C.c_int64),
                ("ms_total", C.c_double), ("ms_init", C.c_double), ("ms_merge", C.c_double),
                ("ms_nodal", C.c_double), ("ms_h2d", C.c_double), ("ms_d2h", C.c_double),
                ("ms_nodal_kernel", C.c_double), ("nodal_kernel_launches", C.c_int64),
                ("nodal_kernel_bytes", C.c_double), ("kernel_launches", C.c_int64),
                ("cub_calls", C.c_int64), ("h2d_bytes", C.c_int64), ("d2h_bytes", C.c_int64),
                ("sweep_graph_launches", C.c_int64),
                ("fp32_nodal_evals", C.c_int64), ("fp32_nodal_flips", C.c_int64),
                ("fp32_merge_evals", C.c_int64), ("fp32_merge_flips", C.c_int64),
                ("fp32_order_flips", C.c_int64), ("fp32_flip_rate", C.c_double),
                ("fp32_err_max", C.c_double), ("fp32_err_mean", C.c_double),
                ("apply_scans", C.c_int64), ("B_init", C.c_int64)]


class Scores(C.Structure):
    _fields_ = [(k, C.c_double) for k in (
        "accuracy", "rand_index", "adjusted_rand_index", "adjusted_rand_index_exact",
        "pairwise_recall", "pairwise_precision", "h_truth", "h_given", "h_truth_given",
        "h_given_truth", "mi", "nmi", "nmi_sqrt", "missed_info", "erroneous_info")] + [
        ("n", C.c_int64), ("b_truth", C.c_int64), ("b_given", C.c_int64)]


class TraceEvent(C.Structure):
    _fields_ = [("kind", C.c_int32), ("stage", C.c_int32), ("itr", C.c_int32),
                ("batch_beg", C.c_int32), ("B", C.c_int32), ("S_q", C.c_int64),
                ("S_ninf", C.c_int32), ("cum_q", C.c_int64), ("cum_ninf", C.c_int32),
                ("moves", C.c_int64), ("h_part", C.c_uint64), ("h_M", C.c_uint64),
                ("h_deg", C.c_uint64)]


TRACE_FN = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(TraceEvent))


class BatchJob(C.Structure):
    _fields_ = [("graph", C.c_int32), ("seed", C.c_uint64), ("out_assign", i32p),
                ("result", Result), ("status", C.c_int32)]


class BatchStats(C.Structure):
    _fields_ = [("ms_total", C.c_double), ("ms_load", C.c_double), ("workers", C.c_int32),
                ("kernel_launches", C.c_int64), ("gang_launches", C.c_int64), ("gang_phases", C.c_int64),
                ("ms_gang", C.c_double)]

class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("workers", C.c_int32), ("memory_budget", C.c_int64),
                ("reserved", C.c_int32 * 4)]


class ServerTiming(C.Structure):
    _fields_ = [("ms_queued", C.c_double), ("ms_running", C.c_double), ("ms_latency", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("queued", C.c_int32), ("running", C.c_int32), ("workers", C.c_int32),
                ("peak_running", C.c_int32), ("completed", C.c_int64), ("failed", C.c_int64),
                ("admitted_bytes", C.c_int64), ("peak_admitted_bytes", C.c_int64),
                ("memory_budget", C.c_int64)]


# every exported symbol of include/usap.h
EXPORTS = ("usap_version", "usap_last_error", "usap_params_default", "usap_partition",
           "usap_evaluate", "usap_evaluate_device", "usap_ctx_evaluate", "usap_ctx_create",
           "usap_ctx_destroy", "usap_ctx_load", "usap_ctx_load_tsv", "usap_ctx_add_edges",
           "usap_ctx_partition_from",
           "usap_ctx_num_nodes", "usap_ctx_partition", "usap_ctx_set_trace", "usap_ctx_test_barrier_timeout", "usap_ctx_adjacency", "usap_op_scc",
           "usap_op_build", "usap_op_entropy", "usap_op_merge_phase", "usap_op_merge_apply",
           "usap_op_nodal_batch", "usap_op_merge_phase_prec", "usap_op_nodal_batch_prec",
           "usap_batch_partition", "usap_entropy_static",
           "usap_server_config_default", "usap_server_create", "usap_server_destroy",
           "usap_server_submit", "usap_server_poll", "usap_server_wait", "usap_server_get_stats")

_lib = None


def lib() -> C.CDLL:
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C usap_b200/csrc` "
                          "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    L.usap_version.restype = C.c_char_p
    L.usap_last_error.restype = C.c_char_p
    L.usap_params_default.argtypes = [C.POINTER(Params)]
    L.usap_params_default.restype = None
    L.usap_partition.argtypes = [C.POINTER(Graph), C.POINTER(Params), i32p, C.POINTER(Result)]
    L.usap_evaluate.argtypes = [i32p, i32p, C.c_int64, C.POINTER(Scores)]
    L.usap_evaluate_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.POINTER(Scores)]
    L.usap_ctx_evaluate.argtypes = [C.c_void_p, i32p, C.POINTER(Scores)]
    L.usap_ctx_load_tsv.argtypes = [C.c_void_p, C.c_char_p, C.c_int64, C.c_int32]
    L.usap_ctx_add_edges.argtypes = [C.c_void_p, C.POINTER(Graph)]
    L.usap_ctx_partition_from.argtypes = [C.c_void_p, C.POINTER(Params), i32p, i32p, C.POINTER(Result)]
    L.usap_ctx_create.argtypes = [C.c_int32, C.POINTER(C.c_void_p)]
    L.usap_ctx_destroy.argtypes = [C.c_void_p]
    L.usap_ctx_load.argtypes = [C.c_void_p, C.POINTER(Graph)]
    L.usap_ctx_num_nodes.argtypes = [C.c_void_p, i32p, i64p]
    L.usap_ctx_partition.argtypes = [C.c_void_p, C.POINTER(Params), i32p, C.POINTER(Result)]
    L.usap_ctx_set_trace.argtypes = [C.c_void_p, TRACE_FN, C.c_void_p]
    L.usap_ctx_test_barrier_timeout.argtypes = [C.c_void_p, C.c_int32, C.c_int64]
    L.usap_ctx_adjacency.argtypes = [C.c_void_p] + [i32p] * 8
    L.usap_op_scc.argtypes = [C.c_void_p, C.c_int32, i32p, i32p]
    L.usap_op_build.argtypes = [C.c_void_p, i32p, C.c_int32, C.c_int32, i32p, i32p, i32p]
    L.usap_op_entropy.argtypes = [C.c_void_p, i32p, C.c_int32, C.c_int32, i64p]
    L.usap_op_merge_phase.argtypes = [C.c_void_p, i32p, C.c_int32, C.c_int32, C.c_int32,
                                      C.c_uint64, i32p, i64p, i32p, i64p]
    L.usap_op_merge_apply.argtypes = [C.c_void_p, i32p, C.c_int32, i32p, i64p, C.c_int32,
                                      i32p, i32p]
    L.usap_op_nodal_batch.argtypes = [C.c_void_p, i32p, C.c_int32, C.c_int32, C.c_int32,
                                      C.c_int32, C.c_int32, C.c_int32, C.c_uint64, i32p, i64p,
                                      i32p, i64p, i32p, i64p]
    f64p = C.POINTER(C.c_double)
    L.usap_op_merge_phase_prec.argtypes = [C.c_void_p, i32p, C.c_int32, C.c_int32, C.c_int32,
                                           C.c_uint64, C.c_int32, i32p, i64p, i32p, i64p, f64p, i64p]
    L.usap_op_nodal_batch_prec.argtypes = [C.c_void_p, i32p, C.c_int32, C.c_int32, C.c_int32,
                                           C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.c_int32, i32p,
                                           i64p, f64p, i32p, i64p, i32p, i64p, i64p]
    L.usap_batch_partition.argtypes = [C.POINTER(Graph), C.c_int32, C.POINTER(Params),
                                       C.POINTER(BatchJob), C.c_int32, C.c_int32, C.c_int32,
                                       C.POINTER(BatchStats)]
    L.usap_entropy_static.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32,
                                      C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
    L.usap_server_config_default.argtypes = [C.POINTER(ServerConfig)]
    L.usap_server_config_default.restype = None
    L.usap_server_create.argtypes = [C.POINTER(ServerConfig), C.POINTER(C.c_void_p)]
    L.usap_server_destroy.argtypes = [C.c_void_p]
    L.usap_server_destroy.restype = None
    L.usap_server_submit.argtypes = [C.c_void_p, C.POINTER(Graph), C.POINTER(Params), i32p, i64p]
    L.usap_server_poll.argtypes = [C.c_void_p, C.c_int64, i32p, C.POINTER(Result), C.POINTER(ServerTiming)]
    L.usap_server_wait.argtypes = [C.c_void_p, C.c_int64, C.POINTER(Result), C.POINTER(ServerTiming)]
    L.usap_server_get_stats.argtypes = [C.c_void_p, C.POINTER(ServerStats)]
    for name in EXPORTS:
        fn = getattr(L, name)
        if name.startswith("usap_") and name not in ("usap_version", "usap_last_error",
                                                     "usap_params_default", "usap_server_config_default",
                                                     "usap_server_destroy"):
            fn.restype = C.c_int32
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != USAP_OK:
        raise UsapError(rc, lib().usap_last_error().decode())


def p32(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(i32p)


def p64(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(i64p)


def pf64(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def default_params(**overrides) -> Params:
    p = Params()
    lib().usap_params_default(C.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise AttributeError(f"unknown parameter {k}")
        setattr(p, k, v)
    return p


def make_graph(src: np.ndarray, dst: np.ndarray, weight: Optional[np.ndarray] = None,
               n: int = 0, one_based: bool = False):
    """Returns (Graph struct, keepalive arrays)."""
    s = np.ascontiguousarray(src, dtype=np.int32)
    d = np.ascontiguousarray(dst, dtype=np.int32)
    w = None if weight is None else np.ascontiguousarray(weight, dtype=np.int32)
    g = Graph(n=int(n), e=int(s.size), src=p32(s), dst=p32(d), weight=p32(w),
              one_based=1 if one_based else 0)
    return g, (s, d, w)


def result_dict(r: Result) -> dict:
    return {f: getattr(r, f) for f, _ in Result._fields_}


def scores_dict(s: Scores) -> dict:
    return {f: getattr(s, f) for f, _ in Scores._fields_}
