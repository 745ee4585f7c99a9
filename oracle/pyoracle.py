"""ctypes wrapper of the C oracle (oracle/usap_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py``, as the reference the CUDA path is
compared against.  The product path never loads it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Callable, List, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle_usap.so")

i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
u32p = C.POINTER(C.c_uint32)
f32p = C.POINTER(C.c_float)


class OgGraph(C.Structure):
    _fields_ = [("n", C.c_int32), ("e", C.c_int64),
                ("src", i32p), ("dst", i32p), ("w", i32p),
                ("out_ptr", i64p), ("in_ptr", i64p),
                ("out_idx", i32p), ("out_w", i32p),
                ("in_idx", i32p), ("in_w", i32p),
                ("kout", i64p), ("kin", i64p),
                ("wtot", C.c_int64), ("logk", C.POINTER(C.c_double))]


class OgBlocks(C.Structure):
    _fields_ = [("B", C.c_int32), ("M", i64p), ("dout", i64p), ("din", i64p)]


class OgParams(C.Structure):
    _fields_ = [("num_agg_proposals_per_block", C.c_int32),
                ("num_block_reduction_rate", C.c_float),
                ("max_num_nodal_itr", C.c_int32),
                ("num_batch_nodal_update", C.c_int32),
                ("delta_entropy_threshold1", C.c_double),
                ("delta_entropy_threshold2", C.c_double),
                ("delta_entropy_moving_avg_window", C.c_int32),
                ("dfs_depth", C.c_int32),
                ("seed", C.c_uint64),
                ("init_mode", C.c_int32),
                ("precision", C.c_int32)]


class OgTraceEvent(C.Structure):
    _fields_ = [("kind", C.c_int32), ("stage", C.c_int32), ("itr", C.c_int32),
                ("batch_beg", C.c_int32), ("B", C.c_int32), ("S_q", C.c_int64),
                ("S_ninf", C.c_int32), ("cum_q", C.c_int64), ("cum_ninf", C.c_int32),
                ("moves", C.c_int64), ("h_part", C.c_uint64), ("h_M", C.c_uint64),
                ("h_deg", C.c_uint64)]


class OgResult(C.Structure):
    _fields_ = [("B", C.c_int32), ("S_q", C.c_int64), ("S", C.c_double), ("stages", C.c_int32),
                ("sweeps", C.c_int64), ("batches", C.c_int64),
                ("nodal_proposals", C.c_int64), ("nodal_moves", C.c_int64),
                ("near_threshold", C.c_int64), ("merge_shortfall", C.c_int64)]


class OgScores(C.Structure):
    _fields_ = [(k, C.c_double) for k in (
        "rand_index", "adjusted_rand_index", "pairwise_recall", "pairwise_precision",
        "h_truth", "h_given", "h_truth_given", "h_given_truth", "mi", "nmi", "nmi_sqrt",
        "missed_info", "erroneous_info", "adjusted_rand_index_exact")] + [
        ("n", C.c_int64), ("b_truth", C.c_int64),
                                             ("b_given", C.c_int64)]


class OgGPoint(C.Structure):
    _fields_ = [("B", C.c_int32), ("S", C.c_double), ("S_q", C.c_int64), ("finite", C.c_int32),
                ("slot", C.c_int32)]


class OgFSum(C.Structure):
    _fields_ = [("s", C.c_double), ("c", C.c_double), ("abs", C.c_double), ("n", C.c_int64),
                ("mode", C.c_int32)]


class OgGolden(C.Structure):
    _fields_ = [("large", OgGPoint), ("med", OgGPoint), ("small", OgGPoint)]


TRACE_FN = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(OgTraceEvent))

_lib = None


def build() -> None:
    """Compile the oracle library (make -C oracle oracle)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.og_philox4x32_10.argtypes = [u32p, u32p, u32p]
        L.og_draw_below.argtypes = [C.c_uint32, C.c_int64]
        L.og_draw_below.restype = C.c_uint32
        L.og_graph_init.argtypes = [C.POINTER(OgGraph), C.c_int32, C.c_int64, i32p, i32p, i32p]
        L.og_graph_free.argtypes = [C.POINTER(OgGraph)]
        L.og_scc.argtypes = [C.POINTER(OgGraph), C.c_int32, i32p]
        L.og_scc.restype = C.c_int32
        L.og_blocks_alloc.argtypes = [C.POINTER(OgBlocks), C.c_int32]
        L.og_blocks_free.argtypes = [C.POINTER(OgBlocks)]
        L.og_build.argtypes = [C.POINTER(OgGraph), i32p, C.POINTER(OgBlocks)]
        L.og_quantize.argtypes = [C.c_double]
        L.og_quantize.restype = C.c_int64
        L.og_model_S.argtypes = [C.c_int64, C.c_int64, C.c_int32]
        L.og_model_S.restype = C.c_double
        L.og_entropy_q.argtypes = [C.POINTER(OgGraph), C.POINTER(OgBlocks)]
        L.og_entropy_q.restype = C.c_int64
        L.og_merge_dq.argtypes = [C.POINTER(OgGraph), C.POINTER(OgBlocks), C.c_int32, C.c_int32]
        L.og_merge_dq.restype = C.c_int64
        L.og_nodal_dq.argtypes = [C.POINTER(OgGraph), i32p, C.POINTER(OgBlocks), C.c_int32,
                                  C.c_int32, i32p]
        L.og_nodal_dq.restype = C.c_int64
        L.og_merge_dq_f32.argtypes = [C.POINTER(OgGraph), C.POINTER(OgBlocks), C.c_int32, C.c_int32,
                                      C.c_int32, C.POINTER(OgFSum)]
        L.og_merge_dq_f32.restype = C.c_int64
        L.og_nodal_dq_f32.argtypes = [C.POINTER(OgGraph), i32p, C.POINTER(OgBlocks), C.c_int32,
                                      C.c_int32, C.c_int32, i32p, C.POINTER(OgFSum)]
        L.og_nodal_dq_f32.restype = C.c_int64
        L.og_merge_propose.argtypes = [C.POINTER(OgGraph), C.POINTER(OgBlocks), C.c_int32,
                                       C.c_int32, C.c_int32, C.c_uint64]
        L.og_merge_propose.restype = C.c_int32
        L.og_nodal_propose.argtypes = [C.POINTER(OgGraph), i32p, C.POINTER(OgBlocks), C.c_int32,
                                       C.c_int32, C.c_int32, C.c_uint64]
        L.og_nodal_propose.restype = C.c_int32
        L.og_merge_phase.argtypes = [C.POINTER(OgGraph), C.POINTER(OgBlocks), C.c_int32,
                                     C.c_int32, C.c_uint64, i32p, i64p]
        L.og_merge_apply.argtypes = [C.c_int32, i32p, C.c_int32, i32p, i64p, C.c_int32, i32p]
        L.og_merge_apply.restype = C.c_int32
        L.og_nodal_batch.argtypes = [C.POINTER(OgGraph), i32p, C.POINTER(OgBlocks), C.c_int32,
                                     C.c_int32, C.c_int32, C.c_int32, C.c_uint64, i32p, i64p,
                                     i32p, i64p, i32p, i64p]
        L.og_nodal_batch.restype = C.c_int64
        L.og_nodal_batch_p.argtypes = [C.POINTER(OgGraph), i32p, C.POINTER(OgBlocks), C.c_int32,
                                       C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.c_int32, i32p,
                                       i64p, i32p, f32p, i64p, i32p, i64p]
        L.og_nodal_batch_p.restype = C.c_int64
        L.og_log_f32.argtypes = [C.c_float]
        L.og_log_f32.restype = C.c_float
        L.og_nodal_ds_ref32.argtypes = [C.POINTER(OgGraph), i32p, C.POINTER(OgBlocks), C.c_int32,
                                        C.c_int32]
        L.og_nodal_ds_ref32.restype = C.c_float
        L.og_golden_init.argtypes = [C.POINTER(OgGolden)]
        L.og_golden_step.argtypes = [C.POINTER(OgGolden), C.c_int32, C.c_double, C.c_int64, C.c_int32,
                                     C.c_float, i32p, i32p, i32p]
        L.og_golden_step.restype = C.c_int
        L.og_params_default.argtypes = [C.POINTER(OgParams)]
        L.og_partition.argtypes = [C.POINTER(OgGraph), C.POINTER(OgParams), i32p,
                                   C.POINTER(OgResult), TRACE_FN, C.c_void_p]
        L.og_partition.restype = C.c_int
        L.og_partition_from.argtypes = [C.POINTER(OgGraph), C.POINTER(OgParams), i32p, i32p,
                                        C.POINTER(OgResult), TRACE_FN, C.c_void_p]
        L.og_partition_from.restype = C.c_int
        L.og_hash_part.argtypes = [i32p, C.c_int32]
        L.og_hash_part.restype = C.c_uint64
        L.og_evaluate.argtypes = [i32p, i32p, C.c_int64, C.POINTER(OgScores)]
        L.og_evaluate.restype = C.c_int
        _lib = L
    return _lib


def _p32(a: np.ndarray):
    return a.ctypes.data_as(i32p)


def _p64(a: np.ndarray):
    return a.ctypes.data_as(i64p)


def philox(ctr, key) -> List[int]:
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().og_philox4x32_10(c, k, o)
    return list(o)


class OracleGraph:
    """Owns an og_graph built from 0-based edge arrays (file order)."""

    def __init__(self, n: int, src: np.ndarray, dst: np.ndarray, w: Optional[np.ndarray] = None):
        self.n = int(n)
        self._src = np.ascontiguousarray(src, dtype=np.int32)
        self._dst = np.ascontiguousarray(dst, dtype=np.int32)
        self._w = None if w is None else np.ascontiguousarray(w, dtype=np.int32)
        self.g = OgGraph()
        rc = lib().og_graph_init(C.byref(self.g), self.n, int(self._src.size), _p32(self._src),
                                 _p32(self._dst), None if self._w is None else _p32(self._w))
        if rc != 0:
            raise ValueError(f"og_graph_init failed ({rc})")

    def __del__(self):
        try:
            lib().og_graph_free(C.byref(self.g))
        except Exception:
            pass

    @property
    def e(self) -> int:
        return int(self.g.e)

    def scc(self, dfs_depth: int = 20):
        part = np.empty(self.n, np.int32)
        B = lib().og_scc(C.byref(self.g), dfs_depth, _p32(part))
        return int(B), part

    def blocks(self, part: np.ndarray, B: int) -> "OracleBlocks":
        return OracleBlocks(self, part, B)

    def partition(self, params: Optional[dict] = None, trace: bool = False, init=None):
        """The whole solve; ``init`` (n labels) starts it from that partition
        instead of the SCC pass."""
        p = OgParams()
        lib().og_params_default(C.byref(p))
        for k, v in (params or {}).items():
            setattr(p, k, v)
        part = np.empty(self.n, np.int32)
        res = OgResult()
        events = []

        def cb(_user, ev):
            e = ev.contents
            events.append({f: getattr(e, f) for f, _ in OgTraceEvent._fields_})

        fn = TRACE_FN(cb) if trace else TRACE_FN()
        if init is None:
            rc = lib().og_partition(C.byref(self.g), C.byref(p), _p32(part), C.byref(res), fn, None)
        else:
            ini = np.ascontiguousarray(init, dtype=np.int32)
            rc = lib().og_partition_from(C.byref(self.g), C.byref(p), _p32(ini), _p32(part), C.byref(res), fn,
                                         None)
        if rc != 0:
            raise RuntimeError(f"og_partition failed ({rc})")
        out = {f: getattr(res, f) for f, _ in OgResult._fields_}
        return part, out, events


class OracleBlocks:
    """Dense interblock counts M and degrees for one partition."""

    def __init__(self, g: OracleGraph, part: np.ndarray, B: int):
        self.g = g
        self.part = np.ascontiguousarray(part, dtype=np.int32).copy()
        self.b = OgBlocks()
        if lib().og_blocks_alloc(C.byref(self.b), int(B)) != 0:
            raise MemoryError
        lib().og_build(C.byref(g.g), _p32(self.part), C.byref(self.b))

    def __del__(self):
        try:
            lib().og_blocks_free(C.byref(self.b))
        except Exception:
            pass

    @property
    def B(self) -> int:
        return int(self.b.B)

    def M(self) -> np.ndarray:
        B = self.B
        return np.ctypeslib.as_array(self.b.M, shape=(B * B,)).reshape(B, B).copy()

    def dout(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.b.dout, shape=(self.B,)).copy()

    def din(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.b.din, shape=(self.B,)).copy()

    def entropy_q(self) -> int:
        return int(lib().og_entropy_q(C.byref(self.g.g), C.byref(self.b)))

    def merge_dq(self, r: int, s: int) -> int:
        return int(lib().og_merge_dq(C.byref(self.g.g), C.byref(self.b), r, s))

    def nodal_dq(self, v: int, s: int):
        ninf = C.c_int32(0)
        q = lib().og_nodal_dq(C.byref(self.g.g), _p32(self.part), C.byref(self.b), v, s,
                              C.byref(ninf))
        return int(q), int(ninf.value)

    def merge_dq_f32(self, r: int, s: int, mode: int = 1):
        """exact dS (Q32) and the sum of the FP32 terms of precision `mode`
        (1: float pairs, 2: plain floats): (q, value, sum |term|, terms)"""
        f = OgFSum()
        q = lib().og_merge_dq_f32(C.byref(self.g.g), C.byref(self.b), r, s, mode, C.byref(f))
        return int(q), f.s + f.c, f.abs, int(f.n)

    def nodal_dq_f32(self, v: int, s: int, mode: int = 1):
        """exact dS (Q32), -inf flag and the sum of the FP32 terms of precision
        `mode`: (q, ninf, value, sum |term|, terms)"""
        ninf = C.c_int32(0)
        f = OgFSum()
        q = lib().og_nodal_dq_f32(C.byref(self.g.g), _p32(self.part), C.byref(self.b), v, s, mode,
                                  C.byref(ninf), C.byref(f))
        return int(q), int(ninf.value), f.s + f.c, f.abs, int(f.n)

    def merge_propose(self, r: int, k: int, stage: int, seed: int) -> int:
        return int(lib().og_merge_propose(C.byref(self.g.g), C.byref(self.b), r, k, stage, seed))

    def nodal_propose(self, v: int, itr: int, stage: int, seed: int) -> int:
        return int(lib().og_nodal_propose(C.byref(self.g.g), _p32(self.part), C.byref(self.b),
                                          v, itr, stage, seed))

    def merge_phase(self, K: int, stage: int, seed: int):
        best_s = np.empty(self.B, np.int32)
        best_q = np.empty(self.B, np.int64)
        lib().og_merge_phase(C.byref(self.g.g), C.byref(self.b), K, stage, seed,
                             _p32(best_s), _p64(best_q))
        return best_s, best_q

    def nodal_ds_ref32(self, v: int, s: int) -> float:
        """The reference's float nodal dS (precision mode 3) of v moving to s."""
        return float(lib().og_nodal_ds_ref32(C.byref(self.g.g), _p32(self.part), C.byref(self.b), v, s))

    def nodal_batch(self, beg: int, end: int, itr: int, stage: int, seed: int, precision: int = 0):
        """Runs one batch in place; returns per-vertex proposals and totals."""
        cnt = end - beg
        ps = np.empty(cnt, np.int32)
        pq = np.empty(cnt, np.int64)
        pn = np.empty(cnt, np.int32)
        pf = np.empty(cnt, np.float32)
        cum_q = C.c_int64(0)
        cum_n = C.c_int32(0)
        near = C.c_int64(0)
        moves = lib().og_nodal_batch_p(C.byref(self.g.g), _p32(self.part), C.byref(self.b), beg,
                                       end, itr, stage, seed, precision, _p32(ps), _p64(pq), _p32(pn),
                                       pf.ctypes.data_as(f32p), C.byref(cum_q), C.byref(cum_n),
                                       C.byref(near))
        return {"prop_s": ps, "prop_q": pq, "prop_ninf": pn, "prop_f": pf, "moves": int(moves),
                "cum_q": int(cum_q.value), "cum_ninf": int(cum_n.value),
                "near": int(near.value)}


def merge_apply(part: np.ndarray, B: int, best_s: np.ndarray, best_q: np.ndarray,
                b_to_merge: int):
    part = np.ascontiguousarray(part, dtype=np.int32).copy()
    best_s = np.ascontiguousarray(best_s, dtype=np.int32)
    best_q = np.ascontiguousarray(best_q, dtype=np.int64)
    merged = C.c_int32(0)
    newB = lib().og_merge_apply(int(part.size), _p32(part), int(B), _p32(best_s), _p64(best_q),
                                int(b_to_merge), C.byref(merged))
    return part, int(newB), int(merged.value)


def golden_sequence(seq, rate: float = 0.5):
    """Feeds (B, S) points through og_golden_step, as the states that finish
    successive nodal phases.  Returns rows (done, large.B, med.B, small.B,
    B to continue from, merges to do next), the reference's own printout."""
    gs = OgGolden()
    lib().og_golden_init(C.byref(gs))
    for pt in (gs.large, gs.med, gs.small):
        pt.slot = -1
    rows = []
    slot = 0
    for B, S in seq:
        restore = C.c_int32(-1)
        btm = C.c_int32(0)
        freed = C.c_int32(-1)
        done = lib().og_golden_step(C.byref(gs), int(B), float(S), quantize(float(S)), slot, rate,
                                    C.byref(restore), C.byref(btm), C.byref(freed))
        if done:
            nextB = gs.med.B
            btm_v = btm.value if not gs.small.finite else 0
        else:
            nextB = gs.large.B if restore.value == gs.large.slot else gs.med.B
            btm_v = btm.value
        rows.append([int(done), gs.large.B, gs.med.B, gs.small.B, nextB, btm_v])
        slot += 1
        if done:
            break
    return rows


def model_S(n: int, e: int, B: int) -> float:
    return float(lib().og_model_S(n, e, B))


def quantize(x: float) -> int:
    return int(lib().og_quantize(x))


def evaluate(truth: np.ndarray, given: np.ndarray) -> dict:
    t = np.ascontiguousarray(truth, dtype=np.int32)
    g = np.ascontiguousarray(given, dtype=np.int32)
    s = OgScores()
    rc = lib().og_evaluate(_p32(t), _p32(g), int(t.size), C.byref(s))
    if rc != 0:
        raise ValueError("og_evaluate failed")
    return {f: getattr(s, f) for f, _ in OgScores._fields_}
