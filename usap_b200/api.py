"""Python mirror of the reference's interface for the SBP path.

``Graph_P`` keeps the names, defaults and behaviour of uSAP's
``sgp::Graph_P<W>`` (include/graph_parallel.hpp:27-245): construct from a
TSV basename (or from arrays), set the public parameters, call
``partition()``, read ``get_partitions()``; ``evaluate(truth, given)``
returns the scores that ``bf::evaluate`` (include/evaluate.hpp:18-266)
prints.  All work goes through the C ABI to the CUDA library; loading an
unreadable file raises ``OSError`` instead of exiting the process
(the reference calls std::exit, graph_parallel.hpp:254-257).
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, List, Optional

import numpy as np

from . import native as nat
from .generator import Graph as GenGraph
from .generator import read_tsv


class Context:
    """A CUDA device context holding one graph resident in HBM."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        nat.check(nat.lib().usap_ctx_create(int(device), C.byref(h)))
        self._h = h
        self._trace_fn = None
        self.n = 0
        self.e = 0

    def close(self) -> None:
        if self._h:
            nat.lib().usap_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load(self, src, dst, weight=None, n: int = 0, one_based: bool = False) -> None:
        g, keep = nat.make_graph(src, dst, weight, n, one_based)
        nat.check(nat.lib().usap_ctx_load(self._h, C.byref(g)))
        nn = C.c_int32()
        ee = C.c_int64()
        nat.check(nat.lib().usap_ctx_num_nodes(self._h, C.byref(nn), C.byref(ee)))
        self.n, self.e = int(nn.value), int(ee.value)

    def partition(self, params: Optional[nat.Params] = None, want_assign: bool = True):
        p = params if params is not None else nat.default_params()
        out = np.empty(self.n, np.int32) if want_assign else None
        res = nat.Result()
        nat.check(nat.lib().usap_ctx_partition(self._h, C.byref(p), nat.p32(out), C.byref(res)))
        return out, nat.result_dict(res)

    def add_edges(self, src, dst, weight=None, n: int = 0, one_based: bool = False) -> None:
        """Streaming input: append an edge batch to the resident graph
        (usap_ctx_add_edges); n grows to cover the new vertices."""
        g, keep = nat.make_graph(src, dst, weight, n, one_based)
        nat.check(nat.lib().usap_ctx_add_edges(self._h, C.byref(g)))
        nn = C.c_int32()
        ee = C.c_int64()
        nat.check(nat.lib().usap_ctx_num_nodes(self._h, C.byref(nn), C.byref(ee)))
        self.n, self.e = int(nn.value), int(ee.value)

    def partition_from(self, init, params: Optional[nat.Params] = None, want_assign: bool = True):
        """partition() started from ``init`` (one block label >= 0 per vertex)
        instead of the SCC pass (usap_ctx_partition_from)."""
        ini = np.ascontiguousarray(init, np.int32)
        if ini.size != self.n:
            raise ValueError(f"init has {ini.size} labels, the graph {self.n} vertices")
        p = params if params is not None else nat.default_params()
        out = np.empty(self.n, np.int32) if want_assign else None
        res = nat.Result()
        nat.check(nat.lib().usap_ctx_partition_from(self._h, C.byref(p), nat.p32(ini), nat.p32(out), C.byref(res)))
        return out, nat.result_dict(res)

    def load_tsv(self, text: bytes, n: int = 0) -> None:
        """load_graph_from_tsv from the bytes of a reference-format .tsv file,
        parsed on the device (usap_ctx_load_tsv); n = 0: N is the largest
        source id."""
        nat.check(nat.lib().usap_ctx_load_tsv(self._h, text, len(text), int(n)))
        nn = C.c_int32()
        ee = C.c_int64()
        nat.check(nat.lib().usap_ctx_num_nodes(self._h, C.byref(nn), C.byref(ee)))
        self.n, self.e = int(nn.value), int(ee.value)

    def evaluate(self, truth) -> dict:
        """Scores of the last partition() result against ``truth``, computed on
        the device where the result lies (usap_ctx_evaluate)."""
        t = np.ascontiguousarray(truth, np.int32)
        if t.size != self.n:
            raise ValueError(f"truth has {t.size} labels, the graph {self.n} vertices")
        s = nat.Scores()
        nat.check(nat.lib().usap_ctx_evaluate(self._h, nat.p32(t), C.byref(s)))
        return nat.scores_dict(s)

    def adjacency(self) -> dict:
        """The resident graph's out/in lists (file order inside each list),
        weights and weighted degrees (usap_ctx_adjacency)."""
        n, e = self.n, self.e
        out = {k: np.empty(n + 1, np.int32) for k in ("out_ptr", "in_ptr")}
        out.update({k: np.empty(e, np.int32) for k in ("out_idx", "out_w", "in_idx", "in_w")})
        out.update({k: np.empty(n, np.int32) for k in ("kout", "kin")})
        nat.check(nat.lib().usap_ctx_adjacency(self._h, *(nat.p32(out[k]) for k in (
            "out_ptr", "out_idx", "out_w", "in_ptr", "in_idx", "in_w", "kout", "kin"))))
        return out

    def test_barrier_timeout(self, hold_cta: int, timeout_ns: int) -> None:
        """Failure injection: the next cooperative nodal-phase launch has CTA
        ``hold_cta`` withhold its grid-barrier arrivals and waits limited to
        ``timeout_ns``, so that solve raises UsapError(-6)."""
        nat.check(nat.lib().usap_ctx_test_barrier_timeout(self._h, int(hold_cta), int(timeout_ns)))

    def set_trace(self, fn: Optional[Callable[[dict], None]]) -> None:
        if fn is None:
            self._trace_fn = nat.TRACE_FN()
        else:
            def cb(_user, ev):
                e = ev.contents
                fn({f: getattr(e, f) for f, _ in nat.TraceEvent._fields_})
            self._trace_fn = nat.TRACE_FN(cb)
        nat.check(nat.lib().usap_ctx_set_trace(self._h, self._trace_fn, None))

    # --- phase-level replay operations ---
    def op_scc(self, dfs_depth: int = 20):
        part = np.empty(self.n, np.int32)
        B = C.c_int32()
        nat.check(nat.lib().usap_op_scc(self._h, dfs_depth, nat.p32(part), C.byref(B)))
        return int(B.value), part

    def op_build(self, part, B: int, dense_max: int = 4096, want_M: bool = True):
        part = np.ascontiguousarray(part, np.int32)
        M = np.empty((B, B), np.int32) if want_M else None
        dout = np.empty(B, np.int32)
        din = np.empty(B, np.int32)
        nat.check(nat.lib().usap_op_build(self._h, nat.p32(part), B, dense_max, nat.p32(M),
                                          nat.p32(dout), nat.p32(din)))
        return M, dout, din

    def op_entropy(self, part, B: int, dense_max: int = 4096) -> int:
        part = np.ascontiguousarray(part, np.int32)
        S = C.c_int64()
        nat.check(nat.lib().usap_op_entropy(self._h, nat.p32(part), B, dense_max, C.byref(S)))
        return int(S.value)

    def op_merge_phase(self, part, B: int, K: int, stage: int, seed: int, precision: int = 0,
                       dense: bool = False):
        """block_merge task on sorted views; with ``dense`` or a precision mode
        (usap_op_merge_phase_prec) on the path a solve takes, the dense tile
        for B <= 4096, and then also the FP32 dS of every proposal and the
        number of blocks whose choice flipped."""
        part = np.ascontiguousarray(part, np.int32)
        best_s = np.empty(B, np.int32)
        best_q = np.empty(B, np.int64)
        ps = np.empty(B * K, np.int32)
        pq = np.empty(B * K, np.int64)
        if not precision and not dense:
            nat.check(nat.lib().usap_op_merge_phase(self._h, nat.p32(part), B, K, stage, seed,
                                                    nat.p32(best_s), nat.p64(best_q), nat.p32(ps),
                                                    nat.p64(pq)))
            return best_s, best_q, ps.reshape(B, K), pq.reshape(B, K)
        pf = np.empty(B * K, np.float64)
        flips = C.c_int64()
        nat.check(nat.lib().usap_op_merge_phase_prec(self._h, nat.p32(part), B, K, stage, seed, precision,
                                                     nat.p32(best_s), nat.p64(best_q), nat.p32(ps),
                                                     nat.p64(pq), nat.pf64(pf), C.byref(flips)))
        return best_s, best_q, ps.reshape(B, K), pq.reshape(B, K), pf.reshape(B, K), int(flips.value)

    def op_merge_apply(self, part, B: int, best_s, best_q, b_to_merge: int):
        part = np.ascontiguousarray(part, np.int32).copy()
        bs = np.ascontiguousarray(best_s, np.int32)
        bq = np.ascontiguousarray(best_q, np.int64)
        Bn = C.c_int32()
        merged = C.c_int32()
        nat.check(nat.lib().usap_op_merge_apply(self._h, nat.p32(part), B, nat.p32(bs),
                                                nat.p64(bq), b_to_merge, C.byref(Bn),
                                                C.byref(merged)))
        return part, int(Bn.value), int(merged.value)

    def op_nodal_batch(self, part, B: int, beg: int, end: int, itr: int, stage: int, seed: int,
                       dense_max: int = 4096, precision: int = 0):
        """one nodal batch; in precision mode 1, 2 or 3 the accept decisions
        are taken on the FP32 dS (mode 3: the reference's float expression),
        returned as prop_f beside the exact prop_q."""
        part = np.ascontiguousarray(part, np.int32).copy()
        cnt = end - beg
        ps = np.empty(cnt, np.int32)
        pq = np.empty(cnt, np.int64)
        pn = np.empty(cnt, np.int32)
        cq = C.c_int64()
        cn = C.c_int32()
        mv = C.c_int64()
        if not precision:
            nat.check(nat.lib().usap_op_nodal_batch(self._h, nat.p32(part), B, dense_max, beg, end,
                                                    itr, stage, seed, nat.p32(ps), nat.p64(pq),
                                                    nat.p32(pn), C.byref(cq), C.byref(cn),
                                                    C.byref(mv)))
            return part, {"prop_s": ps, "prop_q": pq, "prop_ninf": pn, "cum_q": int(cq.value),
                          "cum_ninf": int(cn.value), "moves": int(mv.value)}
        pf = np.empty(cnt, np.float64)
        flips = C.c_int64()
        nat.check(nat.lib().usap_op_nodal_batch_prec(self._h, nat.p32(part), B, dense_max, beg, end,
                                                     itr, stage, seed, precision, nat.p32(ps), nat.p64(pq),
                                                     nat.pf64(pf), nat.p32(pn), C.byref(cq),
                                                     C.byref(cn), C.byref(mv), C.byref(flips)))
        return part, {"prop_s": ps, "prop_q": pq, "prop_f": pf, "prop_ninf": pn,
                      "cum_q": int(cq.value), "cum_ninf": int(cn.value), "moves": int(mv.value),
                      "flips": int(flips.value)}


def partition(src, dst, weight=None, n: int = 0, one_based: bool = False,
              params: Optional[nat.Params] = None):
    """One-shot solve through ``usap_partition`` (host buffers in and out)."""
    g, keep = nat.make_graph(src, dst, weight, n, one_based)
    nn = n if n > 0 else int(np.max(keep[0])) + (0 if one_based else 1)
    out = np.empty(nn, np.int32)
    res = nat.Result()
    p = params if params is not None else nat.default_params()
    nat.check(nat.lib().usap_partition(C.byref(g), C.byref(p), nat.p32(out), C.byref(res)))
    return out, nat.result_dict(res)


def batch_partition(graphs, seeds_per_graph, params: Optional[nat.Params] = None,
                    workers: int = 0, device: int = 0):
    """Solve many (graph, seed) jobs at once on one GPU (usap_batch_partition).

    ``graphs`` is a list of objects with ``src``, ``dst``, ``weight`` and ``n``
    (e.g. generator.Graph); ``seeds_per_graph`` a list of seed lists (one
    chain per seed).  Returns (jobs, stats): jobs is a list of dicts with
    ``graph``, ``seed``, ``assign`` and ``result`` in submission order."""
    structs, keep = [], []
    for g in graphs:
        gs, k = nat.make_graph(g.src, g.dst, g.weight, g.n)
        structs.append(gs)
        keep.append(k)
    garr = (nat.Graph * len(structs))(*structs)
    outs, meta = [], []
    for gi, seeds in enumerate(seeds_per_graph):
        for sd in seeds:
            outs.append(np.empty(graphs[gi].n, np.int32))
            meta.append((gi, int(sd)))
    jarr = (nat.BatchJob * len(meta))()
    for j, (gi, sd) in enumerate(meta):
        jarr[j].graph = gi
        jarr[j].seed = sd
        jarr[j].out_assign = nat.p32(outs[j])
    st = nat.BatchStats()
    p = params if params is not None else nat.default_params()
    rc = nat.lib().usap_batch_partition(garr, len(structs), C.byref(p), jarr, len(meta),
                                        int(workers), int(device), C.byref(st))
    nat.check(rc)
    jobs = [{"graph": gi, "seed": sd, "assign": outs[j], "result": nat.result_dict(jarr[j].result)}
            for j, (gi, sd) in enumerate(meta)]
    return jobs, {f: getattr(st, f) for f, _ in nat.BatchStats._fields_}


class Server:
    """Partition service on one GPU (usap_server_*): submit requests at any
    time, collect them by ticket.  Requests run concurrently on worker
    threads with their own streams, admitted in arrival order as workers and
    device memory (``memory_budget`` bytes, 0 = 80% of free) free up."""

    def __init__(self, device: int = 0, workers: int = 0, memory_budget: int = 0):
        cfg = nat.ServerConfig()
        nat.lib().usap_server_config_default(C.byref(cfg))
        cfg.device, cfg.workers, cfg.memory_budget = int(device), int(workers), int(memory_budget)
        h = C.c_void_p()
        nat.check(nat.lib().usap_server_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._out = {}

    def submit(self, src, dst, weight=None, n: int = 0, one_based: bool = False,
               params: Optional[nat.Params] = None) -> int:
        g, keep = nat.make_graph(src, dst, weight, n, one_based)
        nn = n if n > 0 else int(np.max(keep[0])) + (0 if one_based else 1)
        out = np.empty(nn, np.int32)
        p = params if params is not None else nat.default_params()
        t = C.c_int64()
        nat.check(nat.lib().usap_server_submit(self._h, C.byref(g), C.byref(p), nat.p32(out), C.byref(t)))
        self._out[int(t.value)] = out
        return int(t.value)

    def _finish(self, ticket, rc, res, tm):
        out = self._out.pop(ticket)
        nat.check(rc)
        timing = {f: getattr(tm, f) for f, _ in nat.ServerTiming._fields_}
        return out, nat.result_dict(res), timing

    def poll(self, ticket: int):
        """None while the request runs, else (assign, result, timing)."""
        done = C.c_int32()
        res, tm = nat.Result(), nat.ServerTiming()
        rc = nat.lib().usap_server_poll(self._h, int(ticket), C.byref(done), C.byref(res), C.byref(tm))
        if rc == 0 and not done.value:
            return None
        if not done.value:
            nat.check(rc)
        return self._finish(int(ticket), rc, res, tm)

    def wait(self, ticket: int):
        res, tm = nat.Result(), nat.ServerTiming()
        rc = nat.lib().usap_server_wait(self._h, int(ticket), C.byref(res), C.byref(tm))
        return self._finish(int(ticket), rc, res, tm)

    def stats(self) -> dict:
        st = nat.ServerStats()
        nat.check(nat.lib().usap_server_get_stats(self._h, C.byref(st)))
        return {f: getattr(st, f) for f, _ in nat.ServerStats._fields_}

    def close(self) -> None:
        if self._h:
            nat.lib().usap_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def evaluate(truth, given) -> dict:
    """bf::evaluate's scores (plus NMI) as a dict instead of printed lines."""
    t = np.ascontiguousarray(truth, np.int32)
    g = np.ascontiguousarray(given, np.int32)
    if t.shape != g.shape:
        raise ValueError("truth and given must have the same length")
    s = nat.Scores()
    nat.check(nat.lib().usap_evaluate(nat.p32(t), nat.p32(g), int(t.size), C.byref(s)))
    return nat.scores_dict(s)


def evaluate_device(truth_ptr: int, given_ptr: int, n: int, device: int = 0) -> dict:
    """usap_evaluate_device: the same scores from device arrays (raw int32
    pointers on ``device``, e.g. a torch CUDA tensor's ``data_ptr()``)."""
    s = nat.Scores()
    nat.check(nat.lib().usap_evaluate_device(C.c_void_p(truth_ptr), C.c_void_p(given_ptr), int(n), int(device),
                                             C.byref(s)))
    return nat.scores_dict(s)


class Graph_P:
    """``sgp::Graph_P<W>``-shaped front end (graph_parallel.hpp:27-82).

    Public parameters carry the reference's names and defaults
    (graph_parallel.hpp:40-52); ``seed``, ``init_mode`` and ``dense_max`` are
    additions of this build.  ``num_threads`` is accepted for signature
    compatibility; the work runs on the GPU.
    """

    def __init__(self, FileName: Optional[str] = None, num_threads: int = 16, *,
                 graph: Optional[GenGraph] = None, device: int = 0):
        if graph is None:
            if FileName is None:
                raise ValueError("need a TSV basename or a graph")
            try:
                graph = read_tsv(FileName)
            except OSError as e:
                raise OSError(f"Unable to open file! ({FileName}.tsv)") from e
        self._g = graph
        defaults = nat.default_params()
        self.beta = defaults.beta
        self.block_size = defaults.block_size
        self.num_agg_proposals_per_block = defaults.num_agg_proposals_per_block
        self.num_block_reduction_rate = defaults.num_block_reduction_rate
        self.max_num_nodal_itr = defaults.max_num_nodal_itr
        self.num_batch_nodal_update = defaults.num_batch_nodal_update
        self.delta_entropy_threshold1 = defaults.delta_entropy_threshold1
        self.delta_entropy_threshold2 = defaults.delta_entropy_threshold2
        self.delta_entropy_moving_avg_window = defaults.delta_entropy_moving_avg_window
        self.verbose = False
        self.dfs_depth = defaults.dfs_depth
        self.t_block_num = defaults.t_block_num
        self.seed = 0
        self.init_mode = 0
        self.dense_max = defaults.dense_max
        self.truePartitions: List[int] = [] if graph.truth is None else graph.truth.tolist()
        self._ctx = Context(device)
        self._ctx.load(graph.src, graph.dst, graph.weight, graph.n)
        self._partitions: Optional[np.ndarray] = None
        self.result: dict = {}

    def num_nodes(self) -> int:
        return self._ctx.n

    def num_edges(self) -> int:
        return self._ctx.e

    def _params(self) -> nat.Params:
        return nat.default_params(
            beta=int(self.beta), block_size=int(self.block_size),
            num_agg_proposals_per_block=int(self.num_agg_proposals_per_block),
            num_block_reduction_rate=float(self.num_block_reduction_rate),
            max_num_nodal_itr=int(self.max_num_nodal_itr),
            num_batch_nodal_update=int(self.num_batch_nodal_update),
            delta_entropy_threshold1=float(self.delta_entropy_threshold1),
            delta_entropy_threshold2=float(self.delta_entropy_threshold2),
            delta_entropy_moving_avg_window=int(self.delta_entropy_moving_avg_window),
            verbose=int(bool(self.verbose)), dfs_depth=int(self.dfs_depth),
            t_block_num=int(self.t_block_num), seed=int(self.seed),
            init_mode=int(self.init_mode), dense_max=int(self.dense_max))

    def partition(self) -> None:
        self._partitions, self.result = self._ctx.partition(self._params())

    def get_partitions(self) -> np.ndarray:
        if self._partitions is None:
            raise RuntimeError("partition() has not been called")
        return self._partitions
