"""Precision mode 3 (the reference's own float nodal dS) against the oracle,
through the C ABI.

In mode 3 every nodal proposal's dS is evaluated as the reference's
_propose_new_partition_nodal does it (graph_parallel.hpp:1066-1215): float
terms count * log((float)count / (float)(d_a * d_b)) added to one float
accumulator in the reference's order over all B blocks.  The decision is
that float value < 0, and the convergence test sums the accepted float
values, as the reference's update task does.  The kernels and the oracle
use the same log evaluation (log rounded to float, computed in double with
IEEE operations only), so the float dS, every decision and whole solves
must agree bit for bit.
"""
import numpy as np
import pytest

from usap_b200 import generator as gen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    from usap_b200 import api as a
    return a


def _hub_graph(seed=3):
    G = gen.generate(gen.SBMConfig(n=600, blocks=6, within=0.7, alpha=2, seed=seed))
    rng = np.random.default_rng(seed)
    ins = rng.choice(G.n, 320, replace=False)
    outs = rng.choice(G.n, 160, replace=False)
    src = np.concatenate([G.src, ins, np.full(160, 5), [7, 7, 9], G.src[:20]])
    dst = np.concatenate([G.dst, np.full(320, 5), outs, [7, 7, 9], G.dst[:20]])
    return G.n + 2, src.astype(np.int32), dst.astype(np.int32), None


def _weighted_graph(seed=4):
    G = gen.generate(gen.SBMConfig(n=400, blocks=5, within=0.75, alpha=5, seed=seed))
    w = np.random.default_rng(seed).integers(1, 5, G.num_edges).astype(np.int32)
    return G.n, G.src, G.dst, w


GRAPHS = {
    "c0": lambda: (lambda G: (G.n, G.src, G.dst, None))(gen.generate(gen.config_c0())),
    "hub": _hub_graph,
    "weighted": _weighted_graph,
}


@pytest.fixture(scope="module", params=sorted(GRAPHS))
def case(request, api, oracle):
    n, src, dst, w = GRAPHS[request.param]()
    ctx = api.Context(0)
    ctx.load(src, dst, w, n)
    og = oracle.OracleGraph(n, src, dst, w)
    B_scc, part_scc = og.scc(20)
    rng = np.random.default_rng(11)
    part_rand = rng.integers(0, 7, n).astype(np.int32)
    part_rand[:7] = np.arange(7)
    yield request.param, ctx, og, {"scc": (B_scc, part_scc), "rand7": (7, part_rand)}
    ctx.close()


@pytest.mark.parametrize("dense_max", [4096, 1])
def test_ref32_nodal_batch_exact(case, dense_max):
    """One batch from the same state: proposals, exact dS, the float dS of
    every proposal, the decisions (the state after the batch) and the summed
    float values equal the oracle's; on the dense tile and on sorted views."""
    name, ctx, og, states = case
    for sname, (B, part) in states.items():
        n = part.size
        for beg, end, itr, stage, seed in ((0, n, 0, 0, 1), (n // 3, n // 3 + n // 4, 5, 2, 99)):
            gpart, g = ctx.op_nodal_batch(part, B, beg, end, itr, stage, seed, dense_max, precision=3)
            blk = og.blocks(part, B)
            o = blk.nodal_batch(beg, end, itr, stage, seed, precision=3)
            assert np.array_equal(g["prop_s"], o["prop_s"]), (name, sname)
            assert np.array_equal(g["prop_q"], o["prop_q"]), (name, sname)
            f_gpu = g["prop_f"].astype(np.float32)
            assert np.array_equal(g["prop_f"], f_gpu.astype(np.float64)), "prop_f must hold float values"
            proposed = o["prop_s"] >= 0
            assert np.array_equal(f_gpu[proposed], o["prop_f"][proposed]), (name, sname)
            assert g["moves"] == o["moves"] and g["cum_ninf"] == o["cum_ninf"], (name, sname)
            assert g["cum_q"] == o["cum_q"], (name, sname)
            assert np.array_equal(gpart, blk.part), (name, sname)
            # the flip count is the proposals whose float and exact signs differ
            finite = proposed & (o["prop_ninf"] == 0)
            flips = int(np.sum((o["prop_f"][finite] < 0) != (o["prop_q"][finite] < 0)))
            assert g["flips"] == flips, (name, sname)


def _solve_pair(api, oracle, n, src, dst, w, params, persistent=1):
    from usap_b200 import native as nat
    ctx = api.Context(0)
    ctx.load(src, dst, w, n)
    ev_gpu = []
    ctx.set_trace(ev_gpu.append)
    part_g, res_g = ctx.partition(nat.default_params(persistent=persistent, **params))
    ctx.set_trace(None)
    ctx.close()
    og = oracle.OracleGraph(n, src, dst, w)
    oparams = {k: v for k, v in params.items() if k not in ("dense_max", "fp64_shadow")}
    part_o, res_o, ev_o = og.partition(oparams, trace=True)
    return part_g, res_g, ev_gpu, part_o, res_o, ev_o


@pytest.mark.parametrize("graph,params,persistent", [
    ("c0", {"num_batch_nodal_update": 10, "seed": 0}, 1),
    ("c0", {"num_batch_nodal_update": 10, "seed": 0, "fp64_shadow": 1}, 1),
    ("c0", {"num_batch_nodal_update": 10, "seed": 0}, 0),
    ("c0", {"num_batch_nodal_update": 4, "seed": 3, "dense_max": 16}, 1),
    ("weighted", {"num_batch_nodal_update": 7, "seed": 2}, 1),
    ("hub", {"num_batch_nodal_update": 10, "seed": 9}, 1),
    ("hub", {"num_batch_nodal_update": 10, "seed": 9, "fp64_shadow": 1}, 1),
    ("hub", {"num_batch_nodal_update": 10, "seed": 9, "dense_max": 32}, 0),
    ("hub", {"num_batch_nodal_update": 10, "seed": 9, "dense_max": 32, "fp64_shadow": 1}, 0),
])
def test_ref32_full_solve_trace_exact(api, oracle, graph, params, persistent):
    """Whole solves in mode 3: every trace event (after each merge, batch
    and stage), the final partition, B, S and the counters equal the
    oracle's; persistent and per-batch schedules, dense tile and sorted
    views, with and without the FP64 shadow evaluation (which decides
    nothing in mode 3 and only adds the flip counts)."""
    params = dict(params, precision=3)
    n, src, dst, w = GRAPHS[graph]()
    part_g, res_g, ev_g, part_o, res_o, ev_o = _solve_pair(api, oracle, n, src, dst, w, params, persistent)
    if persistent:
        ev_o = [e for e in ev_o if e["kind"] in (1, 3)]
        ev_g = [e for e in ev_g if e["kind"] in (1, 3)]
    assert len(ev_g) == len(ev_o)
    for i, (a, b) in enumerate(zip(ev_g, ev_o)):
        assert a == b, (graph, i, a, b)
    assert np.array_equal(part_g, part_o)
    for k in ("B", "S_q", "stages", "sweeps", "batches", "nodal_proposals", "nodal_moves",
              "merge_shortfall", "near_threshold"):
        assert res_g[k] == res_o[k], k
    if params.get("fp64_shadow"):
        assert res_g["fp32_nodal_evals"] > 0
        assert res_g["fp32_flip_rate"] == res_g["fp32_nodal_flips"] / res_g["fp32_nodal_evals"]
    else:
        assert res_g["fp32_nodal_evals"] == 0 and res_g["fp32_nodal_flips"] == 0


@pytest.mark.parametrize("within,alpha,seed", [(0.8, 10.0, 0), (0.5, 1.0, 1), (0.8, 1.0, 2),
                                               (0.5, 10.0, 3)])
def test_ref32_c1_solve_exact(api, oracle, within, alpha, seed):
    """N=5000, 19 planted blocks, the four {within, alpha} variants in mode 3:
    final partition, B, S and sweeps equal the oracle's."""
    from usap_b200 import native as nat
    G = gen.generate(gen.config_c1(within=within, alpha=alpha, seed=seed))
    params = {"num_batch_nodal_update": 10, "seed": seed, "precision": 3}
    ctx = api.Context(0)
    ctx.load(G.src, G.dst, None, G.n)
    part_g, res_g = ctx.partition(nat.default_params(**params))
    ctx.close()
    og = oracle.OracleGraph(G.n, G.src, G.dst)
    part_o, res_o, _ = og.partition(params)
    assert np.array_equal(part_g, part_o)
    assert (res_g["B"], res_g["S_q"], res_g["sweeps"]) == (res_o["B"], res_o["S_q"], res_o["sweeps"])
