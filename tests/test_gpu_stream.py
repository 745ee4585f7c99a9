"""Streaming input (usap_ctx_add_edges, usap_ctx_partition_from) against the
oracle, through the C ABI: a solve started from a given partition, and a
two-stage stream (half of the edges, then the rest, the second stage started
from the first stage's result with one new block per new vertex), must give
the oracle's partition, B, S and sweep count bit for bit."""
import numpy as np
import pytest

from usap_b200 import generator as gen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    from usap_b200 import api as a
    return a


def test_partition_from_equals_oracle(api, oracle):
    from usap_b200 import native as nat
    G = gen.generate(gen.config_c1(within=0.5, alpha=1.0, seed=2))
    init = np.random.default_rng(3).integers(0, 400, G.n).astype(np.int32) * 3   # labels with gaps
    params = {"num_batch_nodal_update": 10, "seed": 6}
    ctx = api.Context(0)
    ctx.load(G.src, G.dst, None, G.n)
    pg, rg = ctx.partition_from(init, nat.default_params(**params))
    ctx.close()
    og = oracle.OracleGraph(G.n, G.src, G.dst)
    po, ro, _ = og.partition(params, init=init)
    assert np.array_equal(pg, po)
    assert (rg["B"], rg["S_q"], rg["sweeps"]) == (ro["B"], ro["S_q"], ro["sweeps"])


def test_two_stage_stream_equals_oracle(api, oracle):
    from usap_b200 import native as nat
    G = gen.generate(gen.config_c1(within=0.8, alpha=10.0, seed=5))
    # stage 1: the edges among the first half of the vertices; stage 2: the
    # rest, which brings the other half of the vertices in
    n1 = G.n // 2
    first = (G.src < n1) & (G.dst < n1)
    s1, d1 = G.src[first], G.dst[first]
    s2, d2 = G.src[~first], G.dst[~first]
    src = np.concatenate([s1, s2]).astype(np.int32)
    dst = np.concatenate([d1, d2]).astype(np.int32)
    params = {"num_batch_nodal_update": 10, "seed": 2}
    ctx = api.Context(0)
    ctx.load(s1, d1, None, n1)
    p1, r1 = ctx.partition(nat.default_params(**params))
    ctx.add_edges(s2, d2, n=G.n)
    assert ctx.n == G.n and ctx.e == G.num_edges
    init = np.concatenate([p1, r1["B"] + np.arange(G.n - n1, dtype=np.int32)]).astype(np.int32)
    p2, r2 = ctx.partition_from(init, nat.default_params(**params))
    # the appended graph is the whole edge list in arrival order
    direct = api.Context(0)
    direct.load(src, dst, None, G.n)
    part = np.random.default_rng(1).integers(0, 8, G.n).astype(np.int32)
    part[:8] = np.arange(8)
    assert all(np.array_equal(x, y) for x, y in zip(ctx.op_build(part, 8), direct.op_build(part, 8)))
    direct.close()
    ctx.close()
    og1 = oracle.OracleGraph(n1, s1, d1)
    q1, o1, _ = og1.partition(params)
    assert np.array_equal(p1, q1) and r1["S_q"] == o1["S_q"]
    og2 = oracle.OracleGraph(G.n, src, dst)
    q2, o2, _ = og2.partition(params, init=init)
    assert np.array_equal(p2, q2)
    assert (r2["B"], r2["S_q"], r2["sweeps"]) == (o2["B"], o2["S_q"], o2["sweeps"])


def test_partition_from_rejects_negative_labels(api):
    from usap_b200 import native as nat
    G = gen.generate(gen.config_c0())
    ctx = api.Context(0)
    ctx.load(G.src, G.dst, None, G.n)
    init = np.zeros(G.n, np.int32)
    init[5] = -1
    with pytest.raises(nat.UsapError):
        ctx.partition_from(init)
    ctx.close()
