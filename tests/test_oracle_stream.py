"""The oracle's warm start (og_partition_from), on the CPU: started from
the SCC pass's own blocks it is the plain solve, and block labels are only
names (any labels with the same grouping give the same solve)."""
import numpy as np

from usap_b200 import generator as gen


def test_partition_from_scc_blocks_is_the_plain_solve(oracle):
    G = gen.generate(gen.config_c0())
    og = oracle.OracleGraph(G.n, G.src, G.dst)
    params = {"num_batch_nodal_update": 10, "seed": 5}
    p1, r1, _ = og.partition(params)
    B, init = og.scc(20)
    p2, r2, _ = og.partition(params, init=init)
    assert np.array_equal(p1, p2) and (r1["B"], r1["S_q"], r1["sweeps"]) == (r2["B"], r2["S_q"], r2["sweeps"])


def test_partition_from_labels_are_names(oracle):
    G = gen.generate(gen.SBMConfig(n=400, blocks=5, within=0.75, alpha=5, seed=4))
    og = oracle.OracleGraph(G.n, G.src, G.dst)
    rng = np.random.default_rng(2)
    base = rng.integers(0, 30, G.n).astype(np.int32)
    # the same grouping under labels with gaps, in the same ascending order
    renamed = (base * 7 + 1000).astype(np.int32)
    params = {"num_batch_nodal_update": 8, "seed": 1}
    pa, ra, _ = og.partition(params, init=base)
    pb, rb, _ = og.partition(params, init=renamed)
    assert np.array_equal(pa, pb) and ra["S_q"] == rb["S_q"]
