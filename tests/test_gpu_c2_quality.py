"""The headline graph (N=50000, 44 planted blocks, within 0.5, alpha 1) and
the solve quality against the reference's own runs.

* Whole solves of the N=50000 graph and one-block-per-vertex starts at
  N=5000 equal the oracle's bit for bit (partition, B, S, sweeps).
* Quality: the reference seeds from std::random_device, so it is compared by
  distribution.  tests/golden/ref_quality.json holds the B and NMI of
  repeated runs of the reference's own partition() (make_quality.py) on the
  C1 variants (N=5000), a reduced-N stand-in (N=20000) and the N=50000
  graph.  Sixteen seeded solves in the default precision (the reference's
  float nodal dS) must reach a mean NMI within TOL_NMI of the reference's
  mean.  A reference run that found no structure (NMI below NO_STRUCTURE,
  one of sixteen at N=50000, ending at B=218) is left out of its mean and
  none of ours may end that way, nor at B = 1.
"""
import json
import os

import numpy as np
import pytest

from usap_b200 import generator as gen

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
QUALITY = os.path.join(ROOT, "tests", "golden", "ref_quality.json")
TOL_NMI = 0.01
NO_STRUCTURE = 0.2
SEEDS = 16
B0_BAND = 0.10   # device initial blocks: within 10% of the SCC pass's count
MAX_NO_STRUCTURE = 2


@pytest.fixture(scope="module")
def api():
    from usap_b200 import api as a
    return a


@pytest.mark.parametrize("precision", [0, 3])
def test_c2_solve_exact(api, oracle, precision):
    """N=50000, seed 0: partition, B, S and sweeps equal the oracle's."""
    from usap_b200 import native as nat
    G = gen.generate(gen.config_c2(seed=0))
    params = {"num_batch_nodal_update": 10, "seed": 0, "precision": precision}
    ctx = api.Context(0)
    ctx.load(G.src, G.dst, None, G.n)
    part_g, res_g = ctx.partition(nat.default_params(**params))
    ctx.close()
    part_o, res_o, _ = oracle.OracleGraph(G.n, G.src, G.dst).partition(params)
    assert np.array_equal(part_g, part_o)
    assert (res_g["B"], res_g["S_q"], res_g["sweeps"], res_g["stages"]) == \
        (res_o["B"], res_o["S_q"], res_o["sweeps"], res_o["stages"])


@pytest.mark.parametrize("precision", [0, 3])
def test_identity_init_exact(api, oracle, precision):
    """N=5000 from one block per vertex (B=N, the sorted views until
    B <= dense_max): the whole solve equals the oracle's."""
    from usap_b200 import native as nat
    G = gen.generate(gen.config_c1(within=0.5, alpha=1.0, seed=0))
    params = {"num_batch_nodal_update": 10, "seed": 1, "precision": precision, "init_mode": 1}
    ctx = api.Context(0)
    ctx.load(G.src, G.dst, None, G.n)
    part_g, res_g = ctx.partition(nat.default_params(dense_max=1024, **params))
    ctx.close()
    part_o, res_o, _ = oracle.OracleGraph(G.n, G.src, G.dst).partition(params)
    assert np.array_equal(part_g, part_o)
    assert (res_g["B"], res_g["S_q"], res_g["sweeps"]) == (res_o["B"], res_o["S_q"], res_o["sweeps"])


def _ref_runs():
    with open(QUALITY) as f:
        return json.load(f)


@pytest.mark.parametrize("name", ["c1_f0.8_a10", "c1_f0.5_a10", "c1_f0.8_a1", "c1_f0.5_a1", "n20k", "c2"])
def test_quality_matches_reference_runs(api, name):
    from usap_b200 import native as nat
    rec = _ref_runs()[name]
    c = rec["config"]
    G = gen.generate(gen.SBMConfig(n=c["n"], blocks=c["blocks"], within=c["within"], alpha=c["alpha"],
                                   seed=c["seed"]))
    ref = np.array([r["nmi"] for r in rec["runs"]])
    ctx = api.Context(0)
    ctx.load(G.src, G.dst, None, G.n)
    nmi, Bs = [], []
    for seed in range(SEEDS):
        part, res = ctx.partition(nat.default_params(num_batch_nodal_update=10, seed=seed))
        nmi.append(api.evaluate(G.truth, part)["nmi"])
        Bs.append(res["B"])
    ctx.close()
    nmi = np.array(nmi)
    assert min(Bs) > 1 and nmi.min() >= NO_STRUCTURE, (Bs, nmi)
    ref_ok = ref[ref >= NO_STRUCTURE]
    assert ref_ok.size >= ref.size - 1
    assert abs(nmi.mean() - ref_ok.mean()) <= TOL_NMI, (name, nmi.mean(), ref_ok.mean())


@pytest.mark.parametrize("name", ["c1_f0.5_a1", "c2"])
def test_device_initial_blocks(api, name):
    """init_mode 2, the device stand-in for the host SCC pass (multi-source
    breadth-first cells from one vertex in eight): as many initial blocks
    as the SCC pass within B0_BAND and a deterministic partition.  Over 16
    seeds, the runs that find structure reach a mean NMI within TOL_NMI of
    the reference's runs, as the default path must.  Unlike the default
    path, this start sometimes keeps a large B and finds no structure, as
    the reference itself does (1 of 16 runs at N=50000 here, 1 of 20 in an
    earlier sample): at most MAX_NO_STRUCTURE of 16 may."""
    from usap_b200 import native as nat
    rec = _ref_runs()[name]
    c = rec["config"]
    G = gen.generate(gen.SBMConfig(n=c["n"], blocks=c["blocks"], within=c["within"], alpha=c["alpha"],
                                   seed=c["seed"]))
    ctx = api.Context(0)
    ctx.load(G.src, G.dst, None, G.n)
    _, scc = ctx.partition(nat.default_params(num_batch_nodal_update=10, seed=0))
    nmi, first = [], None
    for seed in range(SEEDS):
        part, res = ctx.partition(nat.default_params(num_batch_nodal_update=10, seed=seed, init_mode=2))
        assert abs(res["B_init"] - scc["B_init"]) <= B0_BAND * scc["B_init"], (res["B_init"], scc["B_init"])
        if first is None:
            first = (part, res)
        nmi.append(api.evaluate(G.truth, part)["nmi"])
    again, res2 = ctx.partition(nat.default_params(num_batch_nodal_update=10, seed=0, init_mode=2))
    assert np.array_equal(again, first[0]) and res2["S_q"] == first[1]["S_q"]
    ctx.close()
    ref = np.array([r["nmi"] for r in rec["runs"]])
    ref_ok = ref[ref >= NO_STRUCTURE]
    nmi = np.array(nmi)
    ok = nmi[nmi >= NO_STRUCTURE]
    assert ok.size >= SEEDS - MAX_NO_STRUCTURE, nmi
    assert abs(ok.mean() - ref_ok.mean()) <= TOL_NMI, (name, ok.mean(), ref_ok.mean())
