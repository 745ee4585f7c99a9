"""The served form (usap_server_*): requests submitted while others run.

Each request's result must equal the one-shot usap_partition result for the
same graph and seed (bit for bit: the solve is deterministic), whatever else
is running; the memory budget must bound what is admitted at once; a request
larger than the whole budget is refused at submit.
"""
import time

import numpy as np
import pytest

from usap_b200 import generator as gen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    from usap_b200 import api as a
    return a


def _mix():
    """Graphs of uneven sizes (N 1k..20k), several seeds each."""
    cfgs = gen.config_c3(seed=7, graphs=6)
    graphs = [gen.generate(c) for c in cfgs]
    jobs = [(gi, sd) for gi in range(len(graphs)) for sd in (1, 2)]
    return graphs, jobs


def test_served_results_equal_alone(api):
    from usap_b200 import native as nat
    graphs, jobs = _mix()
    alone = {}
    for gi, sd in jobs:
        G = graphs[gi]
        alone[(gi, sd)] = api.partition(G.src, G.dst, None, G.n,
                                         params=nat.default_params(num_batch_nodal_update=10, seed=sd))
    srv = api.Server(workers=5)
    tickets = {}
    # staggered arrivals: later requests join while earlier ones run
    for k, (gi, sd) in enumerate(jobs):
        G = graphs[gi]
        tickets[(gi, sd)] = srv.submit(G.src, G.dst, None, G.n,
                                       params=nat.default_params(num_batch_nodal_update=10, seed=sd))
        if k % 3 == 2:
            time.sleep(0.01)
    for key, t in tickets.items():
        part, res, timing = srv.wait(t)
        a_part, a_res = alone[key]
        assert np.array_equal(part, a_part), key
        assert res["S_q"] == a_res["S_q"] and res["B"] == a_res["B"], key
        assert timing["ms_latency"] >= timing["ms_running"] > 0
    st = srv.stats()
    assert st["completed"] == len(jobs) and st["failed"] == 0
    assert 1 <= st["peak_running"] <= 5
    srv.close()


def test_served_budget_bounds_admission(api):
    """With a budget that fits about one request at a time the service runs
    them one by one and still finishes all; poll reports progress."""
    from usap_b200 import native as nat
    G = gen.generate(gen.config_c1(seed=1))
    # one request's estimate is about 340 MiB in the default precision (its
    # dense tile may reach 16384 blocks, here N=5000): one fits, two do not
    srv = api.Server(workers=4, memory_budget=500 << 20)
    ts = [srv.submit(G.src, G.dst, None, G.n, params=nat.default_params(num_batch_nodal_update=10, seed=s))
          for s in range(3)]
    seen = None
    while seen is None:
        seen = srv.poll(ts[-1])
        if seen is None:
            time.sleep(0.005)
    results = [srv.wait(t) for t in ts[:-1]] + [seen]
    st = srv.stats()
    assert st["peak_admitted_bytes"] <= st["memory_budget"]
    assert st["peak_running"] == 1, st
    assert st["completed"] == 3
    ref = api.partition(G.src, G.dst, None, G.n, params=nat.default_params(num_batch_nodal_update=10, seed=0))
    assert np.array_equal(results[0][0], ref[0])
    srv.close()


def test_served_refuses_oversized_request(api):
    from usap_b200 import native as nat
    G = gen.generate(gen.config_c0(seed=0))
    srv = api.Server(workers=1, memory_budget=1 << 20)
    with pytest.raises(nat.UsapError) as e:
        srv.submit(G.src, G.dst, None, G.n)
    assert e.value.code == -4
    srv.close()
