"""Partition scores on the device (usap_evaluate_device, usap_ctx_evaluate)
against the host version, through the C ABI.

Both form the scores from the same exact integer pair counts and the same
fixed-point information sums, so every score must be bit-identical (NaN
accuracy included, for more than 2048 blocks a side); the host version is
itself pinned to the oracle and to the reference's printed scores.
"""
import math

import numpy as np
import pytest

from usap_b200 import generator as gen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    from usap_b200 import api as a
    return a


def _same(a, b):
    assert a.keys() == b.keys()
    for k in a:
        x, y = a[k], b[k]
        if isinstance(x, float) and math.isnan(x):
            assert isinstance(y, float) and math.isnan(y), k
        else:
            assert x == y, (k, x, y)


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.int32)).cuda()


@pytest.mark.parametrize("n,b1,b2,unknown", [
    (500, 7, 7, 0.0),          # small table: counted in shared memory
    (20000, 44, 300, 0.05),    # 13 200 cells: counted in global memory; some truth unknown (-1)
    (50000, 44, 3000, 0.0),    # 132 000 cells, 3000 given blocks: accuracy NaN (> 2048 blocks)
    (3, 2, 2, 0.0),
])
def test_device_scores_equal_host(api, n, b1, b2, unknown):
    rng = np.random.default_rng(n)
    truth = rng.integers(0, b1, n).astype(np.int32)
    given = np.where(rng.random(n) < 0.6, truth % b2, rng.integers(0, b2, n)).astype(np.int32)
    truth[rng.random(n) < unknown] = -1
    host = api.evaluate(truth, given)
    t, g = _dev(truth), _dev(given)
    dev = api.evaluate_device(t.data_ptr(), g.data_ptr(), n)
    _same(dev, host)
    dev2 = api.evaluate_device(t.data_ptr(), g.data_ptr(), n)   # a second call on the same inputs
    _same(dev2, host)


def test_ctx_evaluate_equals_host(api):
    from usap_b200 import native as nat
    G = gen.generate(gen.config_c1(within=0.8, alpha=10.0, seed=2))
    ctx = api.Context(0)
    ctx.load(G.src, G.dst, None, G.n)
    part, res = ctx.partition(nat.default_params(num_batch_nodal_update=10, seed=1))
    dev = ctx.evaluate(G.truth)
    ctx.close()
    host = api.evaluate(G.truth, part)
    _same(dev, host)
    assert dev["b_given"] == res["B"]


def test_device_scores_reject_bad_labels(api):
    from usap_b200 import native as nat
    truth = np.zeros(10, np.int32)
    given = np.zeros(10, np.int32)
    given[3] = -1
    t, g = _dev(truth), _dev(given)
    with pytest.raises(nat.UsapError):
        api.evaluate_device(t.data_ptr(), g.data_ptr(), 10)
    truth[2] = -2
    given[3] = 0
    t, g = _dev(truth), _dev(given)
    with pytest.raises(nat.UsapError):
        api.evaluate_device(t.data_ptr(), g.data_ptr(), 10)
    ctx = api.Context(0)
    with pytest.raises(nat.UsapError):      # nothing loaded or solved yet
        ctx.evaluate(np.zeros(0, np.int32))
    ctx.close()
