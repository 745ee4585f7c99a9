"""Failure detection of the persistent nodal kernel, without a GPU fault.

Every grid barrier of the cooperative kernel waits with a limit; when the
limit runs out the kernel sets an error flag, every CTA returns, and the
host turns the flag into USAP_ERR_INTERNAL.  The test arms the context's
failure injection (one CTA never arrives at its barriers, waits limited to
50 ms), checks that the solve fails with that status and message, and that
the same context then solves the graph again with the result it gave before.
"""
import numpy as np
import pytest

from usap_b200 import generator as gen

pytestmark = pytest.mark.gpu


def test_barrier_timeout_reports_and_recovers():
    from usap_b200 import api, native as nat
    G = gen.generate(gen.config_c0())
    ctx = api.Context(0)
    ctx.load(G.src, G.dst, None, G.n)
    p = nat.default_params(num_batch_nodal_update=10, seed=0)
    part0, res0 = ctx.partition(p)
    ctx.test_barrier_timeout(hold_cta=3, timeout_ns=50_000_000)
    with pytest.raises(nat.UsapError) as e:
        ctx.partition(p)
    assert e.value.code == -6 and "grid barrier timed out" in str(e.value)
    part1, res1 = ctx.partition(p)   # the injection was for one launch only
    assert np.array_equal(part0, part1) and res1["S_q"] == res0["S_q"]
    with pytest.raises(nat.UsapError):
        ctx.test_barrier_timeout(hold_cta=-1, timeout_ns=1000)
    ctx.close()
