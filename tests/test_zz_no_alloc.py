"""usap_entropy_static, the allocation-free scoring entry point, through the C ABI.

It must give the value usap_op_entropy gives for the same graph and
partition.  Both sum the same Q32-rounded terms in int64, so the tolerance
is 0 Q32 units.  Two calls are enqueued back to back on one stream, the
first with more blocks than the second, so the second finds the shared
scratch dirty and must clear it.  This file runs last (its name sorts
last) and also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from usap_b200 import generator as gen

pytestmark = pytest.mark.gpu

TOL_Q32 = 0          # identical terms, order-independent integer sum
MAX_BLOCKS = 1024    # USAP_STATIC_MAX_BLOCKS
MAX_WEIGHT = 1 << 20  # USAP_STATIC_MAX_WEIGHT
INT64_MIN = -(1 << 63)


@pytest.fixture(scope="module")
def env():
    import torch
    from usap_b200 import api, native
    return torch, api, native


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, np.int32)).cuda()


def _call(torch, native, src, dst, w, n, part, B, out):
    st = torch.cuda.current_stream().cuda_stream
    return native.lib().usap_entropy_static(
        C.c_void_p(src.data_ptr()), C.c_void_p(dst.data_ptr()),
        C.c_void_p(w.data_ptr()) if w is not None else None, src.numel(), n,
        C.c_void_p(part.data_ptr()), B, C.c_void_p(out.data_ptr()), C.c_void_p(st))


def _reference(api, G, w, parts):
    ctx = api.Context(0)
    ctx.load(G.src, G.dst, w, G.n)
    vals = [ctx.op_entropy(p, B) for p, B in parts]
    ctx.close()
    return vals


def _weighted(seed=4):
    G = gen.generate(gen.SBMConfig(n=400, blocks=5, within=0.75, alpha=5, seed=seed))
    rng = np.random.default_rng(seed)
    # a few self loops and a repeated edge, which both entry points count
    src = np.concatenate([G.src, [3, 3, 8], G.src[:5]]).astype(np.int32)
    dst = np.concatenate([G.dst, [3, 3, 8], G.dst[:5]]).astype(np.int32)
    w = rng.integers(1, 5, src.size).astype(np.int32)
    return gen.Graph(n=G.n, src=src, dst=dst, weight=w, truth=G.truth), w


@pytest.mark.parametrize("kind", ["c0", "weighted"])
def test_static_equals_op_entropy_two_calls(env, kind):
    torch, api, native = env
    if kind == "c0":
        G, w = gen.generate(gen.config_c0(seed=2)), None
    else:
        G, w = _weighted()
    rng = np.random.default_rng(11)
    big = min(MAX_BLOCKS, G.n)
    parts = [(rng.integers(0, big, G.n).astype(np.int32), big),
             (G.truth.astype(np.int32), int(G.truth.max()) + 1)]
    want = _reference(api, G, w, parts)

    src, dst = _dev(torch, G.src), _dev(torch, G.dst)
    wd = _dev(torch, w) if w is not None else None
    outs = [torch.zeros(1, dtype=torch.int64, device="cuda") for _ in parts]
    dparts = [_dev(torch, p) for p, _ in parts]
    for (p, B), dp, out in zip(parts, dparts, outs):
        rc = _call(torch, native, src, dst, wd, G.n, dp, B, out)
        assert rc == 0, native.lib().usap_last_error()
    torch.cuda.synchronize()
    got = [int(o.item()) for o in outs]
    for g, w_ in zip(got, want):
        assert abs(g - w_) <= TOL_Q32, (got, want)


def test_static_limits_and_bad_ids(env):
    torch, api, native = env
    G = gen.generate(gen.config_c0(seed=2))
    src, dst = _dev(torch, G.src), _dev(torch, G.dst)
    part = _dev(torch, G.truth)
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    # beyond the block limit: rejected on the host, nothing launched
    rc = _call(torch, native, src, dst, None, G.n, part, MAX_BLOCKS + 1, out)
    assert rc == -4
    assert b"static scratch limit" in native.lib().usap_last_error()
    # a block id outside [0, B): the device checks turn it into INT64_MIN
    Bt = int(G.truth.max()) + 1
    bad = G.truth.astype(np.int32).copy()
    bad[17] = 5000
    rc = _call(torch, native, src, dst, None, G.n, _dev(torch, bad), Bt, out)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(out.item()) == INT64_MIN
    # and a good call right after is exact again
    want = _reference(api, G, None, [(G.truth.astype(np.int32), Bt)])[0]
    rc = _call(torch, native, src, dst, None, G.n, part, Bt, out)
    assert rc == 0
    torch.cuda.synchronize()
    assert abs(int(out.item()) - want) <= TOL_Q32


def test_static_calls_allocate_nothing(env):
    """After the first call on a device (which sets up the log table and
    loads the kernels), further calls leave the device's free memory
    unchanged: the entry point allocates nothing."""
    torch, api, native = env
    G = gen.generate(gen.config_c0(seed=3))
    src, dst = _dev(torch, G.src), _dev(torch, G.dst)
    part = _dev(torch, G.truth)
    Bt = int(G.truth.max()) + 1
    outs = [torch.zeros(1, dtype=torch.int64, device="cuda") for _ in range(8)]
    assert _call(torch, native, src, dst, None, G.n, part, Bt, outs[0]) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for out in outs:
        assert _call(torch, native, src, dst, None, G.n, part, Bt, out) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    vals = {int(o.item()) for o in outs}
    assert len(vals) == 1


_FRESH = r"""
import ctypes as C, sys
import numpy as np, torch
sys.path.insert(0, sys.argv[1])
from usap_b200 import api, generator as gen, native
G = gen.generate(gen.config_c0(seed=5))
Bt = int(G.truth.max()) + 1
ctx = api.Context(0); ctx.load(G.src, G.dst, None, G.n)
want = ctx.op_entropy(G.truth.astype(np.int32), Bt); ctx.close()
st = torch.cuda.Stream()          # non-blocking with respect to the legacy stream
with torch.cuda.stream(st):
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.int32)).cuda()
    src, dst, part = d(G.src), d(G.dst), d(G.truth)
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    st.synchronize()
    rc = native.lib().usap_entropy_static(C.c_void_p(src.data_ptr()), C.c_void_p(dst.data_ptr()), None,
                                          src.numel(), G.n, C.c_void_p(part.data_ptr()), Bt,
                                          C.c_void_p(out.data_ptr()), C.c_void_p(st.cuda_stream))
    assert rc == 0, native.lib().usap_last_error()
st.synchronize()
assert int(out.item()) == want, (int(out.item()), want)
print("fresh ok")
"""


def test_static_first_call_on_nonblocking_stream(env):
    """In a fresh process, the very first call (the one that sets up the
    log table) runs on a non-blocking stream and is already exact."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    p = subprocess.run([sys.executable, "-c", _FRESH, root], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    assert "fresh ok" in p.stdout
