"""Edge-list ingest on the device (usap_ctx_load_tsv) against loading the
same edges from arrays, through the C ABI.

The text of a reference-format .tsv file is parsed on the GPU with the
reference loader's field rules (graph_parallel.hpp:264-277): tab-separated
std::stoul / std::stof fields, the weight truncated to an integer, a line
without a second tab taking its source id as weight, N = the largest source
id.  The loaded graph must give the same interblock counts and the same
partition as the arrays it was written from, and malformed lines must come
back as errors naming the line.
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


def _tsv(src, dst, w=None, sep="\n", last=True):
    w = np.ones(len(src), np.int64) if w is None else w
    lines = [f"{s + 1}\t{d + 1}\t{x}" for s, d, x in zip(src, dst, w)]
    return (sep.join(lines) + (sep if last else "")).encode()


def _same_counts(api, ctx_a, ctx_b, n, B=5, seed=3):
    part = np.random.default_rng(seed).integers(0, B, n).astype(np.int32)
    part[:B] = np.arange(B)
    Ma, oa, ia = ctx_a.op_build(part, B)
    Mb, ob, ib = ctx_b.op_build(part, B)
    assert np.array_equal(Ma, Mb) and np.array_equal(oa, ob) and np.array_equal(ia, ib)


@pytest.mark.parametrize("weighted,sep,last", [(False, "\n", True), (True, "\r\n", False)])
def test_tsv_equals_arrays(api, weighted, sep, last):
    from usap_b200 import native as nat
    G = gen.generate(gen.config_c1(within=0.8, alpha=10.0, seed=3))
    w = np.random.default_rng(1).integers(1, 4, G.num_edges).astype(np.int32) if weighted else None
    a = api.Context(0)
    a.load(G.src, G.dst, w, G.n)
    b = api.Context(0)
    b.load_tsv(_tsv(G.src, G.dst, w, sep, last))
    _same_counts(api, a, b, G.n)
    p = nat.default_params(num_batch_nodal_update=10, seed=4)
    pa, ra = a.partition(p)
    pb, rb = b.partition(p)
    assert np.array_equal(pa, pb) and ra["S_q"] == rb["S_q"]
    a.close()
    b.close()


def test_tsv_reference_field_rules(api):
    # two-field line: weight = source id; fractional weight truncated; leading
    # spaces; a one-field line is a self loop of weight = id (the reference's
    # npos arithmetic); N = largest source id (3), target 3 is allowed
    text = b"1\t2\n2\t3\t2.7\n 3\t 1\t1\n2\n"
    src = np.array([0, 1, 2, 1], np.int32)
    dst = np.array([1, 2, 0, 1], np.int32)
    w = np.array([1, 2, 1, 2], np.int32)
    a = api.Context(0)
    a.load(src, dst, w, 3)
    b = api.Context(0)
    b.load_tsv(text)
    _same_counts(api, a, b, 3, B=2)
    a.close()
    b.close()


@pytest.mark.parametrize("text,line", [
    (b"1\t2\t1\n\n2\t1\t1\n", 2),          # empty line
    (b"1\t2\t1\nx\t1\t1\n", 2),            # no digits
    (b"1\t2\t1\n2\t0\t1\n", 2),            # id 0
    (b"1\t2\t1\n2\t1\t0\n3\t1\t-1\n", 2),  # weight 0 (and a negative one later)
    (b"1\t2\t1\n2\t1\t1\n3\t9999999999\t1\n", 3),   # value above 2^31 - 1
])
def test_tsv_malformed_lines(api, text, line):
    from usap_b200 import native as nat
    ctx = api.Context(0)
    with pytest.raises(nat.UsapError) as e:
        ctx.load_tsv(text)
    assert f"tsv line {line}:" in str(e.value)
    ctx.close()


def test_tsv_c2_parse(api):
    """The N=50k graph (~780k lines): same graph as the arrays; parse time
    printed beside numpy's text reader."""
    G = gen.generate(gen.config_c2())
    text = _tsv(G.src, G.dst)
    a = api.Context(0)
    a.load(G.src, G.dst, None, G.n)
    b = api.Context(0)
    b.load_tsv(text)
    t0 = time.perf_counter()
    b.load_tsv(text)
    t1 = time.perf_counter()
    np.loadtxt(text.decode().splitlines()[:100000], dtype=np.int64)
    t2 = time.perf_counter()
    _same_counts(api, a, b, G.n, B=40)
    print(f"tsv load {len(text) / 1e6:.1f} MB: device {1e3 * (t1 - t0):.1f} ms (parse + adjacency + upload); "
          f"numpy loadtxt of 100k lines {1e3 * (t2 - t1):.1f} ms")
    a.close()
    b.close()


def _shuffled(G, seed=9):
    """the same edges in a random file order (not grouped by source)"""
    perm = np.random.default_rng(seed).permutation(G.num_edges)
    return G.src[perm], G.dst[perm]


@pytest.mark.parametrize("case", ["c2", "c2_shuffled", "weighted_crlf", "weighted_shuffled"])
def test_device_adjacency_equals_host(api, case):
    """usap_ctx_load_tsv builds the out- and in-lists on the device (stable
    counting sort by source and by target, file order kept inside each
    list); they equal, byte for byte, the lists the host builds from the
    same edges as arrays (usap_ctx_load), with the weights and weighted
    degrees."""
    if case.startswith("c2"):
        G = gen.generate(gen.config_c2(seed=0))
    else:
        G = gen.generate(gen.config_c1(within=0.5, alpha=1.0, seed=2))
    src, dst = _shuffled(G) if case.endswith("shuffled") else (G.src, G.dst)
    w = np.random.default_rng(5).integers(1, 4, src.size).astype(np.int32) if case.startswith("weighted") else None
    n = int(max(src.max(), dst.max())) + 1
    a = api.Context(0)
    a.load(src, dst, w, n)
    b = api.Context(0)
    b.load_tsv(_tsv(src, dst, w, "\r\n" if case.endswith("crlf") else "\n"), n)
    ha, hb = a.adjacency(), b.adjacency()
    for k in ha:
        assert ha[k].dtype == hb[k].dtype and np.array_equal(ha[k], hb[k]), (case, k)
    # file order inside the lists: the in-list of a vertex lists its sources
    # in the order their edges appear in the input
    v = int(np.argmax(np.bincount(dst, minlength=n)))
    lo, hi = hb["in_ptr"][v], hb["in_ptr"][v + 1]
    assert np.array_equal(hb["in_idx"][lo:hi], src[dst == v])
    a.close()
    b.close()
