"""Seeded synthetic directed degree-corrected SBM graphs (DC-SBM).

The published uSAP numbers were measured on the 2022 GraphChallenge
streaming-partition *static* datasets, whose large edge files are not
available here.  This generator stands in for them with the same kind of
input the reference consumes (``graph_parallel.hpp:251-317``): a directed,
unit-weight edge list with 1-based ids, no self loops, every vertex with at
least one out-edge (the reference takes ``N = max(source id)``,
``graph_parallel.hpp:276``), plus the planted ("true") partition.

Steps (per config):

1. Block sizes ``round(N * Dirichlet(alpha))``, each at least 1, summing to N.
2. Out-degree and in-degree weight per vertex from a power law truncated to
   ``[dmin, dmax]`` (pdf ~ x^-gamma).  The config wording (exponent 2.5,
   range 5..100, mean about 16, ~16k edges at N=1000) is not jointly
   satisfiable: the mean of x^-2.5 on [5, 100] is 11.8.  We keep the range
   and the edge counts, which set the workload size: gamma = 2.0 gives a
   mean of 15.8.
3. Each out-edge of v lands in v's block with probability ``f`` (the
   within-block fraction), else in a uniformly chosen other block; the
   target vertex inside the block is drawn proportional to its in-degree
   weight.
4. Self loops are dropped, duplicates merged (unit weight), ids randomly
   permuted; any vertex left without an out-edge gets one to a random other
   vertex of its block (or of the graph, for singleton blocks).
5. Edges are emitted sorted by (src, dst), the order a TSV file would hold.

Everything is drawn from ``numpy.random.default_rng(seed)``, so a config and
seed name a graph exactly.
"""
from __future__ import annotations

import dataclasses
import os
from typing import Optional

import numpy as np


@dataclasses.dataclass(frozen=True)
class SBMConfig:
    n: int
    blocks: int
    within: float = 0.8      # fraction of each vertex's edges inside its block
    alpha: float = 10.0      # Dirichlet concentration of block sizes
    gamma: float = 2.0       # power-law exponent of degrees (pdf ~ x^-gamma)
    dmin: float = 5.0
    dmax: float = 100.0
    seed: int = 0


@dataclasses.dataclass
class Graph:
    """A directed graph in the reference's input shape.

    ``src``/``dst`` are 0-based int32 arrays in file order; ``truth`` holds
    the planted block of each vertex (0-based).
    """
    n: int
    src: np.ndarray
    dst: np.ndarray
    weight: Optional[np.ndarray]
    truth: Optional[np.ndarray]
    name: str = ""

    @property
    def num_edges(self) -> int:
        return int(self.src.shape[0])

    def write_tsv(self, basename: str) -> None:
        """Write ``basename.tsv`` and ``basename_truePartition.tsv`` in the
        reference's format (1-based ``from<TAB>to<TAB>w`` and
        ``node<TAB>block``)."""
        os.makedirs(os.path.dirname(basename) or ".", exist_ok=True)
        w = self.weight if self.weight is not None else np.ones_like(self.src)
        arr = np.stack([self.src.astype(np.int64) + 1,
                        self.dst.astype(np.int64) + 1,
                        w.astype(np.int64)], axis=1)
        np.savetxt(basename + ".tsv", arr, fmt="%d", delimiter="\t")
        truth = self.truth if self.truth is not None else np.zeros(self.n, np.int64)
        tp = np.stack([np.arange(1, self.n + 1, dtype=np.int64),
                       truth.astype(np.int64) + 1], axis=1)
        np.savetxt(basename + "_truePartition.tsv", tp, fmt="%d", delimiter="\t")


def _power_law(rng: np.random.Generator, size: int, gamma: float,
               lo: float, hi: float) -> np.ndarray:
    """Inverse-CDF draws from pdf ~ x^-gamma on [lo, hi]."""
    u = rng.random(size)
    if abs(gamma - 1.0) < 1e-12:
        return lo * (hi / lo) ** u
    a = 1.0 - gamma
    return (lo ** a + u * (hi ** a - lo ** a)) ** (1.0 / a)


def _block_sizes(rng: np.random.Generator, n: int, b: int, alpha: float) -> np.ndarray:
    if b < 1 or b > n:
        raise ValueError(f"need 1 <= blocks <= n (got blocks={b}, n={n})")
    p = rng.dirichlet(np.full(b, float(alpha)))
    sizes = np.maximum(1, np.round(p * n).astype(np.int64))
    # fix the total by trimming / growing the largest blocks
    diff = int(sizes.sum() - n)
    order = np.argsort(-sizes, kind="stable")
    i = 0
    while diff != 0:
        j = order[i % b]
        if diff > 0 and sizes[j] > 1:
            sizes[j] -= 1
            diff -= 1
        elif diff < 0:
            sizes[j] += 1
            diff += 1
        i += 1
    return sizes


def generate(cfg: SBMConfig) -> Graph:
    """Generate one DC-SBM graph; deterministic in ``cfg``."""
    rng = np.random.default_rng(cfg.seed)
    n, b = int(cfg.n), int(cfg.blocks)
    sizes = _block_sizes(rng, n, b, cfg.alpha)
    block_of = np.repeat(np.arange(b, dtype=np.int64), sizes)       # pre-permutation ids
    starts = np.concatenate([[0], np.cumsum(sizes)])

    dout = np.maximum(1, np.round(_power_law(rng, n, cfg.gamma, cfg.dmin, cfg.dmax))).astype(np.int64)
    theta_in = _power_law(rng, n, cfg.gamma, cfg.dmin, cfg.dmax)

    # per-block cumulative in-weight for target sampling
    cum_in = np.cumsum(theta_in)
    block_in_lo = np.concatenate([[0.0], cum_in])[starts[:-1]]
    block_in_hi = cum_in[starts[1:] - 1]

    src = np.repeat(np.arange(n, dtype=np.int64), dout)
    e = src.shape[0]
    own = block_of[src]
    inside = rng.random(e) < cfg.within
    if b > 1:
        other = rng.integers(0, b - 1, size=e)
        other = other + (other >= own)          # uniform over blocks != own
        tblk = np.where(inside, own, other)
    else:
        tblk = own
    lo = block_in_lo[tblk]
    hi = block_in_hi[tblk]
    x = lo + rng.random(e) * (hi - lo)
    dst = np.searchsorted(cum_in, x, side="right")
    dst = np.clip(dst, starts[tblk], starts[tblk + 1] - 1)

    keep = src != dst
    src, dst = src[keep], dst[keep]

    perm = rng.permutation(n)                    # old id -> new id
    src, dst = perm[src], perm[dst]
    truth = np.empty(n, dtype=np.int64)
    truth[perm] = block_of

    key = np.unique(src * n + dst)               # merge duplicates, sort by (src, dst)
    src, dst = key // n, key % n

    # guarantee one out-edge per vertex (the reference takes N = max source id)
    has_out = np.zeros(n, dtype=bool)
    has_out[src] = True
    missing = np.nonzero(~has_out)[0]
    if missing.size:
        members = [np.nonzero(truth == k)[0] for k in range(b)]
        add_dst = np.empty(missing.size, dtype=np.int64)
        for i, v in enumerate(missing):
            pool = members[truth[v]]
            if pool.size < 2:
                pool = np.arange(n)
            t = v
            while t == v:
                t = int(pool[rng.integers(0, pool.size)])
            add_dst[i] = t
        key = np.unique(np.concatenate([src * n + dst, missing * n + add_dst]))
        src, dst = key // n, key % n

    name = f"dcsbm_n{n}_b{b}_f{cfg.within:g}_a{cfg.alpha:g}_s{cfg.seed}"
    return Graph(n=n, src=src.astype(np.int32), dst=dst.astype(np.int32),
                 weight=None, truth=truth.astype(np.int32), name=name)


def read_tsv(basename: str) -> Graph:
    """Read a reference-format TSV pair (1-based ids).  ``N`` is the largest
    source id, as in ``graph_parallel.hpp:276``."""
    arr = np.loadtxt(basename + ".tsv", dtype=np.int64, ndmin=2)
    src = arr[:, 0] - 1
    dst = arr[:, 1] - 1
    w = arr[:, 2] if arr.shape[1] > 2 else None
    n = int(src.max()) + 1 if src.size else 0
    truth = None
    tp = basename + "_truePartition.tsv"
    if os.path.exists(tp):
        t = np.loadtxt(tp, dtype=np.int64, ndmin=2)
        truth = (t[:, 1] - 1).astype(np.int32)
    weight = None
    if w is not None and not np.all(w == 1):
        weight = w.astype(np.int32)
    return Graph(n=n, src=src.astype(np.int32), dst=dst.astype(np.int32),
                 weight=weight, truth=truth, name=os.path.basename(basename))


# Named workloads (sizes and shapes of the plain-SBP configs).
def config_c0(seed: int = 0) -> SBMConfig:
    """N=1000, 11 planted blocks, within-block 0.8, alpha 10 (~16k edges)."""
    return SBMConfig(n=1000, blocks=11, within=0.8, alpha=10.0, seed=seed)


def config_c1(within: float = 0.8, alpha: float = 10.0, seed: int = 0) -> SBMConfig:
    """N=5000, 19 planted blocks, four {within, alpha} variants (~80k edges)."""
    return SBMConfig(n=5000, blocks=19, within=within, alpha=alpha, seed=seed)


def config_c2(seed: int = 0) -> SBMConfig:
    """N=50000, 44 planted blocks, within-block 0.5, alpha 1 (~800k edges)."""
    return SBMConfig(n=50000, blocks=44, within=0.5, alpha=1.0, seed=seed)


def config_c3(seed: int = 0, graphs: int = 64):
    """Batched workload: ``graphs`` graphs with N log-uniform in [1000, 20000],
    round(N^0.35) planted blocks, within-block fraction uniform in [0.5, 0.8]
    and Dirichlet alpha in {1, 10}; one SBMConfig per graph."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(graphs):
        n = int(round(np.exp(rng.uniform(np.log(1000), np.log(20000)))))
        out.append(SBMConfig(n=n, blocks=max(1, int(round(n ** 0.35))),
                             within=float(rng.uniform(0.5, 0.8)),
                             alpha=float(rng.choice([1.0, 10.0])),
                             seed=int(rng.integers(0, 2**31 - 1))))
    return out


def config_c4(seed: int = 0, graphs: int = 2000):
    """Served workload: ``graphs`` requests with N log-uniform in
    [1000, 200000] and the batched workload's other parameters (blocks
    round(N^0.35), within-block fraction U[0.5, 0.8], alpha in {1, 10})."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(graphs):
        n = int(round(np.exp(rng.uniform(np.log(1000), np.log(200000)))))
        out.append(SBMConfig(n=n, blocks=max(1, int(round(n ** 0.35))),
                             within=float(rng.uniform(0.5, 0.8)),
                             alpha=float(rng.choice([1.0, 10.0])),
                             seed=int(rng.integers(0, 2**31 - 1))))
    return out
