"""Generate the golden fixtures that pin the oracle to the reference.

Runs uSAP's own code (include/graph_parallel.hpp and evaluate.hpp, compiled
unmodified against the Taskflow-API shim by ``make -C oracle ref``) on small
seeded graphs from usap_b200.generator and records what its internal phases
compute:

* ``_scc``                        initial partition (exact)
* ``_initialize_edge_counts``     M and block degrees, dense and sparse
                                  branches (exact)
* ``_compute_overall_entropy``    S, float build and FP64 build
* ``_propose_new_partition_block`` (r, s, dS) per proposal, both builds
* ``_propose_new_partition_nodal`` (v, r, s, dS, accepted), both builds
* ``_carry_out_best_merges``      partition after merging (exact)
* ``_prepare_for_partition_next`` golden-section bracket decisions (exact)
* ``bf::evaluate``                printed scores (square tables: the only
                                  shape it scores correctly)
* ``partition()``                 NMI / pairwise precision / recall of
                                  several full reference runs (statistical)

The reference draws its proposals from libstdc++ engines, so only the
(block, target) pairs it chose and the dS it computed for them are recorded;
the oracle recomputes dS for the same pairs.  This script needs the
reference sources (REF, default /root/reference) and is run by hand; the
committed fixture is read by tests/test_oracle_pin.py.

usage: python tests/golden/make_golden.py [--ref /root/reference]
"""
from __future__ import annotations

import argparse
import gzip
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from usap_b200 import generator as gen  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "ref_fixtures.json.gz")
REF_BIN = os.path.join(ROOT, "oracle", "_ref")

GRAPHS = [
    ("g60", gen.SBMConfig(n=60, blocks=3, within=0.8, alpha=10, seed=11)),
    ("g150", gen.SBMConfig(n=150, blocks=4, within=0.6, alpha=2, seed=12)),
    ("g400", gen.SBMConfig(n=400, blocks=6, within=0.7, alpha=1, seed=13)),
    ("c0", gen.config_c0(seed=0)),
]


def run(binary: str, args, stdin: str = "") -> str:
    p = subprocess.run([os.path.join(REF_BIN, binary)] + [str(a) for a in args],
                       input=stdin, capture_output=True, text=True, timeout=600)
    if p.returncode != 0:
        raise RuntimeError(f"{binary} {args} failed: {p.stderr[:400]}")
    return p.stdout


def state_stdin(B: int, part: np.ndarray) -> str:
    return f"{B}\n" + " ".join(str(int(x)) for x in part) + "\n"


def parse_state(out: str) -> dict:
    d = {}
    for line in out.strip().splitlines():
        k, *rest = line.split()
        vals = [int(x) for x in rest]
        d[k] = vals
    trip = np.array(d["M"], dtype=np.int64).reshape(-1, 3)
    return {"B": d["B"][0], "dout": d["dout"], "din": d["din"], "M": trip.tolist()}


def parse_rows(out: str, types):
    rows = []
    for line in out.strip().splitlines():
        parts = line.split()
        rows.append([t(x) for t, x in zip(types, parts)])
    return rows


def flt(x: str) -> float:
    return float(x)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    args = ap.parse_args()
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={args.ref}"],
                   check=True)
    rng = np.random.default_rng(2024)
    fixtures = {"graphs": {}, "cases": {}}
    with tempfile.TemporaryDirectory() as td:
        for name, cfg in GRAPHS:
            G = gen.generate(cfg)
            base = os.path.join(td, name)
            G.write_tsv(base)
            fixtures["graphs"][name] = {
                "n": G.n, "src": G.src.tolist(), "dst": G.dst.tolist(),
                "truth": G.truth.tolist(), "config": cfg.__dict__,
            }
            case = {}
            # SCC initial partition at two depths
            case["scc"] = {}
            for depth in (20, 3):
                out = run("ref_pin", ["scc", base, 1024, depth]).split("\n")
                B = int(out[0].split()[1])
                part = [int(x) for x in out[1].split()[1:]]
                case["scc"][str(depth)] = {"B": B, "part": part}
            scc_B = case["scc"]["20"]["B"]
            scc_part = np.array(case["scc"]["20"]["part"])
            # a coarse random partition too
            Bc = min(7, G.n)
            rand_part = rng.integers(0, Bc, G.n)
            rand_part[:Bc] = np.arange(Bc)
            states = {"scc": (scc_B, scc_part), "rand": (Bc, rand_part)}
            case["states"] = {}
            for sname, (B, part) in states.items():
                st = {"B": B, "part": [int(x) for x in part]}
                # dense branch (block_size 1024) and sparse branch (block_size 1)
                st["mbuild_dense"] = parse_state(run("ref_pin", ["mbuild", base, 1024],
                                                     state_stdin(B, part)))
                st["mbuild_sparse"] = parse_state(run("ref_pin", ["mbuild", base, 1],
                                                      state_stdin(B, part)))
                for binary, tag in (("ref_pin", "f32"), ("ref_pin_f64", "f64")):
                    out = run(binary, ["entropy", base, 1024], state_stdin(B, part))
                    st[f"entropy_{tag}"] = float(out.split()[1])
                    out = run(binary, ["entropy", base, 1], state_stdin(B, part))
                    st[f"entropy_sparse_{tag}"] = float(out.split()[1])
                    out = run(binary, ["merge_props", base, 1024, 7, 10], state_stdin(B, part))
                    st[f"merge_{tag}"] = parse_rows(out, (int, int, flt))
                    out = run(binary, ["nodal_props", base, 1024, 9], state_stdin(B, part))
                    st[f"nodal_{tag}"] = parse_rows(out, (int, int, int, flt, int))
                # the sparse branch of the proposals too (float build)
                out = run("ref_pin", ["merge_props", base, 1, 5, 4], state_stdin(B, part))
                st["merge_sparse_f32"] = parse_rows(out, (int, int, flt))
                out = run("ref_pin", ["nodal_props", base, 1, 6], state_stdin(B, part))
                st["nodal_sparse_f32"] = parse_rows(out, (int, int, int, flt, int))
                # merge application with distinct dS (the reference's sort is unstable)
                best = rng.integers(0, B, B)
                dS = rng.permutation(B).astype(np.float64) * 0.5 - B / 4
                btm = B // 2
                stdin = state_stdin(B, part) + f"{btm}\n" + " ".join(map(str, best)) + "\n" + \
                    " ".join(repr(float(x)) for x in dS) + "\n"
                out = run("ref_pin", ["carry", base, 1024], stdin).split("\n")
                st["carry"] = {"btm": btm, "best": best.tolist(), "dS": dS.tolist(),
                               "B": int(out[0].split()[1]),
                               "part": [int(x) for x in out[1].split()[1:]]}
                case["states"][sname] = st
            # evaluate() of the scc partition against the truth
            stdin = " ".join(map(str, G.truth)) + "\n" + " ".join(map(str, scc_part)) + "\n"
            case["evaluate_scc"] = run("ref_pin", ["evaluate", base, 1024], stdin)
            # a square contingency table (given uses exactly the truth's label
            # range): the only shape bf::evaluate handles correctly, since
            # its "un-associated columns" loop stops at the row count
            # (evaluate.hpp:93)
            sq = G.truth.copy()
            flip = rng.random(G.n) < 0.15
            sq[flip] = rng.integers(0, int(G.truth.max()) + 1, int(flip.sum()))
            sq[np.argmax(G.truth)] = int(G.truth.max())
            case["given_square"] = sq.tolist()
            stdin = " ".join(map(str, G.truth)) + "\n" + " ".join(map(str, sq)) + "\n"
            case["evaluate_square"] = run("ref_pin", ["evaluate", base, 1024], stdin)
            fixtures["cases"][name] = case
        # golden-section sequences on one graph (the bookkeeping ignores the graph)
        base = os.path.join(td, "g60")
        seqs = [
            [(40, 100.0), (20, 90.0), (10, 95.0), (15, 89.0), (12, 88.5), (13, 88.7), (11, 88.4)],
            [(64, 500.0), (32, 400.0), (16, 300.0), (8, 310.0), (12, 290.0), (10, 295.0),
             (14, 292.0), (13, 289.0)],
            [(30, 10.0), (15, 9.0), (7, 8.0), (3, 8.5), (5, 7.9), (4, 7.95), (6, 7.85)],
            [(2, 5.0), (1, 4.0)],
        ]
        fixtures["golden"] = []
        for seq in seqs:
            stdin = f"{len(seq)}\n" + "".join(f"{b} {s!r}\n" for b, s in seq)
            out = run("ref_pin", ["golden", base, 1024], stdin)
            fixtures["golden"].append({"seq": seq, "rows": parse_rows(out, (int,) * 6)})
        # full reference runs on C0 (num_batch_nodal_update 10), for statistics
        G = gen.generate(gen.config_c0(seed=0))
        base = os.path.join(td, "c0run")
        G.write_tsv(base)
        runs = []
        for i in range(8):
            pf = os.path.join(td, f"p{i}.txt")
            j = json.loads(run("ref_main", [base, 4, 10, pf]))
            part = np.loadtxt(pf, dtype=np.int64)
            j["part"] = part.tolist()
            runs.append(j)
        fixtures["c0_runs"] = runs
    with gzip.open(OUT, "wt") as f:
        json.dump(fixtures, f)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
