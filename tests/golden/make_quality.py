"""Record the solve quality of the reference's own partition() on seeded graphs.

The reference seeds its engines from std::random_device, so its solves are
compared by distribution: for every graph below this script runs
``oracle/_ref/ref_main`` (uSAP's include/graph_parallel.hpp compiled
unmodified against the Taskflow-API shim, ``make -C oracle ref``) several
times with num_batch_nodal_update = 10, as main.cpp:47-62 does, and records
the final block count B and the NMI against the planted partition
(2 MI / (H_truth + H_given), computed here in numpy).

Graphs (usap_b200.generator):
* c1_*   N=5000, 19 planted blocks, the four {within, alpha} variants, seed 0
* n20k   N=20000, 32 planted blocks, within 0.5, alpha 1 (a reduced-N stand-in
         for the N=50000 graph, which takes a minute per reference run)
* c2     N=50000, 44 planted blocks, within 0.5, alpha 1 (seed 0)

Writes tests/golden/ref_quality.json, read by tests/test_gpu_quality.py.
Needs the reference binary; it is run by hand (about 20 minutes on 8 cores).

usage: python tests/golden/make_quality.py [--threads T] [--only name,...]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from usap_b200 import generator as gen  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "ref_quality.json")
REF_MAIN = os.path.join(ROOT, "oracle", "_ref", "ref_main")

GRAPHS = {
    "c1_f0.8_a10": (gen.config_c1(0.8, 10.0, 0), 8),
    "c1_f0.5_a10": (gen.config_c1(0.5, 10.0, 0), 8),
    "c1_f0.8_a1": (gen.config_c1(0.8, 1.0, 0), 8),
    "c1_f0.5_a1": (gen.config_c1(0.5, 1.0, 0), 8),
    "n20k": (gen.SBMConfig(n=20000, blocks=32, within=0.5, alpha=1.0, seed=0), 12),
    "c2": (gen.config_c2(0), 16),
}


def nmi(truth: np.ndarray, given: np.ndarray) -> float:
    """2 MI / (H_truth + H_given) of two labelings (natural logs)."""
    t = np.unique(truth, return_inverse=True)[1]
    g = np.unique(given, return_inverse=True)[1]
    n = t.size
    cell = np.unique(t.astype(np.int64) * (int(g.max()) + 1) + g, return_counts=True)[1] / n
    pt, pg = np.bincount(t) / n, np.bincount(g) / n
    h_t, h_g = -float(np.sum(pt * np.log(pt))), -float(np.sum(pg * np.log(pg)))
    mi = h_t + h_g + float(np.sum(cell * np.log(cell)))
    return 2.0 * mi / (h_t + h_g) if h_t + h_g > 0 else 1.0


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--only", default="")
    args = ap.parse_args()
    names = [n for n in GRAPHS if not args.only or n in args.only.split(",")]
    out = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            out = json.load(f)
    with tempfile.TemporaryDirectory() as td:
        for name in names:
            cfg, runs = GRAPHS[name]
            G = gen.generate(cfg)
            base = os.path.join(td, name)
            G.write_tsv(base)
            rec = []
            for k in range(runs):
                pf = os.path.join(td, f"{name}_{k}.txt")
                p = subprocess.run([REF_MAIN, base, str(args.threads), "10", pf], capture_output=True,
                                   text=True, timeout=3600)
                if p.returncode != 0:
                    raise RuntimeError(f"ref_main failed on {name}: {p.stderr[:300]}")
                j = json.loads(p.stdout.strip().splitlines()[-1])
                part = np.loadtxt(pf, dtype=np.int64)
                rec.append({"B": int(j["B"]), "nmi": nmi(G.truth, part), "seconds": j["ms"] / 1000.0})
                print(name, k, rec[-1], flush=True)
            out[name] = {"config": {"n": cfg.n, "blocks": cfg.blocks, "within": cfg.within, "alpha": cfg.alpha,
                                    "seed": cfg.seed},
                         "threads": args.threads, "num_batch_nodal_update": 10, "runs": rec}
            with open(OUT, "w") as f:
                json.dump(out, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
