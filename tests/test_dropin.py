"""The reference-shaped C++ headers (include/usap/graph_p.hpp,
include/usap/evaluate.hpp) compile and link against the library, and a
driver written against them gives the same partition as the C ABI."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "drop_in", "dropin_main.cpp")


def _build(tmp_path):
    exe = str(tmp_path / "dropin_main")
    lib_dir = os.path.join(ROOT, "usap_b200")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
                    "-L", lib_dir, "-lusap_b200", f"-Wl,-rpath,{lib_dir}"], check=True)
    return exe


def test_dropin_compiles_and_links(tmp_path):
    exe = _build(tmp_path)
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_dropin_matches_c_abi(tmp_path):
    from usap_b200 import api, generator as gen, native as nat
    exe = _build(tmp_path)
    G = gen.generate(gen.SBMConfig(n=800, blocks=6, within=0.8, alpha=5, seed=21))
    base = str(tmp_path / "g")
    G.write_tsv(base)
    out = str(tmp_path / "p.txt")
    r = subprocess.run([exe, base, out, "10"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "Number of nodes: 800" in r.stdout and "Normalized mutual info" in r.stdout
    part_cpp = np.loadtxt(out, dtype=np.int64)
    # same graph through the Python front end (file read back, 1-based ids)
    g2 = gen.read_tsv(base)
    part_py, _ = api.partition(g2.src, g2.dst, g2.weight, g2.n,
                               params=nat.default_params(num_batch_nodal_update=10))
    assert np.array_equal(part_cpp, part_py)
