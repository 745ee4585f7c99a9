"""C ABI checks that need no GPU: the library loads, exports every entry point
include/usap.h declares, its host-side evaluation matches the oracle, and
errors come back as status codes."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from usap_b200 import native as nat

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "usap.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)     # drop comments
    return sorted(set(re.findall(r"\b(usap_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = nat.lib()
    declared = _declared()
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(L, name), name
    assert sorted(nat.EXPORTS) == declared


_MIRRORS = {"usap_graph": "Graph", "usap_params": "Params", "usap_result": "Result",
            "usap_scores": "Scores", "usap_trace_event": "TraceEvent", "usap_batch_job": "BatchJob",
            "usap_batch_stats": "BatchStats", "usap_server_config": "ServerConfig",
            "usap_server_timing": "ServerTiming", "usap_server_stats": "ServerStats"}


def test_struct_layout_matches_header(tmp_path):
    """The Python mirrors of include/usap.h's structs have the header's
    size and every field at the header's offset (a C probe compiled with
    the host compiler prints them)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "usap.h"', "int main(void) {"]
    for cname, pname in _MIRRORS.items():
        lines.append(f'  printf("{cname} . %zu\\n", sizeof({cname}));')
        for f, _ in getattr(nat, pname)._fields_:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    seen = 0
    for line in filter(None, out):
        cname, field, value = line.split()
        st = getattr(nat, _MIRRORS[cname])
        got = C.sizeof(st) if field == "." else getattr(st, field).offset
        assert got == int(value), (cname, field, got, int(value))
        seen += 1
    assert seen == sum(1 + len(getattr(nat, p)._fields_) for p in _MIRRORS.values())


def test_version_and_defaults():
    L = nat.lib()
    assert b"sm_100a" in L.usap_version()
    p = nat.default_params()
    # the reference's defaults (graph_parallel.hpp:40-52)
    assert p.beta == 3 and p.block_size == 1024 and p.num_agg_proposals_per_block == 10
    assert abs(p.num_block_reduction_rate - 0.5) < 1e-7 and p.max_num_nodal_itr == 100
    assert p.num_batch_nodal_update == 4 and p.delta_entropy_moving_avg_window == 3
    assert p.delta_entropy_threshold1 == 5e-4 and p.delta_entropy_threshold2 == 1e-4
    assert p.dfs_depth == 20 and p.t_block_num == 20


def test_evaluate_matches_oracle(oracle):
    rng = np.random.default_rng(5)
    for n, b1, b2 in ((500, 7, 7), (1000, 11, 25), (300, 9, 3)):
        truth = rng.integers(0, b1, n).astype(np.int32)
        given = np.where(rng.random(n) < 0.7, truth % b2, rng.integers(0, b2, n)).astype(np.int32)
        from usap_b200.api import evaluate
        mine = evaluate(truth, given)
        ref = oracle.evaluate(truth, given)
        for k in ("rand_index", "adjusted_rand_index", "adjusted_rand_index_exact",
                  "pairwise_recall", "pairwise_precision", "h_truth", "h_given",
                  "h_truth_given", "h_given_truth", "mi", "nmi", "nmi_sqrt", "missed_info",
                  "erroneous_info"):
            assert abs(mine[k] - ref[k]) <= 1e-12 * max(1.0, abs(ref[k])), k
        assert mine["n"] == ref["n"]


def test_evaluate_accuracy_is_optimal_matching():
    from usap_b200.api import evaluate
    truth = np.array([0, 0, 0, 1, 1, 2, 2, 2, 2], np.int32)
    given = np.array([2, 2, 1, 0, 0, 1, 1, 1, 2], np.int32)
    s = evaluate(truth, given)
    # best matching: 0->2 (2), 1->0 (2), 2->1 (3) = 7 of 9
    assert abs(s["accuracy"] - 7 / 9) < 1e-12


def test_evaluate_rejects_bad_input():
    L = nat.lib()
    t = np.zeros(1, np.int32)
    rc = L.usap_evaluate(nat.p32(t), nat.p32(t), 1, C.byref(nat.Scores()))
    assert rc == -1 and L.usap_last_error()
    rc = L.usap_evaluate(None, nat.p32(t), 1, C.byref(nat.Scores()))
    assert rc == -1


def test_null_arguments_are_errors_not_crashes():
    L = nat.lib()
    assert L.usap_partition(None, None, None, None) == -1
    assert L.usap_ctx_load(None, None) == -1
    assert L.usap_ctx_partition(None, None, None, None) == -1
    assert L.usap_op_build(None, None, 1, 0, None, None, None) == -1


def test_no_device_is_reported(monkeypatch):
    """Without a visible GPU the context refuses with USAP_ERR_NO_DEVICE or
    USAP_ERR_CUDA (never a crash)."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is visible")
    except ImportError:
        pass
    h = C.c_void_p()
    rc = nat.lib().usap_ctx_create(0, C.byref(h))
    assert rc in (-5, -2)
    assert nat.lib().usap_last_error()


def test_batch_rejects_bad_job_index():
    import ctypes as C
    src = np.array([0, 1], np.int32)
    dst = np.array([1, 0], np.int32)
    g, keep = nat.make_graph(src, dst)
    garr = (nat.Graph * 1)(g)
    jobs = (nat.BatchJob * 1)()
    jobs[0].graph = 3
    rc = nat.lib().usap_batch_partition(garr, 1, None, jobs, 1, 0, 0, C.byref(nat.BatchStats()))
    assert rc == -1


def test_server_null_and_no_device():
    """The service's entry points reject null handles, and without a GPU
    usap_server_create reports the missing device instead of crashing."""
    L = nat.lib()
    assert L.usap_server_submit(None, None, None, None, None) == -1
    done = C.c_int32()
    assert L.usap_server_poll(None, 1, C.byref(done), None, None) == -1
    assert L.usap_server_wait(None, 1, None, None) == -1
    assert L.usap_server_get_stats(None, None) == -1
    L.usap_server_destroy(None)
    try:
        import torch
        if torch.cuda.is_available():
            return
    except ImportError:
        pass
    h = C.c_void_p()
    cfg = nat.ServerConfig()
    L.usap_server_config_default(C.byref(cfg))
    rc = L.usap_server_create(C.byref(cfg), C.byref(h))
    assert rc in (-5, -2) and not h.value
    assert L.usap_last_error()
