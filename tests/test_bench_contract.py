"""bench.py on the CPU: the algorithmic byte counts behind every roofline
fraction, the peak it divides by, and the timing defaults of the contract.

The byte counts are pinned at the 2M-vertex disk mesh of the benchmark
(1,998,790 vertices, 13,990,338 block entries, bs 3): values and 32-bit
indices read once, x read once and y written once.
"""
import importlib.util
import json
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N, NNZ, BS = 1_998_790, 13_990_338, 3


@pytest.fixture(scope="module")
def bench():
    argv = sys.argv
    sys.argv = ["bench.py"]
    try:
        spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(REPO, "bench.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
    finally:
        sys.argv = argv
    return mod


def test_spmv_bytes(bench):
    vec = N * BS * 8
    expect = NNZ * (BS * 8 + 4) + (N + 1) * 4 + 2 * vec
    assert bench.kernel_bytes("spmv", N, BS, NNZ) == expect == 495_666_548
    # FP32 values and vectors, 32-bit indices unchanged.
    assert bench.kernel_bytes("spmv32", N, BS, NNZ, sv=4) == NNZ * (BS * 4 + 4) + (N + 1) * 4 + 2 * N * BS * 4


def test_dense_bytes(bench):
    # bs x bs blocks per entry: 1.17 GB in FP64, 0.62 GB in FP32.
    assert bench.kernel_bytes("dense", N, BS, NNZ) == NNZ * (BS * BS * 8 + 4) + (N + 1) * 4 + 2 * N * BS * 8
    assert round(bench.kernel_bytes("dense", N, BS, NNZ) / 1e9, 2) == 1.17
    assert round(bench.kernel_bytes("dense32", N, BS, NNZ, sv=4) / 1e9, 2) == 0.62


def test_split_bytes(bench):
    off = NNZ - N   # every row's diagonal entry moves to the diagonal array
    got = bench.kernel_bytes("split", N, BS, NNZ, off_entries=off)
    assert got == N * BS * 8 + off * (BS * 8 + 4) + (N + 1) * 4 + 2 * N * BS * 8
    assert 480e6 < got < 496e6


def test_ilu_and_reduction_bytes(bench):
    fe = NNZ   # ILU(0): the factor pattern is the matrix pattern
    assert bench.kernel_bytes("ilu", N, BS, NNZ, factor_entries=fe) == (
        fe * (BS * 8 + 4) + 2 * (N + 1) * 4 + N * 4 + N * BS * 8 + 3 * N * BS * 8)
    assert bench.kernel_bytes("dot", N, BS, NNZ, k=16) == 17 * N * BS * 8
    assert bench.kernel_bytes("norm", N, BS, NNZ) == N * BS * 8
    assert bench.kernel_bytes("axpy", N, BS, NNZ) == 3 * N * BS * 8
    with pytest.raises(ValueError):
        bench.kernel_bytes("unknown", N, BS, NNZ)


def test_peak_is_the_measured_copy_bandwidth(bench):
    peak, kind = bench.measured_peaks()
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        assert kind == "measured"
        assert peak == float(json.load(open(path))["hbm_gbs"])
    else:
        assert kind == "fallback" and peak > 0


def test_timing_defaults(bench):
    args = bench.parse([])
    # The headline: the 8M-vertex anisotropic learned-vs-plain workload.
    assert args.gpus == 1 and args.impl == "ours" and args.form == "learned"
    assert args.warmup >= 3 and args.steps >= 1
    assert args.vertices == 8_000_000 and args.seed == 4
    plain = bench.parse(["--form", "plain"])
    assert plain.vertices == 2_000_000 and plain.seed == 1


def test_gnn_layer_counts(bench):
    # One fused layer per vertex: own row 128 B read, new row 128 B written,
    # 8-slot list of 32-bit columns and BF16 weights; [h|m] (128) x Wl^T (64).
    assert bench.gnn_layer_bytes(1000) == 1000 * 304
    assert bench.gnn_layer_flops(1000) == 1000 * 2 * 128 * 64


class _System:
    owned, nnz, bs = 7_991_199, 55_938_393, 3


def test_both_arms_print_one_config(bench):
    # The driver compares the two arms' config objects key for key.
    a = bench.workload_config("learned", _System(), 1)
    b = bench.workload_config("learned", _System(), 1)
    assert a == b and a["workload"] == bench.WORKLOADS["learned"]
    assert {"workload", "vertices", "entries", "block_size", "rtol", "l2", "parallelism"} <= set(a)
    assert "iterations" not in a and "setup_s" not in a


def test_reference_arm_loads_no_project_library(tmp_path):
    """The reference arm's process (bench.py --impl reference) must map only
    the reference build: check which modules its imports pull in by running
    its system-building helpers on a tiny mesh in a child process."""
    code = r"""
import sys, os, json
sys.argv = ["bench.py"]
import importlib.util
spec = importlib.util.spec_from_file_location("b", os.path.join(%r, "bench.py"))
b = importlib.util.module_from_spec(spec); spec.loader.exec_module(b)
b.MESH_CACHE = %r
import oracle
ref = oracle.Reference()
s, _ = b.build_system("learned", 3000, 4, rcm=ref.rcm)
maps = open("/proc/self/maps").read()
print(json.dumps({"n": s.owned, "owtk_b200_so": "libowtk_b200" in maps, "meshgen_so": "meshgen.so" in maps,
                  "native_imported": "owtk_b200.native" in sys.modules}))
""" % (REPO, str(tmp_path))
    import subprocess
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True).stdout
    got = json.loads(out.strip().splitlines()[-1])
    assert got["n"] > 2000
    assert not got["owtk_b200_so"] and not got["meshgen_so"] and not got["native_imported"], got
