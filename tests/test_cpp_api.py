"""The header-only C++ API (owt-krylov_b200/include/owtk/krylov.hpp).

tests/cpp/consumer.cpp is written the way an OWT-Krylov application is
(BlockCsrMatrix, PolicyBlockOperator, Ilu0 / Jacobi / split-SSOR, gmres /
bicgstab / idrs, RCM) with the device execution policy.  On the CPU host it
must compile and link against the C ABI; on a GPU its results are compared
with the CPU oracle.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import cases
from conftest import PKG, REPO, assert_bitwise

SRC = os.path.join(REPO, "tests", "cpp", "consumer.cpp")


def build_consumer(native, out_dir):
    exe = os.path.join(out_dir, "consumer")
    cxx = shutil.which("g++") or "g++"
    lib_dir = os.path.join(PKG, "lib")
    cmd = [cxx, "-std=c++20", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(REPO, "include"),
           "-I", os.path.join(PKG, "include"), SRC, "-L", lib_dir, "-lowtk_b200", f"-Wl,-rpath,{lib_dir}", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_header_api_compiles_and_links(native, tmp_path):
    exe = build_consumer(native, str(tmp_path))
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_consumer_matches_oracle(native, restatement, tmp_path):
    import oracle
    exe = build_consumer(native, str(tmp_path))
    c = cases.lattice_case(side=24, bs=3, seed=21)
    n, bs = c["owned"], c["bs"]
    d = str(tmp_path)
    with open(os.path.join(d, "meta.txt"), "w") as f:
        f.write(f"{n} {bs} {c['cols'].size}\n")
    c["rowptr"].astype(np.uint64).tofile(os.path.join(d, "rowptr.u64"))
    c["cols"].astype(np.uint64).tofile(os.path.join(d, "cols.u64"))
    c["vals"].astype(np.float64).tofile(os.path.join(d, "vals.f64"))
    c["rhs"][: n * bs].astype(np.float64).tofile(os.path.join(d, "rhs.f64"))
    subprocess.run([exe, d], check=True, timeout=300)
    res = {}
    for line in open(os.path.join(d, "results.txt")):
        parts = line.split()
        res[parts[0]] = parts[1:]
    rhs = c["rhs"][: n * bs]
    spmv = np.fromfile(os.path.join(d, "spmv.f64"))
    assert_bitwise(spmv, restatement.bsr_spmv(n, bs, c["rowptr"], c["cols"], c["vals"], rhs), "spmv")
    mat = restatement.make_matrix("bsr", n, 0, bs, c["rowptr"], c["cols"], c["vals"])
    ilu = restatement.ilu(n, bs, c["rowptr"], c["cols"], c["vals"], 0)
    for key, solver, pck, opts, xfile in [
        ("gmres_ilu0", "gmres", "ilu", {}, "x_gmres.f64"),
        ("bicgstab_jacobi", "bicgstab", "jacobi", {"convergence_check_interval": 1}, "x_bicgstab.f64"),
        ("specwave_bicgstab_ilu0", "bicgstab", "ilu", {}, "x_specwave.f64"),
    ]:
        pc = restatement.make_pc(pck, mat, 0.0, ilu if pck == "ilu" else None)
        r, xr = restatement.solve(solver, mat, pc, oracle.default_options(**opts), rhs, np.zeros(n * bs))
        status, reason, iters = (int(v) for v in res[key][:3])
        assert status == 0 and reason == 0
        assert abs(iters - r.iterations) <= 2
        x = np.fromfile(os.path.join(d, xfile))
        assert np.linalg.norm(x - xr) <= 1e-6 * np.linalg.norm(xr)
    assert int(res["idrs_jacobi"][0]) == 0
    orp, oci, diag, off = cases.split_of(c)
    z = np.fromfile(os.path.join(d, "split_ssor.f64"))
    assert_bitwise(z, restatement.split_ssor_apply(n, bs, orp, oci, diag, off, 1.2, rhs), "split ssor")
    rcm = np.fromfile(os.path.join(d, "rcm.u64"), dtype=np.uint64).astype(np.int64)
    np.testing.assert_array_equal(rcm, restatement.rcm(n, c["rowptr"], c["cols"]))
    assert res["epochs"] == ["2"]          # GMRES sized the workspace; BiCGSTAB reused it
    assert res["ilu_updates"] == ["1"]
    assert res["layout_error"] == ["invalid_argument"]
    assert res["specwave_multigrid"] == ["invalid_argument"]
