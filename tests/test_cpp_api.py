"""The header-only C++ API (owt-krylov_b200/include/owtk/krylov.hpp).

tests/cpp/consumer.cpp is written the way an OWT-Krylov application is
(BlockCsrMatrix, PolicyBlockOperator, Ilu0 / Jacobi / split-SSOR, gmres /
bicgstab / idrs, the stability variants, an ArnoldiSnapshot, an application
convergence test, its own matrix-free operator and preconditioner types, the
free BLAS-1 functions and the three reduction classes, RCM) with the device
execution policy.  On the CPU host it
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
    rows_out = np.fromfile(os.path.join(d, "spmv_rows.f64")).reshape(n, bs)
    listed = np.arange(n) % 3 == 0
    assert_bitwise(rows_out[listed], spmv.reshape(n, bs)[listed], "apply_rows, listed rows")
    assert (rows_out[~listed] == 7.0).all(), "apply_rows touched a row it was not given"
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
    # The stability variants against the reference's solve with the same
    # options and reduction (krylov_solvers.hpp:766-809, pipelined_bicgstab.hpp:275-313, :620-661).
    reference = oracle.Reference()
    rm = reference.matrix("bsr", n, 0, bs, c["rowptr"], c["cols"], c["vals"])
    rilu = reference.pc("ilu", rm, 0)
    for name, solver, reduction, interval in [
        ("bicgstab_stable", "bicgstab", "mixed", None),
        ("bicgstab_residual_replacement", "bicgstab", "serial", 7),
        ("bicgstab_mixed_precision", "bicgstab", "mixed", None),
        ("pipelined_bicgstab_stable", "pipelined_bicgstab", "mixed", None),
        ("pipelined_bicgstab_residual_replacement", "pipelined_bicgstab", "serial", 7),
        ("pipelined_bicgstab_mixed_precision", "pipelined_bicgstab", "mixed", None),
        ("communication_hiding_bicgstab_stable", "comm_hiding_bicgstab", "mixed", None),
        ("communication_hiding_bicgstab_residual_replacement", "comm_hiding_bicgstab", "serial", 7),
        ("communication_hiding_bicgstab_mixed_precision", "comm_hiding_bicgstab", "mixed", None),
    ]:
        opts = {} if interval is None else {"residual_replacement_interval": interval}
        rr, xr, _ = reference.solve_ex(solver, rm, rilu, oracle.default_options(**opts), rhs, np.zeros(n * bs),
                                       reduction=reduction)
        status, reason, iters = (int(v) for v in res[name][:3])
        assert status == int(rr.status) == 0, name
        assert abs(iters - int(rr.iterations)) <= 2, (name, iters, rr.iterations)
        x = np.fromfile(os.path.join(d, f"x_{name}.f64"))
        assert np.linalg.norm(x - xr) <= 1e-6 * np.linalg.norm(xr), name
    # FGMRES(6) with an Arnoldi snapshot: the reference's last cycle.
    rr, _, snap = reference.solve_ex("gmres", rm, rilu, oracle.default_options(restart=6), rhs, np.zeros(n * bs),
                                     snapshot=True)
    assert int(res["fgmres_snapshot"][2]) == int(rr.iterations)
    cols = int(res["snapshot_columns"][0])
    assert cols == snap["columns"] > 0
    h = np.fromfile(os.path.join(d, "snapshot_h.f64"))
    want = np.concatenate([snap["h"][: c + 2, c] for c in range(cols)])
    # Restarted cycles carry the reductions' rounding differences forward.
    np.testing.assert_allclose(h, want, rtol=1e-7, atol=1e-12)
    z = np.fromfile(os.path.join(d, "snapshot_basis.f64")).reshape(cols, n * bs)
    assert np.linalg.norm(z - snap["basis"]) <= 1e-7 * np.linalg.norm(snap["basis"])
    assert res["snapshot_range"] == ["out_of_range"]
    # The application convergence test stopping BiCGSTAB at iteration 5.
    rr, xr, _ = reference.solve_ex("bicgstab", rm, rilu, oracle.default_options(), rhs, np.zeros(n * bs), stop_at=5)
    got = [int(v) for v in res["bicgstab_application_test"][:6]]
    assert got[:2] == [0, 0] and got[2:] == [int(rr.iterations), int(rr.operator_applications),
                                             int(rr.preconditioner_applications), int(rr.global_reductions)]
    assert res["application"] == ["1", "6"] and int(rr.converged_by_application) == 1
    # The application's own operator and preconditioner types give the
    # device matrix and Jacobi's bits.
    assert res["bicgstab_matrix_free"][:3] == res["bicgstab_jacobi"][:3]
    assert_bitwise(np.fromfile(os.path.join(d, "x_matrix_free.f64")), np.fromfile(os.path.join(d, "x_bicgstab.f64")),
                   "matrix-free solve")
    # Owned-only BLAS-1 with the reference's rounding (no contraction).
    u0 = 0.25 * (np.arange(n * bs) % 17).astype(np.float64) - 1.5
    u = (u0 + 0.37 * rhs) * -1.7
    assert_bitwise(np.fromfile(os.path.join(d, "blas_u.f64")), u, "axpy + scale")
    assert_bitwise(np.fromfile(os.path.join(d, "blas_w.f64")), 0.5 * rhs + (-1.25) * u, "assign_linear_combination")
    # Reductions: the reference's three classes on the same pair.
    hexv = {k: float.fromhex(res[k][0]) for k in ("dot_serial", "dot_compensated", "dot_mixed", "norm_mixed")}
    ulp = np.spacing(abs(float(rhs @ u)))
    assert abs(hexv["dot_serial"] - reference.dot_kind("serial", n, 0, bs, rhs, u)[0]) <= 64 * ulp
    assert abs(hexv["dot_compensated"] - reference.dot_kind("compensated", n, 0, bs, rhs, u)[0]) <= 2 * ulp
    assert abs(hexv["dot_mixed"] - reference.dot_kind("mixed", n, 0, bs, rhs, u)[0]) <= ulp
    nm = reference.norm_kind("mixed", n, 0, bs, u)
    assert abs(hexv["norm_mixed"] - nm) <= np.spacing(nm)
    assert res["epochs"] == ["2"]          # GMRES sized the workspace; BiCGSTAB reused it
    assert res["ilu_updates"] == ["1"]
    assert res["layout_error"] == ["invalid_argument"]
    assert res["specwave_multigrid"] == ["invalid_argument"]
