"""Device-resident solves through the C ABI against the reference's solves.

The device reductions sum in a different order than the reference's 8-lane
serial reduction, so the bar is: same status, the same
true-residual tolerance reached, iteration counts within +-2 (and identical
work counters whenever the iteration counts agree), and solutions equal to
the reference's to the solver tolerance.
"""
import json
import os

import numpy as np
import pytest

import cases
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

SOLVES = json.load(open(os.path.join(GOLDEN, "reference_solves.json")))
KIND = {"gmres": 0, "fgmres": 0, "bicgstab": 1, "pipelined_bicgstab": 2, "comm_hiding_bicgstab": 3, "idrs": 4}
PCK = {"identity": 0, "jacobi": 1, "ssor": 2, "ilu": 4}
COUNTERS = ["operator_applications", "preconditioner_applications", "global_reductions",
            "reorthogonalizations", "arnoldi_norm_verifications"]


def system(name, problems):
    if name == "solve24":
        c = cases.lattice_case(side=24, bs=3, seed=21)
        return c["owned"], c["bs"], c["rowptr"], c["cols"], c["vals"], c["rhs"]
    s = problems.config0()
    return s.owned, s.bs, s.rowptr, s.cols, s.vals, s.rhs


@pytest.mark.parametrize("key", sorted(SOLVES))
def test_solver_parity(native, ctx, golden, problems, key):
    spec = SOLVES[key]
    case = key.split("/")[0]
    n, bs, rp, ci, v, rhs = system(case, problems)
    m = native.Matrix(ctx, "bsr", n, 0, bs, rp, ci, v)
    pc = native.Preconditioner(m, PCK[spec["pc"]], spec["parameter"])
    b = native.Vector(ctx, n, 0, bs).upload(rhs)
    x = native.Vector(ctx, n, 0, bs)
    o = native.default_options(**spec["options"])
    r = native.solve(KIND[spec["solver"]], m, pc, b, x, o).as_dict()
    assert r["status"] == spec["status"], (r, spec)
    assert abs(r["iterations"] - spec["iterations"]) <= 2, (r["iterations"], spec["iterations"])
    if r["iterations"] == spec["iterations"]:
        for k in COUNTERS:
            assert r[k] == spec[k], (k, r[k], spec[k])
    rnorm = np.linalg.norm(rhs)
    if spec["status"] == 0:
        assert r["true_residual_norm"] <= 1e-8 * rnorm
    else:
        assert r["true_residual_norm"] == pytest.approx(spec["true_residual_norm"], rel=1e-6)
    xs = x.download()
    if case == "solve24":
        xr = golden[f"{key}/x"]
        tol = 1e-6 if spec["status"] == 0 else 1e-9
        assert np.linalg.norm(xs - xr) <= tol * np.linalg.norm(xr)
    else:
        assert np.linalg.norm(xs) == pytest.approx(spec["x_norm"], rel=1e-6)
    # The reported true residual is the one recomputed from x (test_gmres_precision.cpp:63-73).
    y = native.Vector(ctx, n, 0, bs)
    m.apply(x, y)
    assert np.linalg.norm(rhs - y.download()) == pytest.approx(r["true_residual_norm"], rel=1e-8)


def test_workspace_reuse_does_not_reallocate(native, ctx, problems):
    # tests/test_core.cpp:637-650 — allocation_epochs stays fixed across solves.
    n, bs, rp, ci, v, rhs = system("solve24", problems)
    m = native.Matrix(ctx, "bsr", n, 0, bs, rp, ci, v)
    pc = native.Preconditioner(m, native.PC_JACOBI)
    ws = native.Workspace(ctx)
    b = native.Vector(ctx, n, 0, bs).upload(rhs)
    epochs = []
    for kind in (native.BICGSTAB, native.BICGSTAB, native.FGMRES, native.FGMRES, native.BICGSTAB):
        x = native.Vector(ctx, n, 0, bs)
        r = native.solve(kind, m, pc, b, x, native.default_options(), ws)
        assert r.status == 0
        epochs.append(ws.allocation_epochs)
    assert epochs == [1, 1, 3, 3, 3]   # GMRES grows vectors and the scalar block


def test_bicgstab_workspace_slots_match_reference(native, ctx, reference):
    # tests/test_bicgstab_ilu_audit.cpp:584-587 pins the BiCGSTAB slot order.
    import oracle
    c = cases.lattice_case(side=10, bs=2, seed=5)
    n, bs = c["owned"], c["bs"]
    m = native.Matrix(ctx, "bsr", n, 0, bs, c["rowptr"], c["cols"], c["vals"])
    pc = native.Preconditioner(m, native.PC_ILU, 0)
    ws = native.Workspace(ctx)
    b = native.Vector(ctx, n, 0, bs).upload(c["rhs"])
    x = native.Vector(ctx, n, 0, bs)
    opts = dict(maximum_iterations=3, relative_tolerance=1e-14)
    native.solve(native.BICGSTAB, m, pc, b, x, native.default_options(**opts), ws)
    rm = reference.matrix("bsr", n, 0, bs, c["rowptr"], c["cols"], c["vals"])
    rp = reference.pc("ilu", rm, 0)
    rws = reference.L.ref_workspace_create()
    try:
        reference.solve("bicgstab", rm, rp, oracle.default_options(**opts), c["rhs"], np.zeros(n * bs),
                        workspace=rws)
        for slot in range(2, 8):
            mine = ws.vector_data(slot, n * bs)
            theirs = np.zeros(n * bs)
            reference.check(reference.L.ref_workspace_vector(rws, slot, theirs.ctypes.data))
            scale = max(np.abs(theirs).max(), 1e-300)
            assert np.abs(mine - theirs).max() <= 1e-11 * scale, slot
    finally:
        reference.L.ref_workspace_destroy(rws)


def test_non_finite_rhs_is_a_typed_breakdown(native, ctx):
    # tests/test_core.cpp:91-105 — infinite rhs -> breakdown(non_finite_scalar).
    m = native.Matrix(ctx, "bsr", 1, 0, 2, [0, 1], [0], [1.0, 1.0])
    for kind in (native.BICGSTAB, native.FGMRES, native.PIPELINED_BICGSTAB, native.COMM_HIDING_BICGSTAB,
                 native.IDRS):
        b = native.Vector(ctx, 1, 0, 2).upload(np.array([np.inf, 1.0]))
        x = native.Vector(ctx, 1, 0, 2)
        r = native.solve(kind, m, None, b, x, native.default_options(idr_shadow_space=2))
        assert (r.status, r.breakdown_reason) == (2, 9), kind


def test_invalid_options_leave_x_untouched(native, ctx):
    # MANUAL: invalid input returns status invalid_input and does not touch x.
    m = native.Matrix(ctx, "bsr", 2, 0, 1, [0, 1, 2], [0, 1], [2.0, 3.0])
    b = native.Vector(ctx, 2, 0, 1).upload(np.array([1.0, 1.0]))
    x = native.Vector(ctx, 2, 0, 1).upload(np.array([5.0, 6.0]))
    for bad in (dict(relative_tolerance=-1.0), dict(maximum_iterations=0), dict(convergence_check_interval=0),
                dict(breakdown_tolerance=0.0)):
        r = native.solve(native.BICGSTAB, m, None, b, x, native.default_options(**bad))
        assert r.status == 4
        assert x.download().tolist() == [5.0, 6.0]
    r = native.solve(native.FGMRES, m, None, b, x, native.default_options(restart=0))
    assert r.status == 4


def test_exact_preconditioner_converges_in_one_iteration(native, ctx):
    # tests/test_bicgstab_ilu_audit.cpp:616-631 — ILU(0) of a tridiagonal is exact.
    n = 40
    rp, ci, v = [0], [], []
    for r in range(n):
        for c in (r - 1, r, r + 1):
            if 0 <= c < n:
                ci.append(c)
                v.append(4.0 if c == r else -1.0)
        rp.append(len(ci))
    m = native.Matrix(ctx, "bsr", n, 0, 1, rp, ci, v)
    pc = native.Preconditioner(m, native.PC_ILU, 0)
    b = native.Vector(ctx, n, 0, 1).upload(np.linspace(-1, 1, n))
    x = native.Vector(ctx, n, 0, 1)
    r = native.solve(native.BICGSTAB, m, pc, b, x, native.default_options(relative_tolerance=1e-12))
    assert r.status == 0 and r.iterations == 1 and r.preconditioner_applications == 1


def test_solve_host_matches_device_solve(native, ctx, problems):
    n, bs, rp, ci, v, rhs = system("solve24", problems)
    m = native.Matrix(ctx, "bsr", n, 0, bs, rp, ci, v)
    pc = native.Preconditioner(m, native.PC_ILU, 0)
    ws = native.Workspace(ctx)
    xh = np.zeros(n * bs)
    bh = np.ascontiguousarray(rhs)
    r1 = native.solve_host(native.FGMRES, m, pc, bh.ctypes.data, xh.ctypes.data, None, ws)
    b = native.Vector(ctx, n, 0, bs).upload(rhs)
    x = native.Vector(ctx, n, 0, bs)
    r2 = native.solve(native.FGMRES, m, pc, b, x, None, ws)
    assert r1.status == r2.status == 0 and r1.iterations == r2.iterations
    assert np.array_equal(xh, x.download())


def test_float32_solve(native, ctx, problems):
    n, bs, rp, ci, v, rhs = system("solve24", problems)
    m = native.Matrix(ctx, "bsr", n, 0, bs, rp, ci, v, dtype=np.float32)
    pc = native.Preconditioner(m, native.PC_ILU, 0)
    b = native.Vector(ctx, n, 0, bs, dtype=np.float32).upload(rhs)
    x = native.Vector(ctx, n, 0, bs, dtype=np.float32)
    r = native.solve(native.FGMRES, m, pc, b, x, native.default_options(relative_tolerance=1e-5))
    assert r.status == 0
    assert r.true_residual_norm <= 1e-5 * np.linalg.norm(rhs) * 1.01


SPECWAVE = {3: ("COMM_HIDING_BICGSTAB", "SSOR"), 4: ("COMM_HIDING_BICGSTAB", "SSOR"),
            5: ("BICGSTAB", "SSOR"), 7: ("FGMRES", "SSOR"), 8: ("BICGSTAB", "SSOR"), 9: ("BICGSTAB", "ILU"),
            10: ("COMM_HIDING_BICGSTAB", "SSOR"), 11: ("BICGSTAB", "SSOR"), 12: ("PIPELINED_BICGSTAB", "SSOR"),
            13: ("BICGSTAB", "ILU"), 14: ("IDRS", "SSOR"), 15: ("PIPELINED_BICGSTAB", "SSOR"),
            21: ("PIPELINED_BICGSTAB", "ILU"), 22: ("COMM_HIDING_BICGSTAB", "SSOR")}


@pytest.mark.parametrize("solver_id", sorted(SPECWAVE))
def test_specwave_dispatch_matches_direct_calls(native, ctx, solver_id):
    # specwave_compat.hpp:99-249: each legacy id is the named solver with the
    # named preconditioner (SSOR omega = options.relaxation, ILU(0)) and reduction.
    c = cases.lattice_case(side=20, bs=3, seed=21)
    n, bs = c["owned"], c["bs"]
    m = native.Matrix(ctx, "bsr", n, 0, bs, c["rowptr"], c["cols"], c["vals"])
    b = native.Vector(ctx, n, 0, bs).upload(c["rhs"][: n * bs])
    opts = native.default_options(relaxation=1.2, residual_replacement_interval=0 if solver_id == 4 else 50)
    x1, x2 = native.Vector(ctx, n, 0, bs), native.Vector(ctx, n, 0, bs)
    r1 = native.solve_specwave(solver_id, m, b, x1, opts)
    kind, pck = SPECWAVE[solver_id]
    pc = native.Preconditioner(m, getattr(native, "PC_" + pck), 1.2 if pck == "SSOR" else 0)
    direct = native.default_options(relaxation=1.2, residual_replacement_interval=50)
    # specwave_compat.hpp:157-176, :223-243: id 10 reduces in mixed precision,
    # id 22 with compensation.
    reduction = {10: "mixed", 22: "compensated"}.get(solver_id, "serial")
    r2 = native.solve_ex(getattr(native, kind), m, pc, b, x2, direct, reduction=reduction)
    d1, d2 = r1.as_dict(), r2.as_dict()
    d1.pop("solve_seconds", None)
    d2.pop("solve_seconds", None)
    assert d1 == d2
    assert np.array_equal(x1.download().view(np.uint64), x2.download().view(np.uint64))


def test_specwave_petsc_and_rejected_ids(native, ctx):
    c = cases.lattice_case(side=8, bs=3, seed=21)
    n, bs = c["owned"], c["bs"]
    m = native.Matrix(ctx, "bsr", n, 0, bs, c["rowptr"], c["cols"], c["vals"])
    b = native.Vector(ctx, n, 0, bs).upload(c["rhs"][: n * bs])
    x = native.Vector(ctx, n, 0, bs)
    r = native.solve_specwave(6, m, b, x)
    assert r.status == 4 and np.isnan(r.true_residual_norm)      # default SolverResult
    for sid in (0, 1, 2, 16, 17, 18, 19, 20, 23, -1):
        with pytest.raises(native.OwtkError):
            native.solve_specwave(sid, m, b, x)
