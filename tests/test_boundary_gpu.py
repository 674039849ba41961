"""The parts of the reference's solver interface beyond the plain solve,
through the C ABI, against the reference itself (oracle/_ref):

* the compensated and mixed-precision reductions (reduction.hpp:175-299) on
  ill-conditioned dot products, judged by their distance from the exact sum;
* SolverOptions::convergence_test (core.hpp:102-108, krylov_solvers.hpp:122-143)
  in every solver: the same iteration, work counters and
  converged_by_application as the reference;
* the FGMRES ArnoldiSnapshot (core.hpp:462-534): the same columns,
  Hessenberg entries and preconditioned basis as the reference's;
* the stability variants' reductions and options (krylov_solvers.hpp:766-809,
  pipelined_bicgstab.hpp:275-313, :620-661);
* host-callback operators and preconditioners (the duck-typed Operator and
  Preconditioner of docs/MANUAL.tex:676-712);
* every SpecWave id of the device path against the reference's own
  solve_specwave_native (specwave_compat.hpp:99-249).
"""
from fractions import Fraction

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

KIND = {"gmres": 0, "bicgstab": 1, "pipelined_bicgstab": 2, "comm_hiding_bicgstab": 3, "idrs": 4}
COUNTERS = ["iterations", "operator_applications", "preconditioner_applications", "global_reductions"]


@pytest.fixture(scope="module")
def lattice():
    return cases.lattice_case(side=24, bs=3, seed=21)


def _ulp(x):
    return np.spacing(abs(x)) if x != 0 else np.finfo(float).tiny


def _ill_conditioned(n, seed, cond_exp=10):
    """Pairs (a, b) whose dot product cancels to about 10^-cond_exp of sum |a b|."""
    rng = np.random.default_rng(seed)
    half = n // 2
    a1 = rng.uniform(-1, 1, half) * 2.0 ** rng.integers(-20, 20, half)
    b1 = rng.uniform(-1, 1, half)
    a2 = -a1 * (1 + rng.uniform(-1, 1, half) * 10.0 ** (-cond_exp))
    a = np.concatenate([a1, a2])
    b = np.concatenate([b1, b1])
    p = rng.permutation(a.size)
    return a[p], b[p]


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_accurate_dots_against_exact_sums(native, ctx, reference, seed):
    n = 6000
    a, b = _ill_conditioned(n, seed)
    va = native.Vector(ctx, n, 0, 1).upload(a)
    vb = native.Vector(ctx, n, 0, 1).upload(b)
    exact = sum(Fraction(x) * Fraction(y) for x, y in zip(a.tolist(), b.tolist()))
    exact_rounded_products = sum(Fraction(float(x * y)) for x, y in zip(a.tolist(), b.tolist()))
    e_f, er_f = float(exact), float(exact_rounded_products)
    serial, _ = native.dot_ex(va, vb, "serial")
    comp, _ = native.dot_ex(va, vb, "compensated")
    mixed, mixed_lo = native.dot_ex(va, vb, "mixed")
    ref_comp, _ = reference.dot_kind("compensated", n, 0, 1, a, b)
    ref_mixed, _ = reference.dot_kind("mixed", n, 0, 1, a, b)
    # Compensated: the rounded products summed about as exactly as the
    # reference's sequential Neumaier sum.
    assert abs(comp - er_f) <= 2 * abs(ref_comp - er_f) + 2 * _ulp(er_f)
    # Mixed precision (Dot2): within one rounding of the exact dot, at least
    # as close as the reference's long double sum; hi + lo carries the pair.
    assert abs(mixed - e_f) <= max(abs(ref_mixed - e_f), _ulp(e_f))
    assert abs(Fraction(mixed) + Fraction(mixed_lo) - exact) <= abs(Fraction(mixed) - exact)
    # The plain serial sum is far less accurate on this input, which is what
    # the two accurate reductions are for.
    assert abs(serial - e_f) > abs(mixed - e_f)


def test_accurate_norms(native, ctx, reference):
    rng = np.random.default_rng(7)
    v = rng.normal(size=5000) * 2.0 ** rng.integers(-30, 30, 5000)
    x = native.Vector(ctx, v.size, 0, 1).upload(v)
    exact_sq = sum(Fraction(t) ** 2 for t in v.tolist())
    # sqrt of the exact sum of squares, correctly rounded to double
    r = float(exact_sq) ** 0.5
    for _ in range(3):
        r = float((Fraction(r) + exact_sq / Fraction(r)) / 2)
    mixed = native.norm_ex(x, "mixed")
    assert abs(mixed - r) <= _ulp(r)
    assert abs(mixed - reference.norm_kind("mixed", v.size, 0, 1, v)) <= 2 * _ulp(r)
    comp = native.norm_ex(x, "compensated")
    assert comp == pytest.approx(reference.norm_kind("compensated", v.size, 0, 1, v), rel=4e-16)
    # Special values as the reference's scaled norm (reduction.hpp:64-89).
    for special in (np.inf, np.nan):
        w = v.copy()
        w[17] = special
        x.upload(w)
        got = native.norm_ex(x, "mixed")
        want = reference.norm_kind("mixed", w.size, 0, 1, w)
        assert (np.isnan(got) and np.isnan(want)) or got == want
    x.upload(np.zeros_like(v))
    assert native.norm_ex(x, "mixed") == 0.0


def _system(native, ctx, reference, c, pc_kind):
    n, bs = c["owned"], c["bs"]
    m = native.Matrix(ctx, "bsr", n, 0, bs, c["rowptr"], c["cols"], c["vals"])
    pc = native.Preconditioner(m, {"jacobi": native.PC_JACOBI, "ilu": native.PC_ILU}[pc_kind], 0)
    rm = reference.matrix("bsr", n, 0, bs, c["rowptr"], c["cols"], c["vals"])
    rpc = reference.pc(pc_kind, rm, 0)
    return m, pc, rm, rpc


@pytest.mark.parametrize("solver", sorted(KIND))
@pytest.mark.parametrize("reduction", ["serial", "compensated", "mixed"])
def test_solvers_with_each_reduction(native, ctx, reference, lattice, solver, reduction):
    import oracle
    c = lattice
    n, bs = c["owned"], c["bs"]
    m, pc, rm, rpc = _system(native, ctx, reference, c, "jacobi")
    b = native.Vector(ctx, n, 0, bs).upload(c["rhs"])
    x = native.Vector(ctx, n, 0, bs)
    opts = dict(convergence_check_interval=1, idr_shadow_space=2)
    r = native.solve_ex(KIND[solver], m, pc, b, x, native.default_options(**opts), reduction=reduction)
    rr, xr, _ = reference.solve_ex(solver, rm, rpc, oracle.default_options(**opts), c["rhs"], np.zeros(n * bs),
                                   reduction=reduction)
    assert r.status == rr.status == 0
    assert abs(int(r.iterations) - int(rr.iterations)) <= 2
    assert r.true_residual_norm <= 1e-8 * np.linalg.norm(c["rhs"])
    xs = x.download()
    assert np.linalg.norm(xs - xr) <= 1e-6 * np.linalg.norm(xr)


@pytest.mark.parametrize("solver", sorted(KIND))
def test_convergence_test_callback(native, ctx, reference, lattice, solver):
    """The application stops every solver at iteration 5: same iteration,
    same counters, converged_by_application, same candidate passed in."""
    import oracle
    c = lattice
    n, bs = c["owned"], c["bs"]
    m, pc, rm, rpc = _system(native, ctx, reference, c, "ilu")
    b = native.Vector(ctx, n, 0, bs).upload(c["rhs"])
    x = native.Vector(ctx, n, 0, bs)
    seen = []

    def stop_at_five(iteration, candidate):
        seen.append((iteration, float(np.linalg.norm(candidate))))
        return iteration >= 5

    opts = dict(idr_shadow_space=2)
    r = native.solve_ex(KIND[solver], m, pc, b, x, native.default_options(**opts), convergence_test=stop_at_five)
    rr, xr, _ = reference.solve_ex(solver, rm, rpc, oracle.default_options(**opts), c["rhs"], np.zeros(n * bs),
                                   stop_at=5)
    assert r.converged_by_application == rr.converged_by_application == 1
    assert r.status == rr.status == 0
    for k in COUNTERS:
        assert getattr(r, k) == getattr(rr, k), (k, getattr(r, k), getattr(rr, k))
    assert seen[0] == (0, 0.0) and seen[-1][0] == int(rr.iterations)
    xs = x.download()
    assert np.linalg.norm(xs - xr) <= 1e-9 * np.linalg.norm(xr)
    assert r.true_residual_norm == pytest.approx(rr.true_residual_norm, rel=1e-8)


def test_convergence_test_error_propagates(native, ctx, lattice):
    c = lattice
    n, bs = c["owned"], c["bs"]
    m = native.Matrix(ctx, "bsr", n, 0, bs, c["rowptr"], c["cols"], c["vals"])
    b = native.Vector(ctx, n, 0, bs).upload(c["rhs"])
    x = native.Vector(ctx, n, 0, bs)

    def failing(iteration, candidate):
        raise KeyError("application failure")

    with pytest.raises(KeyError):
        native.solve_ex(native.BICGSTAB, m, None, b, x, native.default_options(), convergence_test=failing)


@pytest.mark.parametrize("restart", [6, 30])
def test_arnoldi_snapshot(native, ctx, reference, lattice, restart):
    import oracle
    c = lattice
    n, bs = c["owned"], c["bs"]
    m, pc, rm, rpc = _system(native, ctx, reference, c, "ilu")
    b = native.Vector(ctx, n, 0, bs).upload(c["rhs"])
    x = native.Vector(ctx, n, 0, bs)
    snap = native.ArnoldiSnapshot(ctx)
    r = native.solve_ex(native.FGMRES, m, pc, b, x, native.default_options(restart=restart), snapshot=snap)
    rr, _, ref = reference.solve_ex("gmres", rm, rpc, oracle.default_options(restart=restart), c["rhs"],
                                    np.zeros(n * bs), snapshot=True)
    assert r.iterations == rr.iterations
    assert snap.columns == ref["columns"] > 0
    for col in range(snap.columns):
        for row in range(col + 2):
            # Restarted cycles carry the reductions' rounding differences
            # forward (device and reference sum in different orders).
            assert snap.h_entry(row, col) == pytest.approx(ref["h"][row, col], rel=1e-7, abs=1e-12)
        z = snap.basis(col, n, 0, bs)
        assert np.linalg.norm(z - ref["basis"][col]) <= 1e-7 * np.linalg.norm(ref["basis"][col])
    with pytest.raises(native.OwtkError) as e:
        snap.h_entry(0, snap.columns)
    assert e.value.kind == "out_of_range"
    with pytest.raises(native.OwtkError):
        snap.basis(snap.columns, n, 0, bs)
    # A solve that converges at once clears the snapshot (krylov_solvers.hpp:219-224).
    x.upload(x.download())
    native.solve_ex(native.FGMRES, m, pc, b, x, native.default_options(restart=restart), snapshot=snap)
    assert snap.columns == 0


@pytest.mark.parametrize("variant,solver,reduction,interval", [
    ("bicgstab_stable", "bicgstab", "mixed", None),
    ("bicgstab_residual_replacement", "bicgstab", "serial", 7),
    ("bicgstab_mixed_precision", "bicgstab", "mixed", None),
    ("pipelined_bicgstab_stable", "pipelined_bicgstab", "mixed", None),
    ("pipelined_bicgstab_residual_replacement", "pipelined_bicgstab", "serial", 7),
    ("pipelined_bicgstab_mixed_precision", "pipelined_bicgstab", "mixed", None),
    ("communication_hiding_bicgstab_stable", "comm_hiding_bicgstab", "mixed", None),
    ("communication_hiding_bicgstab_residual_replacement", "comm_hiding_bicgstab", "serial", 7),
    ("communication_hiding_bicgstab_mixed_precision", "comm_hiding_bicgstab", "mixed", None),
])
def test_stability_variants(native, ctx, reference, lattice, variant, solver, reduction, interval):
    """What each named variant runs (the header forwards to these options and
    reductions): against the reference's own solve with the same choices."""
    import oracle
    c = lattice
    n, bs = c["owned"], c["bs"]
    m, pc, rm, rpc = _system(native, ctx, reference, c, "ilu")
    opts = {} if interval is None else {"residual_replacement_interval": interval}
    b = native.Vector(ctx, n, 0, bs).upload(c["rhs"])
    x = native.Vector(ctx, n, 0, bs)
    r = native.solve_ex(KIND[solver], m, pc, b, x, native.default_options(**opts), reduction=reduction)
    rr, xr, _ = reference.solve_ex(solver, rm, rpc, oracle.default_options(**opts), c["rhs"], np.zeros(n * bs),
                                   reduction=reduction)
    assert r.status == rr.status == 0, variant
    assert abs(int(r.iterations) - int(rr.iterations)) <= 2, variant
    assert np.linalg.norm(x.download() - xr) <= 1e-6 * np.linalg.norm(xr)


def test_callback_operator_and_preconditioner(native, ctx, restatement, lattice):
    """A matrix-free operator and a host Jacobi preconditioner supplied as
    Python functions give the same solve as the device matrix and Jacobi."""
    c = lattice
    n, bs = c["owned"], c["bs"]
    calls = {"op": 0, "pc": 0}
    inv = 1.0 / np.concatenate([c["vals"].reshape(-1, bs)[c["rowptr"][i]:c["rowptr"][i + 1]][
        c["cols"][c["rowptr"][i]:c["rowptr"][i + 1]] == i][0] for i in range(n)])

    def op(vin, vout):
        calls["op"] += 1
        vout[: n * bs] = restatement.bsr_spmv(n, bs, c["rowptr"], c["cols"], c["vals"], vin[: n * bs].copy())

    def jacobi(vin, vout):
        calls["pc"] += 1
        vout[: n * bs] = inv * vin[: n * bs]

    A = native.CallbackOperator(ctx, n, 0, bs, op)
    M = native.CallbackPreconditioner(ctx, n, 0, bs, jacobi)
    b = native.Vector(ctx, n, 0, bs).upload(c["rhs"])
    x = native.Vector(ctx, n, 0, bs)
    o = native.default_options(convergence_check_interval=1)
    r = native.solve_ex(native.BICGSTAB, A, M, b, x, o)
    dm = native.Matrix(ctx, "bsr", n, 0, bs, c["rowptr"], c["cols"], c["vals"])
    dj = native.Preconditioner(dm, native.PC_JACOBI, 0)
    x2 = native.Vector(ctx, n, 0, bs)
    r2 = native.solve(native.BICGSTAB, dm, dj, b, x2, o)
    assert r.status == r2.status == 0
    assert r.iterations == r2.iterations
    assert calls["op"] == r.operator_applications and calls["pc"] == r.preconditioner_applications
    np.testing.assert_array_equal(x.download(), x2.download())
    # Preconditioners that need coefficients reject a callback operator.
    with pytest.raises(native.OwtkError):
        native.Preconditioner(A, native.PC_JACOBI, 0)
    with pytest.raises(native.OwtkError):
        native.Preconditioner(A, native.PC_ILU, 0)


SPECWAVE_IDS = [3, 4, 5, 7, 8, 9, 10, 11, 12, 13, 14, 15, 21, 22]


@pytest.mark.parametrize("solver_id", SPECWAVE_IDS)
def test_specwave_ids_against_reference(native, ctx, reference, lattice, solver_id):
    import oracle
    c = lattice
    n, bs = c["owned"], c["bs"]
    m = native.Matrix(ctx, "bsr", n, 0, bs, c["rowptr"], c["cols"], c["vals"])
    rm = reference.matrix("bsr", n, 0, bs, c["rowptr"], c["cols"], c["vals"])
    opts = dict(relaxation=1.1, idr_shadow_space=2, maximum_iterations=400)
    b = native.Vector(ctx, n, 0, bs).upload(c["rhs"])
    x = native.Vector(ctx, n, 0, bs)
    r = native.solve_specwave(solver_id, m, b, x, native.default_options(**opts))
    rr, xr = reference.solve_specwave(solver_id, rm, oracle.default_options(**opts), c["rhs"], np.zeros(n * bs))
    assert r.status == rr.status, (solver_id, r.as_dict(), rr.as_dict())
    assert abs(int(r.iterations) - int(rr.iterations)) <= 2, (solver_id, r.iterations, rr.iterations)
    if r.iterations == rr.iterations:
        for k in COUNTERS:
            assert getattr(r, k) == getattr(rr, k), (solver_id, k)
    if rr.status == 0:
        assert np.linalg.norm(x.download() - xr) <= 1e-6 * np.linalg.norm(xr)


def test_specwave_rejects_off_path_ids(native, ctx, reference, lattice):
    c = lattice
    n, bs = c["owned"], c["bs"]
    m = native.Matrix(ctx, "bsr", n, 0, bs, c["rowptr"], c["cols"], c["vals"])
    b = native.Vector(ctx, n, 0, bs).upload(c["rhs"])
    x = native.Vector(ctx, n, 0, bs)
    for sid in (0, 1, 2, 16, 17, 18, 19, 20):
        with pytest.raises(native.OwtkError) as e:
            native.solve_specwave(sid, m, b, x)
        assert e.value.kind == "invalid_argument"
    r = native.solve_specwave(6, m, b, x)
    assert r.status == 4
