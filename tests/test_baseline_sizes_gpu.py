"""Parity at the benchmark configurations' own sizes, against the reference
(oracle/_ref), through the C ABI:

* the 2M-vertex Poisson-disk/Delaunay disk mesh (bs 3): this library's RCM
  order equals the reference's reverse_cuthill_mckee_order bit for bit
  (ordering.hpp:138-180); the ILU(0) factors computed on the device equal the
  reference's (preconditioner.hpp:439-485) bit for bit; GMRES(30) + ILU(0)
  reaches true-residual rtol 1e-8 within 2 iterations of the reference; in
  the Hilbert order the ILU(0) apply (the chain sweep) equals the reference's;
* the anisotropic unit-square mesh at 200k vertices (the training size of the
  learned form): plain ILU(0)-GMRES(30) against the reference, and the
  learned FGMRES with the committed trained network reaching the same
  tolerance, its solution against the reference's;
* the dense 3x3 form at 200k vertices: the FP32 and BF16 mixed-precision
  solves against the reference's own FP64 solution of the same system;
* the batched form: a sample of the 256 systems (smallest, largest and
  spread in between) against the reference's per-system BiCGSTAB + Jacobi.

These build large meshes (tens of seconds each) and run the reference's
single-threaded solves, so they run with the GPU suite.
"""
import os

import numpy as np
import pytest

from conftest import PKG

pytestmark = pytest.mark.gpu

WEIGHTS = os.path.join(PKG, "weights", "learned_anisotropic_bs3.owtkgnn")


@pytest.fixture(scope="module")
def disk2m(problems):
    xy, edges = problems.disk_mesh(2_000_000, 1)
    return xy, edges


def test_cfg1_rcm_factors_and_gmres_at_2m(native, ctx, reference, problems, disk2m):
    import oracle
    xy, edges = disk2m
    n = xy.shape[0]
    rp, cp = problems.pattern(n, edges)
    ours = native.rcm_order(n, rp, cp)
    theirs = reference.rcm(n, rp, cp)
    np.testing.assert_array_equal(ours, theirs)
    s = problems.component_diagonal_system(xy, edges, 3, np.random.default_rng(1), order=ours)
    bs = s.bs
    m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals)
    pc = native.Preconditioner(m, native.PC_ILU, 0)
    rm = reference.matrix("bsr", n, 0, bs, s.rowptr, s.cols, s.vals)
    rpc = reference.pc("ilu", rm, 0)
    frp, fci, fv, finv = pc.ilu_factors()
    grp, gci, gv, ginv = rpc.ilu_factors()
    np.testing.assert_array_equal(frp.astype(np.int64), grp)
    np.testing.assert_array_equal(fci.astype(np.int64), gci)
    np.testing.assert_array_equal(fv.view(np.uint64), gv.view(np.uint64))
    np.testing.assert_array_equal(finv.view(np.uint64), ginv.view(np.uint64))
    b = native.Vector(ctx, n, 0, bs).upload(s.rhs)
    x = native.Vector(ctx, n, 0, bs)
    r = native.solve(native.FGMRES, m, pc, b, x, native.default_options(restart=30))
    rr, xr = reference.solve("gmres", rm, rpc, oracle.default_options(restart=30), s.rhs, np.zeros(n * bs))
    bnorm = np.linalg.norm(s.rhs)
    assert r.status == rr.status == 0
    assert abs(int(r.iterations) - int(rr.iterations)) <= 2, (r.iterations, rr.iterations)
    assert r.true_residual_norm <= 1e-8 * bnorm
    xs = x.download()
    assert np.linalg.norm(xs - xr) <= 1e-6 * np.linalg.norm(xr)


def test_cfg1_hilbert_chain_sweep_at_2m(native, ctx, reference, problems, disk2m):
    """The same 2M mesh in the Hilbert order (the sweep over both orderings):
    the ILU(0) apply takes the chain sweep and equals the reference's apply
    (preconditioner.hpp:320-363) bit for bit."""
    xy, edges = disk2m
    s = problems.component_diagonal_system(xy, edges, 3, np.random.default_rng(1), order="hilbert")
    n, bs = s.owned, s.bs
    m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals)
    pc = native.Preconditioner(m, native.PC_ILU, 0)
    assert pc.chain_windows() > 0
    x = native.Vector(ctx, n, 0, bs).upload(s.rhs)
    y = native.Vector(ctx, n, 0, bs)
    pc.apply(x, y)
    rm = reference.matrix("bsr", n, 0, bs, s.rowptr, s.cols, s.vals)
    want = reference.pc("ilu", rm, 0).apply(s.rhs)
    np.testing.assert_array_equal(y.download().view(np.uint64), want.view(np.uint64))


def test_cfg4_anisotropic_200k_plain_and_learned(native, ctx, reference, problems):
    import oracle
    from owtk_b200 import checkpoint
    s = problems.config4(200_000, seed=4)
    n, bs = s.owned, s.bs
    bnorm = np.linalg.norm(s.rhs)
    m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals)
    ilu = native.Preconditioner(m, native.PC_ILU, 0)
    rm = reference.matrix("bsr", n, 0, bs, s.rowptr, s.cols, s.vals)
    rilu = reference.pc("ilu", rm, 0)
    rr, xr = reference.solve("gmres", rm, rilu, oracle.default_options(restart=30), s.rhs, np.zeros(n * bs))
    b = native.Vector(ctx, n, 0, bs).upload(s.rhs)
    x = native.Vector(ctx, n, 0, bs)
    r = native.solve(native.FGMRES, m, ilu, b, x, native.default_options(restart=30))
    assert r.status == rr.status == 0
    assert abs(int(r.iterations) - int(rr.iterations)) <= 2
    assert r.true_residual_norm <= 1e-8 * bnorm
    # The learned preconditioner with the committed weights.
    net = native.Learned(m, seed=1)
    ck = checkpoint.load_network(WEIGHTS, net, with_optimizer=False)
    assert ck["metadata"]["draws"] == 500
    pcl = native.LearnedPreconditioner(net, ilu)
    x.fill(0.0)
    rl = native.solve(native.FGMRES, m, pcl, b, x, native.default_options(restart=30))
    assert rl.status == 0 and rl.true_residual_norm <= 1e-8 * bnorm
    assert rl.iterations <= rr.iterations
    xs = x.download()
    assert np.linalg.norm(xs - xr) <= 1e-6 * np.linalg.norm(xr)


def test_cfg2_mixed_error_against_reference_solution(native, ctx, reference, problems):
    """Dense 3x3 blocks at 200k vertices: the mixed FP32 / BF16 solves to
    rtol 1e-10, their error taken against the reference's FP64 solution
    (its GMRES(30) on the DenseBlockCsrMatrix to rtol 1e-13; the reference
    has no preconditioner for dense blocks)."""
    import oracle
    s = problems.config2(200_000)
    n, bs = s.owned, s.bs
    rm = reference.matrix("dense", n, 0, bs, s.rowptr, s.cols, s.vals)
    rr, xr = reference.solve("gmres", rm, reference.pc("identity", rm, 0.0),
                             oracle.default_options(relative_tolerance=1e-13, maximum_iterations=5000),
                             s.rhs, np.zeros(n * bs))
    assert rr.status == 0
    m = native.Matrix(ctx, "dense", n, 0, bs, s.rowptr, s.cols, s.vals)
    b = native.Vector(ctx, n, 0, bs).upload(s.rhs)
    for storage in (native.F32, native.BF16):
        pc = native.Preconditioner(m, native.PC_BLOCK_ILU, 0, storage=storage, mixed_inner=4)
        x = native.Vector(ctx, n, 0, bs)
        r = native.solve(native.FGMRES, m, pc, b, x, native.default_options(relative_tolerance=1e-10))
        assert r.status == 0 and r.true_residual_norm <= 1e-10 * np.linalg.norm(s.rhs)
        err = np.linalg.norm(x.download() - xr) / np.linalg.norm(xr)
        assert err <= 1e-8, (storage, err)


def test_cfg3_batch_sample_against_reference(native, ctx, reference, problems):
    import oracle
    systems = problems.batch_systems(count=256, seed=3)
    batch = native.Batch(ctx, systems)
    rhs = np.concatenate([y.rhs for y in systems])
    rv = native.Vector(ctx, rhs.size, 0, 1).upload(rhs)
    xv = native.Vector(ctx, rhs.size, 0, 1)
    res = batch.solve(rv, xv)
    xs = xv.download()
    sizes = np.array([y.owned * y.bs for y in systems])
    order = np.argsort(sizes)
    sample = sorted(set(order[np.linspace(0, len(systems) - 1, 8).astype(int)].tolist()))
    offsets = batch.offsets
    for i in sample:
        y = systems[i]
        rm = reference.matrix("bsr", y.owned, 0, y.bs, y.rowptr, y.cols, y.vals)
        rr, xr = reference.solve("bicgstab", rm, reference.pc("jacobi", rm, 0.0), oracle.default_options(), y.rhs,
                                 np.zeros(y.owned * y.bs))
        got = res[i]
        assert got.status == rr.status == 0, i
        assert abs(int(got.iterations) - int(rr.iterations)) <= 2, (i, got.iterations, rr.iterations)
        xi = xs[offsets[i]:offsets[i + 1]]
        true_res = np.linalg.norm(y.rhs - _spmv(y, xi))
        assert true_res <= 1e-8 * np.linalg.norm(y.rhs) * (1 + 1e-9)
        assert np.linalg.norm(xi - xr) <= 1e-5 * np.linalg.norm(xr)


def _spmv(y, x):
    bs = y.bs
    rows = np.repeat(np.arange(y.owned), np.diff(y.rowptr))
    prod = y.vals.reshape(-1, bs) * x.reshape(-1, bs)[y.cols]
    out = np.zeros((y.owned, bs))
    np.add.at(out, rows, prod)
    return out.reshape(-1)
