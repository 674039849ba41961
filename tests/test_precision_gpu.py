"""Mixed-precision form: dense-block ILU(0), FP32/BF16 factor storage, and the
FP64 flexible GMRES around an FP32 inner solve.

The dense-block ILU has no reference counterpart; its checker is the C
restatement in oracle/owtk_oracle.c (bit-exact in FP64).  Low-precision
results are held to stated error bounds against the FP64 oracle, and the
mixed solves must reach the requested FP64 true-residual tolerance with a
solution equal to the FP64 oracle solution to the tolerance's accuracy.
"""
import numpy as np
import pytest

import cases
from conftest import assert_bitwise

pytestmark = pytest.mark.gpu

BLOCK_CASES = [dict(side=5, bs=3, seed=18), dict(side=4, bs=2, seed=19), dict(side=6, bs=4, seed=31),
               dict(side=7, bs=1, seed=32)]


def dense_matrix(native, ctx, c):
    return native.Matrix(ctx, "dense", c["owned"], 0, c["bs"], c["rowptr"], c["cols"], c["vals"])


@pytest.mark.parametrize("kw", BLOCK_CASES, ids=lambda k: f"bs{k['bs']}")
def test_block_ilu_bitwise(native, ctx, restatement, kw):
    c = cases.dense_case(**kw)
    n, bs = c["owned"], c["bs"]
    m = dense_matrix(native, ctx, c)
    p = native.Preconditioner(m, native.PC_BLOCK_ILU)
    ref = restatement.block_ilu(n, bs, c["rowptr"], c["cols"], c["vals"])
    assert ref.status == 0
    rv, rd = ref.factors()
    _, _, v, d = p.ilu_factors()
    assert_bitwise(v, rv, "block factors")
    assert_bitwise(d, rd, "inverse diagonal blocks")
    x = native.Vector(ctx, n, 0, bs).upload(c["x"])
    y = native.Vector(ctx, n, 0, bs)
    p.apply(x, y)
    assert_bitwise(y.download(), ref.apply(c["x"]), "block apply")
    p.apply(x, x)   # in place
    assert_bitwise(x.download(), ref.apply(c["x"]), "in-place block apply")
    ctx.synchronize()


@pytest.mark.parametrize("side,bs", [(120, 3), (90, 4)])
def test_block_ilu_bitwise_many_levels(native, ctx, restatement, side, bs):
    # Hundreds of levels: block rows publish as soon as their own
    # dependencies arrive, and a row of the backward sweep publishes once all
    # of its block rows are final.
    c = cases.dense_case(side=side, bs=bs, seed=side)
    n = c["owned"]
    m = dense_matrix(native, ctx, c)
    p = native.Preconditioner(m, native.PC_BLOCK_ILU)
    ref = restatement.block_ilu(n, bs, c["rowptr"], c["cols"], c["vals"])
    assert ref.status == 0
    x = native.Vector(ctx, n, 0, bs).upload(c["x"])
    y = native.Vector(ctx, n, 0, bs)
    expect = ref.apply(c["x"])
    for rep in range(2):
        p.apply(x, y)
        assert_bitwise(y.download(), expect, f"block apply {rep}")
    ctx.synchronize()


def test_block_ilu_update_values(native, ctx, restatement):
    c = cases.dense_case(side=5, bs=3, seed=18)
    n, bs = c["owned"], c["bs"]
    m = dense_matrix(native, ctx, c)
    p = native.Preconditioner(m, native.PC_BLOCK_ILU)
    vals2 = c["vals"] * 1.05
    m.update_values(vals2)
    p.update_values(m)
    assert p.numeric_updates == 2
    ref = restatement.block_ilu(n, bs, c["rowptr"], c["cols"], vals2)
    _, _, v, _ = p.ilu_factors()
    assert_bitwise(v, ref.factors()[0], "refactored blocks")


@pytest.mark.parametrize("storage,tol", [("F32", 2e-6), ("BF16", 3e-2)])
def test_stored_precision_ilu(native, ctx, restatement, storage, tol):
    # FP64 factorisation, factors rounded to the storage type, FP32 applies:
    # relative error against the FP64 apply bounded by a few storage ulps
    # amplified by the triangular solves.
    code = native.F32 if storage == "F32" else native.BF16
    c = cases.lattice_case(side=24, bs=3, seed=21)
    n, bs = c["owned"], c["bs"]
    m = native.Matrix(ctx, "bsr", n, 0, bs, c["rowptr"], c["cols"], c["vals"])
    p = native.Preconditioner(m, native.PC_ILU, 0, storage=code)
    x = native.Vector(ctx, n, 0, bs, dtype=np.float32).upload(c["x"][: n * bs])
    y = native.Vector(ctx, n, 0, bs, dtype=np.float32)
    p.apply(x, y)
    got = y.download().astype(np.float64)
    ilu = restatement.ilu(n, bs, c["rowptr"], c["cols"], c["vals"], 0)
    expect = ilu.apply(c["x"][: n * bs].astype(np.float32).astype(np.float64))
    err = np.linalg.norm(got - expect) / np.linalg.norm(expect)
    assert err <= tol, err
    # FP64 vectors are rejected by stored-precision factors.
    with pytest.raises(native.OwtkError):
        p.apply(native.Vector(ctx, n, 0, bs), native.Vector(ctx, n, 0, bs))


@pytest.mark.parametrize("storage", ["F32", "BF16"])
@pytest.mark.parametrize("inner", [0, 4])
def test_mixed_fgmres_component_diagonal(native, ctx, restatement, storage, inner):
    import oracle
    code = native.F32 if storage == "F32" else native.BF16
    c = cases.lattice_case(side=24, bs=3, seed=21)
    n, bs = c["owned"], c["bs"]
    rhs = c["rhs"][: n * bs]
    m = native.Matrix(ctx, "bsr", n, 0, bs, c["rowptr"], c["cols"], c["vals"])
    p = native.Preconditioner(m, native.PC_ILU, 0, storage=code, mixed_inner=inner)
    b = native.Vector(ctx, n, 0, bs).upload(rhs)
    x = native.Vector(ctx, n, 0, bs)
    r = native.solve(native.FGMRES, m, p, b, x, native.default_options(relative_tolerance=1e-10))
    assert r.status == 0, r.as_dict()
    assert r.true_residual_norm <= 1e-10 * np.linalg.norm(rhs)
    mat = restatement.make_matrix("bsr", n, 0, bs, c["rowptr"], c["cols"], c["vals"])
    ilu = restatement.ilu(n, bs, c["rowptr"], c["cols"], c["vals"], 0)
    _, xr = restatement.solve("gmres", mat, restatement.make_pc("ilu", mat, 0, ilu),
                              oracle.default_options(relative_tolerance=1e-13), rhs, np.zeros(n * bs))
    assert np.linalg.norm(x.download() - xr) <= 1e-8 * np.linalg.norm(xr)


@pytest.mark.parametrize("storage", ["F32", "BF16"])
def test_mixed_fgmres_dense_blocks(native, ctx, restatement, storage):
    # The dense 3x3 form (FP32/BF16 block factors, FP32 inner SpMV) to rtol 1e-10.
    code = native.F32 if storage == "F32" else native.BF16
    c = cases.dense_case(side=20, bs=3, seed=33)
    n, bs = c["owned"], c["bs"]
    m = dense_matrix(native, ctx, c)
    p = native.Preconditioner(m, native.PC_BLOCK_ILU, 0, storage=code, mixed_inner=4)
    b = native.Vector(ctx, n, 0, bs).upload(c["rhs"])
    x = native.Vector(ctx, n, 0, bs)
    r = native.solve(native.FGMRES, m, p, b, x, native.default_options(relative_tolerance=1e-10))
    assert r.status == 0, r.as_dict()
    assert r.true_residual_norm <= 1e-10 * np.linalg.norm(c["rhs"])
    # Error against the FP64 solution of the same system (dense LAPACK solve).
    A = np.zeros((n * bs, n * bs))
    vals = c["vals"].reshape(-1, bs, bs)
    for row in range(n):
        for e in range(c["rowptr"][row], c["rowptr"][row + 1]):
            col = c["cols"][e]
            A[row * bs:(row + 1) * bs, col * bs:(col + 1) * bs] = vals[e]
    xr = np.linalg.solve(A, c["rhs"])
    assert np.linalg.norm(x.download() - xr) <= 1e-8 * np.linalg.norm(xr)
