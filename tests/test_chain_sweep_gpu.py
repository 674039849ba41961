"""ILU(k) applies on near-sequential DAGs by one warp per component
(kernels_chain_sweep.cu) against the oracle and against the level-scheduled
sweep: the same bits.  Hilbert-ordered meshes (the order that makes the
factors' DAGs about as deep as the matrix is long), fill levels 0-2, block
sizes 1-4, FP64 and FP32, in place, repeated applies; a hub row with more
factor entries than one window stages (read from global memory) and
dependencies beyond the shared-memory ring of 8192 results; a whole GMRES
solve."""
import numpy as np
import pytest

from conftest import assert_bitwise

pytestmark = pytest.mark.gpu


def _hilbert_system(problems, side, bs, seed):
    rng = np.random.default_rng(seed)
    xy, edges = problems.lattice(side, side, 0.2, rng)
    return problems.component_diagonal_system(xy, edges, bs, rng, order="hilbert")


def _pair(native, m, fill, monkeypatch):
    """The chain-sweep preconditioner and one on the level-scheduled sweep."""
    pc = native.Preconditioner(m, native.PC_ILU, fill)
    monkeypatch.setenv("OWTK_CHAIN_SWEEP", "0")
    plain = native.Preconditioner(m, native.PC_ILU, fill)
    monkeypatch.delenv("OWTK_CHAIN_SWEEP")
    return pc, plain


@pytest.mark.parametrize("side,bs,fill", [(120, 3, 0), (140, 1, 0), (90, 2, 1), (70, 4, 2), (130, 3, 1)])
def test_chain_ilu_apply_bitwise(native, ctx, restatement, problems, monkeypatch, side, bs, fill):
    s = _hilbert_system(problems, side, bs, 7 + side)
    n = s.owned
    m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals)
    pc, plain = _pair(native, m, fill, monkeypatch)
    assert pc.chain_windows() >= n // 32, pc.chain_windows()
    assert plain.chain_windows() == 0
    _, _, dl, du = pc.levels()
    assert n / dl < 8 and n / du < 8, (n, dl, du)
    x = np.random.default_rng(side).uniform(-1, 1, n * bs)
    xv = native.Vector(ctx, n, 0, bs).upload(x)
    y1, y2 = native.Vector(ctx, n, 0, bs), native.Vector(ctx, n, 0, bs)
    for _ in range(3):   # repeated applies reuse the ring and the stages
        pc.apply(xv, y1)
    plain.apply(xv, y2)
    want = restatement.ilu(n, bs, s.rowptr, s.cols, s.vals, fill).apply(x)
    assert_bitwise(y1.download(), want, "chain sweep vs oracle")
    assert_bitwise(y2.download(), want, "level-scheduled sweep vs oracle")
    z = native.Vector(ctx, n, 0, bs).upload(x)   # in place (preconditioner.hpp:320-363 allows in == out)
    pc.apply(z, z)
    assert_bitwise(z.download(), want, "chain sweep in place")


def test_chain_ilu_apply_fp32(native, ctx, problems, monkeypatch):
    s = _hilbert_system(problems, 110, 3, 5)
    n, bs = s.owned, s.bs
    m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals, dtype=np.float32)
    pc, plain = _pair(native, m, 0, monkeypatch)
    assert pc.chain_windows() > 0
    x = np.random.default_rng(3).uniform(-1, 1, n * bs).astype(np.float32)
    xv = native.Vector(ctx, n, 0, bs, dtype=np.float32).upload(x)
    y1 = native.Vector(ctx, n, 0, bs, dtype=np.float32)
    y2 = native.Vector(ctx, n, 0, bs, dtype=np.float32)
    pc.apply(xv, y1)
    plain.apply(xv, y2)
    np.testing.assert_array_equal(y1.download().view(np.uint32), y2.download().view(np.uint32))


def _hub_system(n, bs, seed):
    """Row 0 is joined to every row and row i to row i+1: a DAG of depth n,
    row 0's factor row (n entries) larger than a stage, and rows past 8192
    reading row 0 from beyond the ring."""
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        nb = {i}
        if i == 0:
            nb.update(range(n))
        else:
            nb.update({0, i - 1})
            if i + 1 < n:
                nb.add(i + 1)
        rows.append(sorted(nb))
    rowptr = np.zeros(n + 1, np.int64)
    rowptr[1:] = np.cumsum([len(r) for r in rows])
    cols = np.concatenate([np.array(r, np.int64) for r in rows])
    vals = rng.uniform(-1.0, -0.1, (cols.size, bs))
    for i in range(n):
        e0, e1 = rowptr[i], rowptr[i + 1]
        d = e0 + rows[i].index(i)
        vals[d] = 1.2 * np.abs(vals[e0:e1]).sum(axis=0) + 1.0
    return rowptr, cols, vals.reshape(-1)


def test_chain_ilu_hub_row_and_far_dependencies(native, ctx, restatement, monkeypatch):
    n, bs = 10_000, 2
    rowptr, cols, vals = _hub_system(n, bs, 11)
    m = native.Matrix(ctx, "bsr", n, 0, bs, rowptr, cols, vals)
    pc, plain = _pair(native, m, 0, monkeypatch)
    assert pc.chain_windows() > 0
    x = np.random.default_rng(4).uniform(-1, 1, n * bs)
    xv = native.Vector(ctx, n, 0, bs).upload(x)
    y1, y2 = native.Vector(ctx, n, 0, bs), native.Vector(ctx, n, 0, bs)
    pc.apply(xv, y1)
    plain.apply(xv, y2)
    want = restatement.ilu(n, bs, rowptr, cols, vals, 0).apply(x)
    assert_bitwise(y1.download(), want, "chain sweep, hub row")
    assert_bitwise(y2.download(), want, "level-scheduled sweep, hub row")


def test_chain_gmres_solve_equals_level_scheduled(native, ctx, problems, monkeypatch):
    s = _hilbert_system(problems, 150, 3, 19)
    n, bs = s.owned, s.bs
    m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals)
    pc, plain = _pair(native, m, 0, monkeypatch)
    b = native.Vector(ctx, n, 0, bs).upload(s.rhs)
    x1, x2 = native.Vector(ctx, n, 0, bs), native.Vector(ctx, n, 0, bs)
    opts = native.default_options(restart=30)
    r1 = native.solve(native.FGMRES, m, pc, b, x1, opts)
    r2 = native.solve(native.FGMRES, m, plain, b, x2, opts)
    assert r1.status == r2.status == 0 and r1.iterations == r2.iterations
    assert r1.true_residual_norm <= 1e-8 * np.linalg.norm(s.rhs)
    assert_bitwise(x1.download(), x2.download(), "chain vs level-scheduled solve")
