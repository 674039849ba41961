"""ILU applies on packed factor segments (the default for FP64/FP32 ILU with
block size <= 32): the lower and upper entries of every row stored in task
order, gathered by each numeric factorisation.  Against the oracle and
against the applies that read the factor in place (OWTK_PACKED_SWEEP=0):
the same bits, for RCM and natural orders, fill 0-2, block sizes 1-5, FP32,
in place, after update_values, and for whole solves."""
import numpy as np
import pytest

from conftest import assert_bitwise

pytestmark = pytest.mark.gpu


def _system(problems, side, bs, order, seed):
    rng = np.random.default_rng(seed)
    xy, edges = problems.lattice(side, side, 0.2, rng)
    return problems.component_diagonal_system(xy, edges, bs, rng, order=order)


def _pair(native, m, fill, monkeypatch):
    packed = native.Preconditioner(m, native.PC_ILU, fill)
    monkeypatch.setenv("OWTK_PACKED_SWEEP", "0")
    in_place = native.Preconditioner(m, native.PC_ILU, fill)
    monkeypatch.delenv("OWTK_PACKED_SWEEP")
    return packed, in_place


@pytest.mark.parametrize("side,bs,order,fill", [(120, 3, "rcm", 0), (110, 1, "rcm", 0), (90, 4, "natural", 0),
                                                (100, 2, "rcm", 1), (70, 3, "rcm", 2), (60, 5, "natural", 1)])
def test_packed_ilu_apply_bitwise(native, ctx, restatement, problems, monkeypatch, side, bs, order, fill):
    s = _system(problems, side, bs, order, 70 + side)
    n = s.owned
    m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals)
    packed, in_place = _pair(native, m, fill, monkeypatch)
    x = np.random.default_rng(side + bs).uniform(-1, 1, n * bs)
    xv = native.Vector(ctx, n, 0, bs).upload(x)
    y1, y2 = native.Vector(ctx, n, 0, bs), native.Vector(ctx, n, 0, bs)
    for _ in range(2):
        packed.apply(xv, y1)
    in_place.apply(xv, y2)
    want = restatement.ilu(n, bs, s.rowptr, s.cols, s.vals, fill).apply(x)
    assert_bitwise(y1.download(), want, "packed sweep vs oracle")
    assert_bitwise(y2.download(), want, "in-place sweep vs oracle")
    z = native.Vector(ctx, n, 0, bs).upload(x)
    packed.apply(z, z)
    assert_bitwise(z.download(), want, "packed sweep in place")


def test_packed_after_numeric_update(native, ctx, restatement, problems, monkeypatch):
    s = _system(problems, 100, 3, "rcm", 4)
    n, bs = s.owned, s.bs
    m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals)
    packed, _ = _pair(native, m, 0, monkeypatch)
    x = np.random.default_rng(8).uniform(-1, 1, n * bs)
    xv, y = native.Vector(ctx, n, 0, bs).upload(x), native.Vector(ctx, n, 0, bs)
    packed.apply(xv, y)
    vals2 = s.vals * np.random.default_rng(9).uniform(0.9, 1.1, s.vals.size)
    m.update_values(vals2)
    packed.update_values()
    packed.apply(xv, y)
    want = restatement.ilu(n, bs, s.rowptr, s.cols, vals2, 0).apply(x)
    assert_bitwise(y.download(), want, "packed sweep after update_values")


def test_packed_fp32(native, ctx, problems, monkeypatch):
    s = _system(problems, 110, 3, "rcm", 12)
    n, bs = s.owned, s.bs
    m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals, dtype=np.float32)
    packed, in_place = _pair(native, m, 0, monkeypatch)
    x = np.random.default_rng(13).uniform(-1, 1, n * bs).astype(np.float32)
    xv = native.Vector(ctx, n, 0, bs, dtype=np.float32).upload(x)
    y1 = native.Vector(ctx, n, 0, bs, dtype=np.float32)
    y2 = native.Vector(ctx, n, 0, bs, dtype=np.float32)
    packed.apply(xv, y1)
    in_place.apply(xv, y2)
    np.testing.assert_array_equal(y1.download().view(np.uint32), y2.download().view(np.uint32))


def test_packed_solve_equals_in_place(native, ctx, problems, monkeypatch):
    s = _system(problems, 130, 3, "rcm", 21)
    n, bs = s.owned, s.bs
    m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals)
    packed, in_place = _pair(native, m, 0, monkeypatch)
    b = native.Vector(ctx, n, 0, bs).upload(s.rhs)
    x1, x2 = native.Vector(ctx, n, 0, bs), native.Vector(ctx, n, 0, bs)
    r1 = native.solve(native.FGMRES, m, packed, b, x1)
    r2 = native.solve(native.FGMRES, m, in_place, b, x2)
    assert r1.status == r2.status == 0 and r1.iterations == r2.iterations
    assert_bitwise(x1.download(), x2.download(), "solution")
