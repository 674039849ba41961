"""ILU(k) applies level by level on one thread-block cluster
(kernels_lockstep_sweep.cu, opt-in with OWTK_LOCKSTEP_SWEEP=1, taken when
every level fits the cluster's lanes) against the oracle and against the
level-scheduled sweep (the default): the same bits.  RCM and natural orders, block
sizes 1-4, fill levels 0-2, FP32, in place, repeated applies, numeric
updates (the factor values are re-gathered), whole solves."""
import numpy as np
import pytest

from conftest import assert_bitwise

pytestmark = pytest.mark.gpu


def _system(problems, side, bs, order, seed):
    rng = np.random.default_rng(seed)
    xy, edges = problems.lattice(side, side, 0.2, rng)
    return problems.component_diagonal_system(xy, edges, bs, rng, order=order)


def _pair(native, m, fill, monkeypatch):
    monkeypatch.setenv("OWTK_LOCKSTEP_SWEEP", "1")
    pc = native.Preconditioner(m, native.PC_ILU, fill)
    monkeypatch.delenv("OWTK_LOCKSTEP_SWEEP")
    plain = native.Preconditioner(m, native.PC_ILU, fill)
    return pc, plain


@pytest.mark.parametrize("side,bs,order,fill", [(160, 3, "rcm", 0), (140, 1, "rcm", 0), (150, 4, "natural", 0),
                                                (140, 2, "rcm", 1), (100, 3, "rcm", 2)])
def test_lockstep_ilu_apply_bitwise(native, ctx, restatement, problems, monkeypatch, side, bs, order, fill):
    s = _system(problems, side, bs, order, 51 + side)
    n = s.owned
    m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals)
    pc, plain = _pair(native, m, fill, monkeypatch)
    ctas, dl, du = pc.lockstep_schedule()
    assert ctas in (8, 16) and dl > 16 and du > 16, (ctas, dl, du)
    assert plain.lockstep_schedule()[0] == 0
    x = np.random.default_rng(side).uniform(-1, 1, n * bs)
    xv = native.Vector(ctx, n, 0, bs).upload(x)
    y1, y2 = native.Vector(ctx, n, 0, bs), native.Vector(ctx, n, 0, bs)
    for _ in range(3):
        pc.apply(xv, y1)
    plain.apply(xv, y2)
    want = restatement.ilu(n, bs, s.rowptr, s.cols, s.vals, fill).apply(x)
    assert_bitwise(y1.download(), want, "lockstep sweep vs oracle")
    assert_bitwise(y2.download(), want, "level-scheduled sweep vs oracle")
    z = native.Vector(ctx, n, 0, bs).upload(x)
    pc.apply(z, z)
    assert_bitwise(z.download(), want, "lockstep sweep in place")


def test_lockstep_after_numeric_update(native, ctx, restatement, problems, monkeypatch):
    s = _system(problems, 130, 3, "rcm", 9)
    n, bs = s.owned, s.bs
    m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals)
    pc, _ = _pair(native, m, 0, monkeypatch)
    assert pc.lockstep_schedule()[0] > 0
    x = np.random.default_rng(2).uniform(-1, 1, n * bs)
    xv, y = native.Vector(ctx, n, 0, bs).upload(x), native.Vector(ctx, n, 0, bs)
    pc.apply(xv, y)
    vals2 = s.vals * np.random.default_rng(3).uniform(0.9, 1.1, s.vals.size)
    m.update_values(vals2)
    pc.update_values()
    pc.apply(xv, y)
    want = restatement.ilu(n, bs, s.rowptr, s.cols, vals2, 0).apply(x)
    assert_bitwise(y.download(), want, "lockstep sweep after update_values")


def test_lockstep_fp32(native, ctx, problems, monkeypatch):
    s = _system(problems, 150, 3, "rcm", 77)
    n, bs = s.owned, s.bs
    m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals, dtype=np.float32)
    pc, plain = _pair(native, m, 0, monkeypatch)
    assert pc.lockstep_schedule()[0] > 0
    x = np.random.default_rng(3).uniform(-1, 1, n * bs).astype(np.float32)
    xv = native.Vector(ctx, n, 0, bs, dtype=np.float32).upload(x)
    y1 = native.Vector(ctx, n, 0, bs, dtype=np.float32)
    y2 = native.Vector(ctx, n, 0, bs, dtype=np.float32)
    pc.apply(xv, y1)
    plain.apply(xv, y2)
    np.testing.assert_array_equal(y1.download().view(np.uint32), y2.download().view(np.uint32))


def test_lockstep_solve_equals_level_scheduled(native, ctx, problems, monkeypatch):
    s = _system(problems, 170, 3, "rcm", 5)
    n, bs = s.owned, s.bs
    m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals)
    pc, plain = _pair(native, m, 0, monkeypatch)
    b = native.Vector(ctx, n, 0, bs).upload(s.rhs)
    x1, x2 = native.Vector(ctx, n, 0, bs), native.Vector(ctx, n, 0, bs)
    r1 = native.solve(native.FGMRES, m, pc, b, x1)
    r2 = native.solve(native.FGMRES, m, plain, b, x2)
    assert r1.status == r2.status == 0 and r1.iterations == r2.iterations
    assert_bitwise(x1.download(), x2.download(), "solution")
