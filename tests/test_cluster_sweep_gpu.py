"""ILU(k) applies on one thread-block cluster (dependency values through
distributed shared memory, kernels_cluster_sweep.cu; opt-in with
OWTK_CLUSTER_SWEEP=1, with the lockstep schedule off) against the oracle and
against the level-scheduled sweep: the same bits, FP64 and FP32, block sizes 1-4, fill
levels 0 and 1, in place and out of place."""
import numpy as np
import pytest

from conftest import assert_bitwise

pytestmark = pytest.mark.gpu


def _pair(native, m, fill, monkeypatch):
    """The cluster sweep is opt-in (OWTK_CLUSTER_SWEEP=1 at creation): one
    preconditioner on it and one on the default level-scheduled sweep."""
    monkeypatch.setenv("OWTK_LOCKSTEP_SWEEP", "0")
    monkeypatch.setenv("OWTK_CLUSTER_SWEEP", "1")
    pc = native.Preconditioner(m, native.PC_ILU, fill)
    monkeypatch.delenv("OWTK_CLUSTER_SWEEP")
    plain = native.Preconditioner(m, native.PC_ILU, fill)
    monkeypatch.delenv("OWTK_LOCKSTEP_SWEEP")
    return pc, plain


def _system(problems, side, bs, order, seed):
    rng = np.random.default_rng(seed)
    xy, edges = problems.lattice(side, side, 0.2, rng)
    return problems.component_diagonal_system(xy, edges, bs, rng, order=order)


@pytest.mark.parametrize("side,bs,order,fill", [(160, 3, "rcm", 0), (140, 1, "rcm", 0), (150, 4, "natural", 0),
                                                (140, 2, "rcm", 1)])
def test_cluster_ilu_apply_bitwise(native, ctx, restatement, problems, monkeypatch, side, bs, order, fill):
    s = _system(problems, side, bs, order, 31 + side)
    n = s.owned
    m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals)
    pc, plain = _pair(native, m, fill, monkeypatch)
    ctas, k, ring = pc.sweep_schedule()
    assert ctas in (8, 16) and k >= 2 and ring > 0, (ctas, k, ring)
    assert plain.sweep_schedule()[0] == 0
    x = np.random.default_rng(side).uniform(-1, 1, n * bs)
    xv = native.Vector(ctx, n, 0, bs).upload(x)
    y1, y2 = native.Vector(ctx, n, 0, bs), native.Vector(ctx, n, 0, bs)
    for _ in range(3):   # repeated applies reuse the rings
        pc.apply(xv, y1)
    plain.apply(xv, y2)
    ilu = restatement.ilu(n, bs, s.rowptr, s.cols, s.vals, fill)
    want = ilu.apply(x)
    assert_bitwise(y1.download(), want, "cluster sweep vs oracle")
    assert_bitwise(y2.download(), want, "level-scheduled sweep vs oracle")
    # In place (preconditioner.hpp:320-363 allows in == out).
    z = native.Vector(ctx, n, 0, bs).upload(x)
    pc.apply(z, z)
    assert_bitwise(z.download(), want, "cluster sweep in place")


def test_cluster_ilu_apply_fp32(native, ctx, problems, monkeypatch):
    s = _system(problems, 150, 3, "rcm", 77)
    n, bs = s.owned, s.bs
    m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals, dtype=np.float32)
    pc, plain = _pair(native, m, 0, monkeypatch)
    assert pc.sweep_schedule()[0] in (8, 16)
    x = np.random.default_rng(3).uniform(-1, 1, n * bs).astype(np.float32)
    xv = native.Vector(ctx, n, 0, bs, dtype=np.float32).upload(x)
    y1 = native.Vector(ctx, n, 0, bs, dtype=np.float32)
    y2 = native.Vector(ctx, n, 0, bs, dtype=np.float32)
    pc.apply(xv, y1)
    plain.apply(xv, y2)
    assert_bitwise(y1.download(), y2.download(), "FP32 cluster vs level-scheduled sweep")


def test_cluster_solve_matches_plain_sweep(native, ctx, problems, monkeypatch):
    """GMRES(30)+ILU(0) gives the same bits with either schedule."""
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
