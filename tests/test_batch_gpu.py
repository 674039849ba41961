"""Batched BiCGSTAB + Jacobi: many uneven systems in one persistent,
graph-captured launch with per-system convergence masks.

Checker: the reference's bicgstab + JacobiPreconditioner restated in
oracle/owtk_oracle.c, run system by system.  The batched kernel uses the same
element-wise arithmetic and SpMV bit for bit but its own reduction order, so
each system must reach the same status, iterations within +-2, counters equal
whenever the iteration counts are, the FP64 true-residual tolerance (checked
again on the host), and the oracle's solution to the accuracy that tolerance
implies.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

COUNTERS = ["status", "breakdown_reason", "iterations", "operator_applications", "preconditioner_applications",
            "global_reductions"]


def small_batch(count=10, seed=5):
    from owtk_b200 import problems
    return problems.batch_systems(count=count, seed=seed, n_min=200, n_max=6000)


def oracle_solve(restatement, s, x0=None, **opts):
    import oracle
    mat = restatement.make_matrix("bsr", s.owned, 0, s.bs, s.rowptr, s.cols, s.vals)
    pc = restatement.make_pc("jacobi", mat, 0.0, None)
    x0 = np.zeros(s.owned * s.bs) if x0 is None else x0
    return restatement.solve("bicgstab", mat, pc, oracle.default_options(**opts), s.rhs, x0)


def run_batch(native, ctx, batch, rhs, x0, **opts):
    rv = native.Vector(ctx, rhs.size, 0, 1).upload(rhs)
    xv = native.Vector(ctx, rhs.size, 0, 1).upload(x0)
    res = batch.solve(rv, xv, native.default_options(**opts))
    return res, xv.download()


def check_against_oracle(restatement, systems, offsets, res, x, rtol=1e-8, x0s=None, **opts):
    for i, s in enumerate(systems):
        x0 = None if x0s is None else x0s[i]
        r, xr = oracle_solve(restatement, s, x0, relative_tolerance=rtol, **opts)
        d, e = res[i].as_dict(), r.as_dict()
        assert d["status"] == e["status"], (i, d, e)
        assert abs(d["iterations"] - e["iterations"]) <= 2, (i, d["iterations"], e["iterations"])
        if d["iterations"] == e["iterations"]:
            for k in COUNTERS:
                assert d[k] == e[k], (i, k, d[k], e[k])
        xi = x[offsets[i]:offsets[i + 1]]
        if d["status"] == 0:
            thr = rtol * np.linalg.norm(s.rhs)
            assert d["true_residual_norm"] <= thr
            resid = s.rhs - restatement.bsr_spmv(s.owned, s.bs, s.rowptr, s.cols, s.vals, xi)
            assert np.linalg.norm(resid) <= thr * (1 + 1e-6)
            assert np.linalg.norm(xi - xr) <= 1e-5 * max(np.linalg.norm(xr), 1e-300)


def test_batch_matches_per_system_reference(native, ctx, restatement):
    systems = small_batch()
    assert {s.bs for s in systems} >= {1, 2, 3, 4}
    b = native.Batch(ctx, systems)
    rhs = np.concatenate([s.rhs for s in systems])
    assert b.unknowns == rhs.size
    assert list(np.diff(b.offsets)) == [s.owned * s.bs for s in systems]
    res, x = run_batch(native, ctx, b, rhs, np.zeros_like(rhs))
    check_against_oracle(restatement, systems, b.offsets, res, x)
    # Same systems through the single-system device path: identical element-
    # wise arithmetic, so the same iteration counts up to reduction order.
    s = systems[3]
    m = native.Matrix(ctx, "bsr", s.owned, 0, s.bs, s.rowptr, s.cols, s.vals)
    pc = native.Preconditioner(m, native.PC_JACOBI)
    bv = native.Vector(ctx, s.owned, 0, s.bs).upload(s.rhs)
    xv = native.Vector(ctx, s.owned, 0, s.bs)
    r1 = native.solve(native.BICGSTAB, m, pc, bv, xv)
    assert abs(r1.iterations - res[3].iterations) <= 2


def test_batch_counters_when_capped_and_checked_every_iteration(native, ctx, restatement):
    systems = small_batch(count=6, seed=9)
    b = native.Batch(ctx, systems)
    rhs = np.concatenate([s.rhs for s in systems])
    # Iteration cap: every system stops at maximum_iterations with the final
    # true residual; counters equal the reference's exactly.
    res, x = run_batch(native, ctx, b, rhs, np.zeros_like(rhs), maximum_iterations=3)
    for i, s in enumerate(systems):
        r, _ = oracle_solve(restatement, s, maximum_iterations=3)
        d, e = res[i].as_dict(), r.as_dict()
        for k in COUNTERS:
            assert d[k] == e[k], (i, k, d[k], e[k])
        assert d["status"] == 1
    # Convergence checked every iteration plus residual replacement: the
    # true-residual branch and restarts are exercised.
    res, x = run_batch(native, ctx, b, rhs, np.zeros_like(rhs), convergence_check_interval=1,
                       residual_replacement_interval=7)
    check_against_oracle(restatement, systems, b.offsets, res, x, convergence_check_interval=1,
                         residual_replacement_interval=7)


def test_batch_masks_graph_replay_and_host_path(native, ctx, restatement):
    systems = small_batch(count=8, seed=11)
    b = native.Batch(ctx, systems)
    off = b.offsets
    rhs = np.concatenate([s.rhs for s in systems])
    x0 = np.zeros_like(rhs)
    # System 0 starts at the oracle's solution (converges with 0 iterations),
    # system 1 has a zero right-hand side (r0 = 0 <= threshold).
    _, xr0 = oracle_solve(restatement, systems[0], relative_tolerance=1e-13)
    x0[off[0]:off[1]] = xr0
    rhs[off[1]:off[2]] = 0.0
    systems[1].rhs = np.zeros(systems[1].owned * systems[1].bs)
    rv = native.Vector(ctx, rhs.size, 0, 1).upload(rhs)
    xv = native.Vector(ctx, rhs.size, 0, 1).upload(x0)
    res1 = b.solve(rv, xv)
    xa = xv.download()
    assert res1[0].iterations == 0 and res1[0].status == 0
    assert res1[1].iterations == 0 and res1[1].status == 0
    x0s = [x0[off[i]:off[i + 1]] for i in range(len(systems))]
    check_against_oracle(restatement, systems, off, res1, xa, x0s=x0s)
    # Replay: same vectors and options -> the captured graph is relaunched and
    # the results repeat bit for bit.
    xv.upload(x0)
    res2 = b.solve(rv, xv)
    assert np.array_equal(xv.download().view(np.uint64), xa.view(np.uint64))
    assert [r.as_dict() for r in res2] == [r.as_dict() for r in res1] or all(
        {k: v for k, v in r2.as_dict().items() if k != "solve_seconds"}
        == {k: v for k, v in r1.as_dict().items() if k != "solve_seconds"} for r1, r2 in zip(res1, res2))
    captures, launches = b.graph_counts()
    assert captures == 1 and launches == 2
    # Plain launches give the same bits.
    b.use_graph(False)
    xv.upload(x0)
    b.solve(rv, xv)
    assert np.array_equal(xv.download().view(np.uint64), xa.view(np.uint64))
    b.use_graph(True)
    # Host buffers in and out.
    hx = x0.copy()
    rh = np.ascontiguousarray(rhs)
    b.solve_host(rh.ctypes.data, hx.ctypes.data)
    assert np.array_equal(hx.view(np.uint64), xa.view(np.uint64))


def test_batch_autotune(native, ctx, restatement):
    systems = small_batch(count=12, seed=13)
    b = native.Batch(ctx, systems)
    bps, vpw = b.autotune()
    assert bps >= 1
    for s in systems:
        assert vpw[s.bs] >= 1
    assert b.config() == (bps, vpw)
    rhs = np.concatenate([s.rhs for s in systems])
    res, x = run_batch(native, ctx, b, rhs, np.zeros_like(rhs))
    check_against_oracle(restatement, systems, b.offsets, res, x)
    # A manual shape gives the same SpMV bits; only reduction order may move.
    b.set_config(blocks_per_sm=1, bs=3, vertices_per_warp=1)
    res, x = run_batch(native, ctx, b, rhs, np.zeros_like(rhs))
    check_against_oracle(restatement, systems, b.offsets, res, x)


@pytest.mark.parametrize("blocks_per_sm", [2, 3, 4, 5, 6, 8])
def test_batch_every_register_budget(native, ctx, restatement, blocks_per_sm):
    """Each resident-CTA count launches the build whose register budget allows
    it (2 to 8 CTAs of 256 threads per SM, the leaner ones spilling); every one
    solves like the reference, and a repeated solve gives the same bits (the
    reduction order depends on the shape, not on the run)."""
    systems = small_batch(count=9, seed=31)
    b = native.Batch(ctx, systems)
    b.set_config(blocks_per_sm=blocks_per_sm)
    assert b.config()[0] == blocks_per_sm
    rhs = np.concatenate([s.rhs for s in systems])
    res, x = run_batch(native, ctx, b, rhs, np.zeros_like(rhs))
    check_against_oracle(restatement, systems, b.offsets, res, x)
    b.set_config(blocks_per_sm=blocks_per_sm)
    res2, x2 = run_batch(native, ctx, b, rhs, np.zeros_like(rhs))
    assert np.array_equal(x.view(np.uint64), x2.view(np.uint64))


def test_batch_rejections(native, ctx):
    systems = small_batch(count=2, seed=17)
    s = systems[0]
    bad = s.vals.copy().reshape(-1, s.bs)
    rows = np.repeat(np.arange(s.owned), np.diff(s.rowptr))
    bad[(s.cols == rows).nonzero()[0][0]] = 0.0          # singular diagonal
    with pytest.raises(native.OwtkError):
        native.Batch(ctx, [(s.owned, s.bs, s.rowptr, s.cols, bad.reshape(-1)), systems[1]])
    cols = s.cols.copy()
    cols[0] = s.owned                                      # column outside the system
    with pytest.raises(native.OwtkError):
        native.Batch(ctx, [(s.owned, s.bs, s.rowptr, cols, s.vals)])
    with pytest.raises(native.OwtkError):                 # block size above 32
        native.Batch(ctx, [(2, 33, [0, 1, 2], [0, 1], np.ones(66))])
    b = native.Batch(ctx, systems)
    rhs = np.concatenate([y.rhs for y in systems])
    res, x = run_batch(native, ctx, b, rhs, np.zeros_like(rhs), relative_tolerance=-1.0)
    assert all(r.status == 4 for r in res)
    assert not x.any()                                     # x untouched
