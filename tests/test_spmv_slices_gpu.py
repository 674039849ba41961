"""The component-diagonal BSR SpMV on its row-slice copy (slices of 32 rows,
lanes longest row first, steps packed without padding; rows longer than 48
entries through the row-list kernel), against the CPU restatement of
block_csr.hpp:192-215: FP64 bit for bit, FP32 bit for bit against the same
sequence evaluated in float32.  Row lengths mix empty rows, one-entry rows,
ordinary rows and long rows; the last slice is partial; columns reach the
ghosts; value updates refresh the copy.
"""
import numpy as np
import pytest

from conftest import assert_bitwise

pytestmark = pytest.mark.gpu


def mixed_rows(n, ghosts, bs, seed, long_every=97):
    rng = np.random.default_rng(seed)
    rowptr, cols = [0], []
    for r in range(n):
        if r % long_every == 5:
            length = int(rng.integers(49, 140))     # past the slice limit
        elif r % 13 == 7:
            length = 0                              # an empty row
        else:
            length = int(rng.integers(1, 12))
        row = rng.integers(0, n + ghosts, size=length)
        if length:
            row[0] = r
        cols.extend(row.tolist())
        rowptr.append(len(cols))
    rowptr = np.array(rowptr, np.int64)
    cols = np.array(cols, np.int64)
    vals = rng.uniform(-1.0, 1.0, size=cols.size * bs)
    x = rng.uniform(-1.0, 1.0, size=(n + ghosts) * bs)
    return rowptr, cols, vals, x


def float32_sequence(n, bs, rowptr, cols, vals, x):
    """y[r][c] = 0 + v0 x0 + v1 x1 + ... in float32 with every product and
    sum rounded, entry order (the FP32 instance of the reference loop)."""
    v = vals.astype(np.float32).reshape(-1, bs)
    xs = x.astype(np.float32).reshape(-1, bs)
    y = np.zeros((n, bs), np.float32)
    lens = np.diff(rowptr)
    for k in range(int(lens.max(initial=0))):
        rows = np.nonzero(lens > k)[0]
        e = rowptr[rows] + k
        y[rows] = (y[rows] + (v[e] * xs[cols[e]]).astype(np.float32)).astype(np.float32)
    return y.reshape(-1)


@pytest.mark.parametrize("n,ghosts,bs", [(1000, 7, 3), (517, 0, 1), (333, 3, 2), (2049, 11, 4), (31, 2, 3)])
def test_slices_bitwise_mixed_rows(native, ctx, restatement, n, ghosts, bs):
    rowptr, cols, vals, x = mixed_rows(n, ghosts, bs, seed=n + bs)
    m = native.Matrix(ctx, "bsr", n, ghosts, bs, rowptr, cols, vals)
    xv = native.Vector(ctx, n, ghosts, bs).upload(x)
    y = native.Vector(ctx, n, ghosts, bs).upload(np.full((n + ghosts) * bs, 9.0))
    m.apply(xv, y)
    out = y.download()
    assert_bitwise(out[: n * bs], restatement.bsr_spmv(n, bs, rowptr, cols, vals, x), "row-slice spmv")
    assert (out[n * bs:] == 9.0).all(), "SpMV wrote ghost entries"
    # New values through update_values: the slice copy follows them.
    vals2 = -2.0 * vals[::-1].copy()
    m.update_values(vals2)
    m.apply(xv, y)
    assert_bitwise(y.download()[: n * bs], restatement.bsr_spmv(n, bs, rowptr, cols, vals2, x),
                   "row-slice spmv after update_values")
    # FP32 storage: the same sequence in float32.
    m32 = native.Matrix(ctx, "bsr", n, ghosts, bs, rowptr, cols, vals, dtype=np.float32)
    x32 = native.Vector(ctx, n, ghosts, bs, dtype=np.float32).upload(x)
    y32 = native.Vector(ctx, n, ghosts, bs, dtype=np.float32)
    m32.apply(x32, y32)
    assert_bitwise(y32.download()[: n * bs], float32_sequence(n, bs, rowptr, cols, vals, x), "FP32 row-slice spmv")


def test_slices_repeated_applies_identical(native, ctx, restatement):
    """Thousands of slices over many resident warps: repeated applies give
    the same bits."""
    n, bs = 60_000, 3
    rowptr, cols, vals, x = mixed_rows(n, 0, bs, seed=5, long_every=4001)
    m = native.Matrix(ctx, "bsr", n, 0, bs, rowptr, cols, vals)
    xv = native.Vector(ctx, n, 0, bs).upload(x)
    y = native.Vector(ctx, n, 0, bs)
    want = restatement.bsr_spmv(n, bs, rowptr, cols, vals, x)
    for _ in range(3):
        m.apply(xv, y)
        assert_bitwise(y.download(), want, "row-slice spmv, repeated")


def float32_dense_sequence(n, bs, rowptr, cols, vals, x):
    """The dense-block loop in float32: per entry and block row the
    contribution from +0 over the block columns, then added to the row sum."""
    v = vals.astype(np.float32).reshape(-1, bs, bs)
    xs = x.astype(np.float32).reshape(-1, bs)
    y = np.zeros((n, bs), np.float32)
    lens = np.diff(rowptr)
    for k in range(int(lens.max(initial=0))):
        rows = np.nonzero(lens > k)[0]
        e = rowptr[rows] + k
        part = np.zeros((rows.size, bs), np.float32)
        for bc in range(bs):
            part = (part + (v[e, :, bc] * xs[cols[e], bc][:, None]).astype(np.float32)).astype(np.float32)
        y[rows] = (y[rows] + part).astype(np.float32)
    return y.reshape(-1)


@pytest.mark.parametrize("n,ghosts,bs", [(1000, 5, 3), (417, 0, 2), (655, 3, 4), (300, 0, 1)])
def test_dense_slices_bitwise_mixed_rows(native, ctx, restatement, n, ghosts, bs):
    """Dense bs x bs blocks on the row-slice copy: empty, ordinary and long
    rows, a partial last slice, ghost columns, value updates, FP32."""
    rowptr, cols, _, x = mixed_rows(n, ghosts, bs, seed=3 * n + bs)
    vals = np.random.default_rng(n).uniform(-1.0, 1.0, size=cols.size * bs * bs)
    m = native.Matrix(ctx, "dense", n, ghosts, bs, rowptr, cols, vals)
    xv = native.Vector(ctx, n, ghosts, bs).upload(x)
    y = native.Vector(ctx, n, ghosts, bs).upload(np.full((n + ghosts) * bs, 4.0))
    m.apply(xv, y)
    out = y.download()
    assert_bitwise(out[: n * bs], restatement.dense_spmv(n, bs, rowptr, cols, vals, x), "dense row-slice spmv")
    assert (out[n * bs:] == 4.0).all(), "SpMV wrote ghost entries"
    vals2 = 0.5 * vals[::-1].copy()
    m.update_values(vals2)
    m.apply(xv, y)
    assert_bitwise(y.download()[: n * bs], restatement.dense_spmv(n, bs, rowptr, cols, vals2, x),
                   "dense row-slice spmv after update_values")
    m32 = native.Matrix(ctx, "dense", n, ghosts, bs, rowptr, cols, vals, dtype=np.float32)
    x32 = native.Vector(ctx, n, ghosts, bs, dtype=np.float32).upload(x)
    y32 = native.Vector(ctx, n, ghosts, bs, dtype=np.float32)
    m32.apply(x32, y32)
    assert_bitwise(y32.download()[: n * bs], float32_dense_sequence(n, bs, rowptr, cols, vals, x),
                   "FP32 dense row-slice spmv")
