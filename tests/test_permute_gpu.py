"""Device permutation and ingestion from an application's split layout
(split_block_csr.hpp:17-28), through the C ABI.

The permutation is the reference's own RCM order; P A P^T built on the device
from device-resident diagonal/edge arrays must equal the same matrix permuted
on the host (rows relabelled, entries sorted by new column): its SpMV and its
ILU(0) factors are compared bit for bit with the oracle on the host-permuted
arrays.  The numeric update re-gathers new coefficients on the device."""
import numpy as np
import pytest

import cases
from conftest import assert_bitwise

pytestmark = pytest.mark.gpu


def host_permuted(n, bs, orp, oci, diag, off, n2o):
    o2n = np.empty_like(n2o)
    o2n[n2o] = np.arange(n)
    rowptr, cols, vals = [0], [], []
    d = diag.reshape(n, bs)
    f = off.reshape(-1, bs)
    for i in range(n):
        o = n2o[i]
        row = [(i, d[o])] + [(int(o2n[oci[k]]), f[k]) for k in range(orp[o], orp[o + 1])]
        row.sort(key=lambda t: t[0])
        cols += [c for c, _ in row]
        vals += [v for _, v in row]
        rowptr.append(len(cols))
    return np.array(rowptr, np.int64), np.array(cols, np.int64), np.concatenate(vals)


def test_permuted_split_ingestion(native, ctx, restatement, reference):
    c = cases.lattice_case(side=24, bs=3, seed=21)
    n, bs = c["owned"], c["bs"]
    orp, oci, diag, off = cases.split_of(c)
    n2o = reference.rcm(n, c["rowptr"], c["cols"])
    np.testing.assert_array_equal(native.inverse_permutation(n2o), reference.inverse_permutation(n2o))
    P = native.Permutation(ctx, n2o)
    d_diag = native.Vector(ctx, n, 0, bs).upload(diag)
    d_off = native.Vector(ctx, off.size // bs, 0, bs).upload(off)
    A = P.permuted_split_matrix(bs, orp, oci, d_diag, d_off)
    rp, ci, v = host_permuted(n, bs, orp, oci, diag, off, n2o)
    x = c["x"][: n * bs]
    xv = native.Vector(ctx, n, 0, bs).upload(x)
    y = native.Vector(ctx, n, 0, bs)
    A.apply(xv, y)
    assert_bitwise(y.download(), restatement.bsr_spmv(n, bs, rp, ci, v, x), "permuted SpMV")
    pc = native.Preconditioner(A, native.PC_ILU, 0)
    _, _, fv, finv = pc.ilu_factors()
    ilu = restatement.ilu(n, bs, rp, ci, v, 0)
    _, _, gv, ginv, _, _ = ilu.factors()
    assert_bitwise(fv, gv, "ILU(0) factors of P A P^T")
    assert_bitwise(finv, ginv, "inverse diagonal of P A P^T")
    # Numeric update: new coefficients in the borrowed arrays, gathered again.
    off2 = off * 1.5
    d_off.upload(off2)
    native.update_permuted_split(A, d_diag, d_off)
    A.apply(xv, y)
    rp2, ci2, v2 = host_permuted(n, bs, orp, oci, diag, off2, n2o)
    assert_bitwise(y.download(), restatement.bsr_spmv(n, bs, rp2, ci2, v2, x), "SpMV after the numeric update")


def test_vector_permute(native, ctx, reference):
    rng = np.random.default_rng(5)
    n, ghost, bs = 1000, 3, 4
    n2o = rng.permutation(n)
    P = native.Permutation(ctx, n2o)
    src = rng.uniform(-1, 1, (n + ghost) * bs)
    a = native.Vector(ctx, n, ghost, bs).upload(src)
    b = native.Vector(ctx, n, ghost, bs).upload(np.full(src.size, 7.0))
    P.apply(a, b)
    got = b.download()
    assert_bitwise(got[: n * bs], src[: n * bs].reshape(n, bs)[n2o].reshape(-1), "forward")
    assert np.all(got[n * bs:] == 7.0)   # ghosts untouched
    back = native.Vector(ctx, n, ghost, bs)
    P.apply(b, back, inverse=True)
    assert_bitwise(back.download()[: n * bs], src[: n * bs], "inverse undoes forward")
    with pytest.raises(native.OwtkError):
        native.Permutation(ctx, np.array([0, 1, 1, 3]))
    with pytest.raises(native.OwtkError):
        P.apply(a, a)
