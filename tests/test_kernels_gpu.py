"""Device kernels through the C ABI against the reference-pinned fixtures.

FP64 SpMV, Jacobi, SSOR, split SSOR and ILU(k) results must equal the
reference's CPU results bit for bit (the device evaluates every term with the
reference's rounding order); FP32 kernels are held to a stated tolerance
against the FP64 reference.
"""
import numpy as np
import pytest

import cases
from conftest import assert_bitwise

pytestmark = pytest.mark.gpu


def dvec(native, ctx, c, values=None, fill=None):
    v = native.Vector(ctx, c["owned"], c["ghost"], c["bs"])
    if values is not None:
        v.upload(values)
    elif fill is not None:
        v.upload(np.full(v.size, fill))
    return v


def device_array(native, ctx, values, dtype=np.float64):
    """Plain device buffer holding `values` (for borrowed split coefficients)."""
    values = np.ascontiguousarray(values, dtype=dtype)
    v = native.Vector(ctx, max(values.size, 1), 0, 1, dtype=dtype)
    if values.size:
        v.upload(values)
    return v


def bsr(native, ctx, c, dtype=np.float64):
    return native.Matrix(ctx, "bsr", c["owned"], c["ghost"], c["bs"], c["rowptr"], c["cols"], c["vals"], dtype=dtype)


def split_matrix(native, ctx, c, keep):
    orp, oci, diag, off = cases.split_of(c)
    d, o = device_array(native, ctx, diag), device_array(native, ctx, off)
    keep += [d, o]
    return native.Matrix(ctx, "split", c["owned"], c["ghost"], c["bs"], orp, oci, diag_ptr=d.data_ptr,
                         off_ptr=o.data_ptr), d, o


@pytest.mark.parametrize("name", list(cases.SPMV_CASES))
def test_spmv_bitwise(native, ctx, golden, name):
    c = cases.build(name)
    n, bs = c["owned"], c["bs"]
    m = bsr(native, ctx, c)
    x = dvec(native, ctx, c, c["x"])
    y = dvec(native, ctx, c, fill=77.0)
    m.apply(x, y)
    out = y.download()
    assert_bitwise(out[: n * bs], golden[f"{name}/spmv"], "bsr spmv")
    assert (out[n * bs:] == 77.0).all(), "SpMV wrote ghost entries"
    keep = []
    sm, _, _ = split_matrix(native, ctx, c, keep)
    sm.apply(x, y)
    assert_bitwise(y.download()[: n * bs], golden[f"{name}/split_spmv"], "split spmv")


@pytest.mark.parametrize("name", list(cases.SPMV_CASES))
def test_apply_rows_bitwise(native, ctx, golden, name):
    """apply_rows (block_csr.hpp:198-215, split_block_csr.hpp:95-119): the
    listed rows (unsorted, one repeated) equal the whole apply's; the others
    and the ghosts keep what they held; an empty list changes nothing; a row
    past the owned ones is out of range."""
    c = cases.build(name)
    n, bs = c["owned"], c["bs"]
    rng = np.random.default_rng(n)
    rows = rng.permutation(n)[: max(1, n // 3)]
    rows = np.concatenate([rows, rows[:1]])
    listed = np.zeros(n, bool)
    listed[rows] = True
    x = dvec(native, ctx, c, c["x"])
    keep = []
    for kind, m, want in [("bsr", bsr(native, ctx, c), golden[f"{name}/spmv"]),
                          ("split", split_matrix(native, ctx, c, keep)[0], golden[f"{name}/split_spmv"])]:
        y = dvec(native, ctx, c, fill=77.0)
        m.apply_rows(x, y, rows)
        out = y.download()
        got = out[: n * bs].reshape(n, bs)
        assert_bitwise(got[listed], want.reshape(n, bs)[listed], f"{kind} apply_rows")
        assert (got[~listed] == 77.0).all() and (out[n * bs:] == 77.0).all(), f"{kind} apply_rows wrote other rows"
        m.apply_rows(x, y, np.zeros(0, np.uint64))
        assert_bitwise(y.download(), out, f"{kind} empty apply_rows")
        with pytest.raises(native.OwtkError) as err:
            m.apply_rows(x, y, [n])
        assert "out of range" in str(err.value)


@pytest.mark.parametrize("name", list(cases.DENSE_CASES))
def test_dense_apply_rows_bitwise(native, ctx, golden, name):
    c = cases.dense_case(**cases.DENSE_CASES[name])
    n, bs = c["owned"], c["bs"]
    m = native.Matrix(ctx, "dense", n, 0, bs, c["rowptr"], c["cols"], c["vals"])
    rows = np.arange(n)[::-2]
    listed = np.zeros(n, bool)
    listed[rows] = True
    x = dvec(native, ctx, c, c["x"])
    y = dvec(native, ctx, c, fill=5.0)
    m.apply_rows(x, y, rows)
    got = y.download().reshape(n, bs)
    assert_bitwise(got[listed], golden[f"{name}/spmv"].reshape(n, bs)[listed], "dense apply_rows")
    assert (got[~listed] == 5.0).all()


@pytest.mark.parametrize("side,bs", [(420, 3), (300, 2), (161, 5)])
def test_spmv_bitwise_many_tiles_per_cta(native, ctx, restatement, side, bs):
    # Thousands of 2048-value tiles: every persistent CTA streams several
    # tiles through its shared-memory ring (wrap-around of the stages), and
    # array lengths that are not whole 16-byte granules end in plain loads.
    c = cases.lattice_case(side=side, bs=bs, seed=side)
    n = c["owned"]
    expect = restatement.bsr_spmv(n, bs, c["rowptr"], c["cols"], c["vals"], c["x"])
    m = bsr(native, ctx, c)
    x = dvec(native, ctx, c, c["x"])
    y = dvec(native, ctx, c, fill=5.0)
    m.apply(x, y)
    assert_bitwise(y.download()[: n * bs], expect, "bsr spmv")
    orp, oci, diag, off = cases.split_of(c)
    expect = restatement.split_spmv(n, bs, orp, oci, diag, off, c["x"])
    keep = []
    sm, _, _ = split_matrix(native, ctx, c, keep)
    sm.apply(x, y)
    assert_bitwise(y.download()[: n * bs], expect, "split spmv")
    # Borrowed coefficients that are 8-byte but not 16-byte aligned take the
    # per-tile kernel; the result is the same.
    d = device_array(native, ctx, diag)
    o = device_array(native, ctx, np.concatenate([[0.0], off]))
    shifted = native.Matrix(ctx, "split", n, 0, bs, orp, oci, diag_ptr=d.data_ptr, off_ptr=o.data_ptr + 8)
    shifted.apply(x, y)
    assert_bitwise(y.download()[: n * bs], expect, "split spmv, unaligned coefficients")
    with pytest.raises(native.OwtkError):   # not even element-aligned
        native.Matrix(ctx, "split", n, 0, bs, orp, oci, diag_ptr=d.data_ptr, off_ptr=o.data_ptr + 4)
    # FP32 values through the same pipeline (4096-byte-smaller stages).
    m32 = bsr(native, ctx, c, dtype=np.float32)
    x32 = native.Vector(ctx, n, 0, bs, dtype=np.float32).upload(c["x"])
    y32 = native.Vector(ctx, n, 0, bs, dtype=np.float32)
    m32.apply(x32, y32)
    got = y32.download().astype(np.float64)
    ref = restatement.bsr_spmv(n, bs, c["rowptr"], c["cols"], c["vals"].astype(np.float32).astype(np.float64),
                               c["x"].astype(np.float32).astype(np.float64))
    bound = restatement.bsr_spmv(n, bs, c["rowptr"], c["cols"], np.abs(c["vals"]), np.abs(c["x"]))
    deg = np.repeat(np.diff(c["rowptr"]), bs)
    assert (np.abs(got - ref) <= (deg + 2) * np.finfo(np.float32).eps * bound + 1e-30).all()
    ctx.synchronize()


@pytest.mark.parametrize("name", list(cases.DENSE_CASES))
def test_dense_spmv_bitwise(native, ctx, golden, name):
    c = cases.dense_case(**cases.DENSE_CASES[name])
    m = native.Matrix(ctx, "dense", c["owned"], 0, c["bs"], c["rowptr"], c["cols"], c["vals"])
    x = dvec(native, ctx, c, c["x"])
    y = dvec(native, ctx, c)
    m.apply(x, y)
    assert_bitwise(y.download(), golden[f"{name}/spmv"], "dense spmv")


def test_spmv_known_answer(native, ctx):
    # tests/test_core.cpp:31-58
    m = native.Matrix(ctx, "bsr", 2, 0, 3, [0, 2, 4], [0, 1, 0, 1], [4, 5, 6, 1, 1, 1, 2, 2, 2, 3, 4, 5])
    x = native.Vector(ctx, 2, 0, 3).upload(np.arange(1.0, 7.0))
    y = native.Vector(ctx, 2, 0, 3)
    m.apply(x, y)
    assert y.download().tolist() == [8, 15, 24, 14, 24, 36]


@pytest.mark.parametrize("name", ["lattice8_bs3", "unsorted30_bs33", "long_rows_bs4"])
def test_spmv_fp32(native, ctx, golden, name):
    # FP32 values and FP32 accumulation: |y32 - y64| <= 8 * eps32 * sum|a||x| per entry.
    c = cases.build(name)
    n, bs = c["owned"], c["bs"]
    m = bsr(native, ctx, c, dtype=np.float32)
    x = native.Vector(ctx, n, c["ghost"], bs, dtype=np.float32).upload(c["x"])
    y = native.Vector(ctx, n, c["ghost"], bs, dtype=np.float32)
    m.apply(x, y)
    got = y.download()[: n * bs].astype(np.float64)
    ref = golden[f"{name}/spmv"]
    import oracle
    bound = oracle.Restatement().bsr_spmv(n, bs, c["rowptr"], c["cols"], np.abs(c["vals"]), np.abs(c["x"]))
    deg = np.repeat(np.diff(c["rowptr"]), bs)
    assert (np.abs(got - ref) <= (deg + 2) * np.finfo(np.float32).eps * bound + 1e-30).all()


def test_blas_bitwise_and_reductions(native, ctx, restatement):
    rng = np.random.default_rng(3)
    n, g, bs = 5003, 7, 3
    a, b = rng.uniform(-1, 1, (n + g) * bs), rng.uniform(-1, 1, (n + g) * bs)
    va = native.Vector(ctx, n, g, bs).upload(a)
    vb = native.Vector(ctx, n, g, bs).upload(b)
    m = n * bs
    native.axpy(0.37, va, vb)
    expect = b.copy()
    expect[:m] = b[:m] + 0.37 * a[:m]
    assert_bitwise(vb.download(), expect, "axpy (ghosts untouched)")
    native.scale(-1.5, vb)
    expect[:m] *= -1.5
    assert_bitwise(vb.download(), expect, "scale")
    out = native.Vector(ctx, n, g, bs)
    native.assign_linear_combination(out, 2.0, va, -0.5, vb)
    assert_bitwise(out.download()[:m], 2.0 * a[:m] + -0.5 * expect[:m], "linear combination")
    # Reductions: device tree order differs from the reference's 8-lane sum,
    # so FP64 results agree to 1e-13 relative (owned entries only).
    d = native.dot(va, vb)
    assert abs(d - restatement.dot(a[:m], expect[:m])) <= 1e-13 * np.abs(a[:m] * expect[:m]).sum()
    nr = native.norm(va)
    assert abs(nr - restatement.norm(a[:m])) <= 1e-14 * nr
    basis = [native.Vector(ctx, n, g, bs).upload(rng.uniform(-1, 1, (n + g) * bs)) for _ in range(9)]
    got = native.dot_batch(va, basis)
    host = [bv.download()[:m] for bv in basis]
    for j in range(9):
        assert abs(got[j] - restatement.dot(a[:m], host[j])) <= 1e-13 * m
    assert abs(got[9] - restatement.dot(a[:m], a[:m])) <= 1e-13 * m


def test_norm_edge_cases(native, ctx):
    # tests/test_foundation.cpp:72-105: owned-only, scaled, Inf/NaN survive.
    f = np.finfo(np.float64)
    v = native.Vector(ctx, 2, 1, 1)
    for mag in (1.0, f.max / 8, f.tiny * 4, np.nextafter(0, 1) * 4):
        v.upload(np.array([3 * mag, -4 * mag, np.inf]))
        got = native.norm(v)
        assert abs(got - 5 * mag) <= 1e-14 * 5 * mag or (mag < f.tiny and abs(got - 5 * mag) <= mag), mag
    v.upload(np.array([0.0, 0.0, np.nan]))
    assert native.norm(v) == 0.0
    v.upload(np.array([f.max, f.max, 0.0]))
    assert np.isinf(native.norm(v))
    v.upload(np.array([np.inf, 0.0, 0.0]))
    assert np.isinf(native.norm(v))
    v.upload(np.array([np.inf, np.nan, 0.0]))
    assert np.isnan(native.norm(v))


@pytest.mark.parametrize("name", list(cases.SPMV_CASES))
def test_jacobi_and_ssor_bitwise(native, ctx, golden, name):
    c = cases.build(name)
    n, bs = c["owned"], c["bs"]
    m = bsr(native, ctx, c)
    x = dvec(native, ctx, c, c["x"])
    y = dvec(native, ctx, c, fill=77.0)
    native.Preconditioner(m, native.PC_JACOBI).apply(x, y)
    assert_bitwise(y.download()[: n * bs], golden[f"{name}/jacobi"], "jacobi")
    for om in (1.0, 1.3):
        p = native.Preconditioner(m, native.PC_SSOR, om)
        p.apply(x, y)
        out = y.download()
        assert_bitwise(out[: n * bs], golden[f"{name}/ssor{om}"], f"ssor {om}")
        assert (out[n * bs:] == 77.0).all()
    keep = []
    sm, _, _ = split_matrix(native, ctx, c, keep)
    for om in (1.0, 1.4):
        p = native.Preconditioner(sm, native.PC_SPLIT_SSOR, om)
        p.apply(x, y)
        assert_bitwise(y.download()[: n * bs], golden[f"{name}/split_ssor{om}"], f"split ssor {om}")
        # In-place apply (overlapping views, tests/test_split_ssor.cpp:84-129).
        z = dvec(native, ctx, c, c["x"])
        p.apply(z, z)
        assert_bitwise(z.download()[: n * bs], golden[f"{name}/split_ssor{om}"], f"in-place split ssor {om}")
    ctx.synchronize()


def test_split_ssor_sees_borrowed_updates(native, ctx, restatement):
    c = cases.build("lattice8_bs3")
    n, bs = c["owned"], c["bs"]
    keep = []
    sm, d, o = split_matrix(native, ctx, c, keep)
    p = native.Preconditioner(sm, native.PC_SPLIT_SSOR, 1.0)
    orp, oci, diag, off = cases.split_of(c)
    x = dvec(native, ctx, c, c["x"])
    y = dvec(native, ctx, c)
    for rep in range(3):
        p.apply(x, y)
        expect = restatement.split_ssor_apply(n, bs, orp, oci, diag, off, 1.0, c["x"])
        assert_bitwise(y.download()[: n * bs], expect, f"repetition {rep}")
        diag = diag + 0.25
        d.upload(diag)          # borrowed coefficients: no update_values call
    p.update_values()
    assert p.numeric_updates == 2


@pytest.mark.parametrize("name", cases.ILU_CASES)
@pytest.mark.parametrize("level", [0, 1, 2])
def test_ilu_bitwise(native, ctx, golden, name, level):
    c = cases.build(name)
    n, bs = c["owned"], c["bs"]
    m = bsr(native, ctx, c)
    p = native.Preconditioner(m, native.PC_ILU, level)
    rp, ci, v, inv = p.ilu_factors()
    np.testing.assert_array_equal(rp.astype(np.int64), golden[f"{name}/ilu{level}_rowptr"])
    np.testing.assert_array_equal(ci.astype(np.int64), golden[f"{name}/ilu{level}_cols"])
    assert_bitwise(v, golden[f"{name}/ilu{level}_vals"], "factors")
    assert_bitwise(inv, golden[f"{name}/ilu{level}_inv"], "inverse diagonal")
    x = dvec(native, ctx, c, c["x"])
    y = dvec(native, ctx, c, fill=77.0)
    p.apply(x, y)
    out = y.download()
    assert_bitwise(out[: n * bs], golden[f"{name}/ilu{level}_apply"], "apply")
    assert (out[n * bs:] == 77.0).all(), "ILU wrote ghost entries"
    p.apply(x, x)   # in place (preconditioner.hpp:328-333)
    assert_bitwise(x.download()[: n * bs], golden[f"{name}/ilu{level}_apply"], "in-place apply")
    ctx.synchronize()


@pytest.mark.parametrize("side,bs", [(200, 3), (160, 1), (120, 4)])
def test_sweeps_bitwise_many_levels(native, ctx, restatement, side, bs):
    # Hundreds of levels and thousands of warp tasks: every lane publishes its
    # row from inside its polling loop while other lanes of its warp still
    # wait, and rows of later levels poll rows published by other warps.
    c = cases.lattice_case(side=side, bs=bs, seed=side + bs)
    n = c["owned"]
    m = bsr(native, ctx, c)
    x = dvec(native, ctx, c, c["x"])
    y = dvec(native, ctx, c, fill=77.0)
    p = native.Preconditioner(m, native.PC_ILU, 0)
    lo, up, dl, du = p.levels()
    assert dl > 100 and du > 100
    ref = restatement.ilu(n, bs, c["rowptr"], c["cols"], c["vals"], 0)
    for rep in range(2):
        p.apply(x, y)
        assert_bitwise(y.download()[: n * bs], ref.apply(c["x"]), f"ilu(0) apply {rep}")
    for om in (1.0, 1.3):
        code, expect = restatement.ssor_apply(n, bs, c["rowptr"], c["cols"], c["vals"], om, c["x"])
        assert code == 0
        native.Preconditioner(m, native.PC_SSOR, om).apply(x, y)
        assert_bitwise(y.download()[: n * bs], expect, f"ssor {om}")
    ctx.synchronize()


def test_ilu_levels_match_oracle(native, ctx, restatement):
    c = cases.build("lattice8_bs3")
    m = bsr(native, ctx, c)
    p = native.Preconditioner(m, native.PC_ILU, 0)
    lo, up, dl, du = p.levels()
    rp, ci, _, _ = p.ilu_factors()
    rlo, rup = restatement.levels(c["owned"], rp.astype(np.int64), ci.astype(np.int64))
    np.testing.assert_array_equal(lo, rlo)
    np.testing.assert_array_equal(up, rup)


def test_ilu_update_values(native, ctx, restatement):
    c = cases.build("lattice8_bs3")
    n, bs = c["owned"], c["bs"]
    m = bsr(native, ctx, c)
    p = native.Preconditioner(m, native.PC_ILU, 0)
    vals2 = c["vals"] * 1.1 + 0.01
    m.update_values(vals2)
    p.update_values(m)
    assert p.numeric_updates == 2
    ilu = restatement.ilu(n, bs, c["rowptr"], c["cols"], vals2, 0)
    _, _, v, inv, _, _ = ilu.factors()
    _, _, gv, ginv = p.ilu_factors()
    assert_bitwise(gv, v, "refactored values")
    assert_bitwise(ginv, inv, "refactored inverse diagonal")
    # A different pattern is rejected (preconditioner.hpp:286-302).
    other = cases.build("lattice7_bs1_ghost")
    m2 = native.Matrix(ctx, "bsr", n, 0, bs, c["rowptr"], np.roll(c["cols"], 1) % n, c["vals"])
    with pytest.raises(native.OwtkError) as e:
        p.update_values(m2)
    assert e.value.kind == "invalid_argument"
    del other


def test_preconditioner_errors(native, ctx):
    # Zero pivot (preconditioner.hpp:450-452, 478-481).
    m = native.Matrix(ctx, "bsr", 2, 0, 1, [0, 2, 4], [0, 1, 0, 1], [0.0, 1.0, 1.0, 1.0])
    with pytest.raises(native.OwtkError) as e:
        native.Preconditioner(m, native.PC_ILU, 0)
    assert e.value.kind == "zero_pivot"
    # Missing diagonal (preconditioner.hpp:422-424, block_csr.hpp:231-233).
    m = native.Matrix(ctx, "bsr", 2, 0, 1, [0, 1, 2], [1, 0], [1.0, 1.0])
    for kind in (native.PC_ILU, native.PC_JACOBI, native.PC_SSOR):
        with pytest.raises(native.OwtkError) as e:
            native.Preconditioner(m, kind, 1.0 if kind == native.PC_SSOR else 0.0)
        assert e.value.kind == "invalid_argument"
    # Duplicate columns (preconditioner.hpp:392-393).
    m = native.Matrix(ctx, "bsr", 2, 0, 1, [0, 2, 3], [0, 0, 1], [1.0, 1.0, 1.0])
    with pytest.raises(native.OwtkError) as e:
        native.Preconditioner(m, native.PC_ILU, 0)
    assert e.value.kind == "invalid_argument"
    # Singular diagonal (preconditioner.hpp:62-67) and SSOR omega range (:135-137).
    m = native.Matrix(ctx, "bsr", 2, 0, 1, [0, 1, 2], [0, 1], [1.0, 0.0])
    with pytest.raises(native.OwtkError):
        native.Preconditioner(m, native.PC_JACOBI)
    m = native.Matrix(ctx, "bsr", 2, 0, 1, [0, 1, 2], [0, 1], [1.0, 2.0])
    for om in (0.0, 2.0, -1.0):
        with pytest.raises(native.OwtkError):
            native.Preconditioner(m, native.PC_SSOR, om)
    # Layout mismatch (preconditioner.hpp:98-105).
    p = native.Preconditioner(m, native.PC_JACOBI)
    with pytest.raises(native.OwtkError):
        p.apply(native.Vector(ctx, 3, 0, 1), native.Vector(ctx, 3, 0, 1))
    # Invalid matrix storage (block_csr.hpp:281-300).
    with pytest.raises(native.OwtkError):
        native.Matrix(ctx, "bsr", 2, 0, 1, [0, 2, 1], [0, 1], [1.0, 1.0])
    with pytest.raises(native.OwtkError):
        native.Matrix(ctx, "bsr", 2, 0, 1, [0, 1, 2], [0, 5], [1.0, 1.0])
    ctx.synchronize()
