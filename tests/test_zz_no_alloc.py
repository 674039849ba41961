"""owtk_dot_batch_f64_noalloc — the allocation-free batched dot product.

Callers that cannot allocate device memory (a framework that owns the
device allocator, or code where cudaMalloc is forbidden) use this entry
point: it takes caller-owned device inputs and outputs and keeps its
reduction scratch in a static device array.  This test drives it through
the C ABI and checks it, on two calls in a row (the scratch keeps the
previous call's contents, so the second call shows nothing stale leaks
through), against owtk_dot_batch, the allocating entry point, and against an
independent host answer: the exactly rounded sum (math.fsum) of the same
products.  It builds its own data, so it passes alone in a fresh process as
well as after the other tests.
"""
import ctypes
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def entry(native):
    fn = native.lib().owtk_dot_batch_f64_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t, ctypes.c_size_t,
                   ctypes.c_void_p, ctypes.c_void_p]
    return fn


def run_noalloc(native, ctx, fn, w, basis, out):
    ptrs = (ctypes.c_void_p * max(1, len(basis)))(*[b.data_ptr for b in basis])
    n = w.owned * w.bs
    code = fn(w.data_ptr, ptrs, len(basis), n, out.data_ptr, ctx.stream)
    native.check(code)
    ctx.synchronize()
    return out.download()[: len(basis) + 1]


def test_noalloc_dot_batch_matches_allocating_entry_point(native, ctx):
    fn = entry(native)
    rng = np.random.default_rng(2024)
    owned, ghost, bs, k = 33335, 4, 3, 7
    size = (owned + ghost) * bs
    w = native.Vector(ctx, owned, ghost, bs).upload(rng.uniform(-1, 1, size))
    basis = [native.Vector(ctx, owned, ghost, bs).upload(rng.uniform(-1, 1, size)) for _ in range(k)]
    out = native.Vector(ctx, k + 1, 0, 1)
    for call in range(2):
        if call == 1:   # new data for the second call
            w.upload(rng.uniform(-2, 2, size))
            basis[3].upload(rng.uniform(-3, 3, size))
        got = run_noalloc(native, ctx, fn, w, basis, out)
        expect = native.dot_batch(w, basis)
        wh = w.download()[: owned * bs]
        for j in range(k + 1):
            other = basis[j].download()[: owned * bs] if j < k else wh
            products = wh * other
            scale = np.abs(products).sum()
            exact = math.fsum(products.tolist())
            assert abs(got[j] - exact) <= 1e-13 * scale, (call, j, got[j], exact)
            assert abs(got[j] - expect[j]) <= 1e-13 * scale, (call, j, got[j], expect[j])


def test_noalloc_limits(native, ctx):
    fn = entry(native)
    w = native.Vector(ctx, 100, 0, 1).upload(np.ones(100))
    basis = [native.Vector(ctx, 100, 0, 1).upload(np.full(100, float(j))) for j in range(32)]
    out = native.Vector(ctx, 33, 0, 1)
    got = run_noalloc(native, ctx, fn, w, basis[:31], out)        # the maximum batch
    assert np.allclose(got, [100.0 * j for j in range(31)] + [100.0])
    ptrs = (ctypes.c_void_p * 32)(*[b.data_ptr for b in basis])
    code = fn(w.data_ptr, ptrs, 32, 100, out.data_ptr, ctx.stream)  # one too many
    assert native.STATUS[code] == "invalid_argument"
    assert "at most 31" in native.lib().owtk_last_error().decode()
