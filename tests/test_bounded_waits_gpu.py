"""Failure detection without a GPU fault: every device-side wait of the
library is bounded, and a wait that runs out ends its launch with a status
bit that the host turns into OWTK_ERR_TIMEOUT while the context stays usable.

The hook owtk_debug_unpublished_dependency runs a two-row ILU forward sweep
whose only dependency is never published (a value that nothing writes), with
a short poll limit, so the wait runs out on purpose."""
import time

import numpy as np
import pytest

import cases
from conftest import assert_bitwise

pytestmark = pytest.mark.gpu


def test_unpublished_dependency_times_out(native, ctx, restatement):
    t = time.time()
    code = native.lib().owtk_debug_unpublished_dependency(ctx.h, 20000)
    elapsed = time.time() - t
    assert native.STATUS[code] == "timeout", native.lib().owtk_last_error()
    assert b"gave up waiting" in native.lib().owtk_last_error()
    assert elapsed < 30
    # The status word was cleared and the context still works: a sweep right
    # after is bit-exact against the oracle.
    c = cases.build("lattice8_bs3")
    n, bs = c["owned"], c["bs"]
    m = native.Matrix(ctx, "bsr", n, 0, bs, c["rowptr"], c["cols"], c["vals"])
    pc = native.Preconditioner(m, native.PC_ILU, 0)
    x = native.Vector(ctx, n, 0, bs).upload(c["x"][: n * bs])
    y = native.Vector(ctx, n, 0, bs)
    pc.apply(x, y)
    ilu = restatement.ilu(n, bs, c["rowptr"], c["cols"], c["vals"], 0)
    assert_bitwise(y.download(), ilu.apply(c["x"][: n * bs]), "ILU(0) apply after a timeout")


def test_poll_limit_is_validated(native, ctx):
    for bad in (0, (1 << 22) + 1):
        assert native.STATUS[native.lib().owtk_debug_unpublished_dependency(ctx.h, bad)] == "invalid_argument"
