"""Damped Jacobi corrections after the learned preconditioner's network step
(owtk_pc_learned_set_correction): z += omega D^-1 (v - A z), with D^-1 the
FP32 reciprocal diagonal the network uses, every operation rounded as written.
Checked bit for bit against the same arithmetic in numpy on the network's own
output, and through FGMRES (converged, the reused product still A z).
"""
import numpy as np
import pytest

import cases
from conftest import assert_bitwise

pytestmark = pytest.mark.gpu


def setup(native, ctx, side=30, seed=61):
    c = cases.lattice_case(side=side, bs=3, seed=seed)
    n = c["owned"]
    m = native.Matrix(ctx, "bsr", n, 0, 3, c["rowptr"], c["cols"], c["vals"])
    net = native.Learned(m, seed=3)          # untrained decoder: the network step is q = r / d
    ilu = native.Preconditioner(m, native.PC_ILU, 0)
    return c, n, m, net, ilu


@pytest.mark.parametrize("steps,omega", [(1, 1.0), (1, 0.7), (2, 0.7)])
def test_correction_bits(native, ctx, steps, omega):
    c, n, m, net, ilu = setup(native, ctx)
    plain = native.LearnedPreconditioner(net, ilu)
    corrected = native.LearnedPreconditioner(net, ilu)
    corrected.set_correction(steps, omega)
    r = np.random.default_rng(4).uniform(-1, 1, 3 * n)
    x = native.Vector(ctx, n, 0, 3).upload(r)
    y = native.Vector(ctx, n, 0, 3)
    plain.apply(x, y)
    z = y.download()
    assert plain.counts() == (1, 0), "the network step was not accepted"
    dinv = (1.0 / m.diagonal()).astype(np.float32).astype(np.float64)
    zv, az = native.Vector(ctx, n, 0, 3), native.Vector(ctx, n, 0, 3)
    for _ in range(steps):
        zv.upload(z)
        m.apply(zv, az)
        z = z + omega * (dinv * (r - az.download()))
    corrected.apply(x, y)
    assert corrected.counts() == (1, 0)
    assert_bitwise(y.download(), z, f"{steps} correction(s), omega {omega}")


def test_correction_in_fgmres(native, ctx):
    c, n, m, net, ilu = setup(native, ctx, side=40, seed=62)
    b = native.Vector(ctx, n, 0, 3).upload(c["rhs"][: 3 * n])
    opts = native.default_options(restart=30, relative_tolerance=1e-8)
    results = {}
    for steps in (0, 1):
        pc = native.LearnedPreconditioner(net, ilu)
        pc.set_correction(steps, 0.7)
        x = native.Vector(ctx, n, 0, 3)
        r = native.solve(native.FGMRES, m, pc, b, x, opts)
        assert r.status == 0, r.as_dict()
        assert r.true_residual_norm <= 1e-8 * np.linalg.norm(c["rhs"][: 3 * n])
        results[steps] = r
    # One more smoothing step per application: no more iterations than without.
    assert results[1].iterations <= results[0].iterations, (results[1].iterations, results[0].iterations)


def test_correction_arguments(native, ctx):
    c, n, m, net, ilu = setup(native, ctx, side=8)
    pc = native.LearnedPreconditioner(net, ilu)
    for steps, omega in [(9, 1.0), (1, 0.0), (1, 2.0)]:
        with pytest.raises(native.OwtkError):
            pc.set_correction(steps, omega)
    with pytest.raises(native.OwtkError):
        native.LearnedPreconditioner.set_correction(ilu, 1, 1.0)
