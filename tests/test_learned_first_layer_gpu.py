"""Inference with the encoder folded into the first message-passing layer
(block sizes 1-4): against the FP64 network restatement (oracle/gnn.py) and
against the unfused kernels (encoder, then the first layer; selected with
OWTK_GNN_FUSED_FIRST=0).  Both evaluate the same network with BF16 operands,
rounded at different points (the folded path rounds the inputs and their
aggregate, the unfused one the encoder output), so they agree to BF16 level,
not bit for bit.  Rows with more than 8 neighbours take the CSR continuation.
"""
import numpy as np
import pytest

import cases
from conftest import assert_bitwise
from test_learned_gpu import bf16_weights, unflat

pytestmark = pytest.mark.gpu


def build(native, ctx, case, monkeypatch):
    from oracle import gnn
    n, bs = case["owned"], case["bs"]
    m = native.Matrix(ctx, "bsr", n, 0, bs, case["rowptr"], case["cols"], case["vals"])
    fused = native.Learned(m, seed=3)
    monkeypatch.setenv("OWTK_GNN_FUSED_FIRST", "0")
    plain = native.Learned(m, seed=3)
    monkeypatch.delenv("OWTK_GNN_FUSED_FIRST")
    return m, fused, plain, gnn.Graph(n, bs, case["rowptr"], case["cols"], case["vals"])


@pytest.mark.parametrize("bs,shape", [(1, "lattice"), (2, "lattice"), (3, "lattice"), (4, "lattice"),
                                      (3, "dense_rows")])
def test_fused_first_layer(native, ctx, monkeypatch, bs, shape):
    from oracle import gnn
    if shape == "lattice":
        case = cases.lattice_case(side=36, bs=bs, seed=40 + bs)
    else:   # about 13 off-diagonal neighbours per row: every tile continues past the 8 slots
        case = cases.unsorted_case(n=700, bs=bs, seed=44, extra=14)
    n = case["owned"]
    m, fused, plain, g = build(native, ctx, case, monkeypatch)
    v = bf16_weights(bs, 9)
    fused.set_parameters(v)
    plain.set_parameters(v)
    r = np.random.default_rng(bs).uniform(-1, 1, n * bs)
    x = native.Vector(ctx, n, 0, bs).upload(r)
    yf, yp = native.Vector(ctx, n, 0, bs), native.Vector(ctx, n, 0, bs)
    fused.apply(x, yf)
    plain.apply(x, yp)
    got, base = yf.download(), yp.download()
    ref = gnn.forward(g, unflat(v, bs), r)
    jac = (r.reshape(n, bs) / g.diag).reshape(-1)
    err = np.linalg.norm((got - jac) - (ref - jac)) / np.linalg.norm(ref - jac)
    assert err <= 5e-2, err
    diff = np.linalg.norm((got - jac) - (base - jac)) / np.linalg.norm(base - jac)
    assert diff <= 2e-2, diff
    # Positive homogeneity stays exact: scaling by 2 moves no rounding.
    x2 = native.Vector(ctx, n, 0, bs).upload(2.0 * r)
    fused.apply(x2, yf)
    assert_bitwise(yf.download(), 2.0 * got, "M(2r) = 2 M(r)")
    # The stage timer reports the folded layer only where it ran.
    assert fused.stage_times(x, yf, 2)["encoder_first_layer"] > 0.0
    assert plain.stage_times(x, yp, 2)["encoder_first_layer"] == 0.0


def test_fused_first_layer_follows_new_weights(native, ctx, monkeypatch):
    """The folded operand is rebuilt whenever the weights change (set or
    trained): after an Adam step the fused and unfused passes still agree."""
    case = cases.lattice_case(side=30, bs=3, seed=51)
    n = case["owned"]
    m, fused, plain, _ = build(native, ctx, case, monkeypatch)
    rng = np.random.default_rng(8)
    r = native.Vector(ctx, n, 0, 3).upload(rng.uniform(-1, 1, 3 * n))
    e = native.Vector(ctx, n, 0, 3).upload(rng.uniform(-1, 1, 3 * n))
    v = bf16_weights(3, 12)
    for net in (fused, plain):
        net.set_parameters(v)
        net.loss_grad(r, e)
        net.adam_step(1e-2)
    assert np.array_equal(fused.parameters(), plain.parameters())
    yf, yp = native.Vector(ctx, n, 0, 3), native.Vector(ctx, n, 0, 3)
    fused.apply(r, yf)
    plain.apply(r, yp)
    a, b = yf.download(), yp.download()
    assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b), np.linalg.norm(a - b) / np.linalg.norm(b)


def test_fused_first_layer_many_tiles_per_cta(native, ctx, monkeypatch):
    """More 128-row tiles than resident CTAs (90,000 vertices against at most
    4 CTAs on each SM): every CTA walks several tiles, taking the next tile's
    slot lists ahead and alternating its two output tiles."""
    case = cases.lattice_case(side=300, bs=3, seed=57)
    n = case["owned"]
    assert n > 148 * 4 * 128
    m, fused, plain, _ = build(native, ctx, case, monkeypatch)
    v = bf16_weights(3, 14)
    fused.set_parameters(v)
    plain.set_parameters(v)
    r = np.random.default_rng(57).uniform(-1, 1, 3 * n)
    x = native.Vector(ctx, n, 0, 3).upload(r)
    yf, yp = native.Vector(ctx, n, 0, 3), native.Vector(ctx, n, 0, 3)
    fused.apply(x, yf)
    plain.apply(x, yp)
    a, b = yf.download(), yp.download()
    assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b), np.linalg.norm(a - b) / np.linalg.norm(b)
    again = native.Vector(ctx, n, 0, 3)
    fused.apply(x, again)
    assert_bitwise(again.download(), a, "repeated application")
