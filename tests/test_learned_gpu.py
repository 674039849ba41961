"""Learned preconditioner on the GPU: forward and gradients of the tensor-core
network against the FP64 restatement (oracle/gnn.py), training by the
device's own backward and Adam kernels, the preconditioner with its ILU(0)
fallback, and what training gains over the untrained (Jacobi) network.

Tolerances: activations and layer weights are BF16 (8-bit mantissa) with
FP32 accumulation, through four layers; the network's correction is held to
5% relative error; with the error loss gradients are held to cosine
similarity >= 0.99 and <= 10% relative error per weight tensor (the residual
term, which multiplies the output by A, to 0.98 and 20%).  Exact properties are checked exactly:
positive homogeneity (scaling by 2 is exact in every rounding), the untrained
network equals Jacobi, and a network whose every step fails hands each step
to ILU(0), reproducing ILU(0)-FGMRES bit for bit.
"""
import numpy as np
import pytest

import cases
from conftest import assert_bitwise

pytestmark = pytest.mark.gpu


def flat(p):
    return np.concatenate([p["we"].reshape(-1)] + [w.reshape(-1) for w in p["wl"]]
                          + [np.pad(p["wd"], ((0, 8 - p["wd"].shape[0]), (0, 0))).reshape(-1)]).astype(np.float32)


def unflat(v, bs):
    from oracle import gnn
    we = v[:64 * 16].reshape(64, 16).astype(np.float64)
    wl = [v[1024 + l * 8192: 1024 + (l + 1) * 8192].reshape(64, 128).astype(np.float64) for l in range(4)]
    wd = v[1024 + 4 * 8192:].reshape(8, 64)[:bs].astype(np.float64)
    return {"we": we, "wl": wl, "wd": wd}


def setup(native, ctx, side=24, bs=3, seed=21):
    from oracle import gnn
    c = cases.lattice_case(side=side, bs=bs, seed=seed)
    n = c["owned"]
    m = native.Matrix(ctx, "bsr", n, 0, bs, c["rowptr"], c["cols"], c["vals"])
    net = native.Learned(m, seed=3)
    g = gnn.Graph(n, bs, c["rowptr"], c["cols"], c["vals"])
    return c, m, net, g


def bf16_weights(bs, seed):
    """Random weights already representable in BF16 (so both sides use the same values)."""
    import torch
    from oracle import gnn
    p = gnn.init_weights(bs, seed)
    p["wd"] = np.random.default_rng(seed + 1).normal(0, 0.3, size=p["wd"].shape)
    v = flat(p)
    v = torch.from_numpy(v).to(torch.bfloat16).float().numpy()
    return v


def test_forward_matches_restatement(native, ctx):
    from oracle import gnn
    c, m, net, g = setup(native, ctx)
    n, bs = c["owned"], c["bs"]
    v = bf16_weights(bs, 7)
    net.set_parameters(v)
    assert np.array_equal(net.parameters(), v)
    r = np.random.default_rng(5).uniform(-1, 1, n * bs)
    x = native.Vector(ctx, n, 0, bs).upload(r)
    y = native.Vector(ctx, n, 0, bs)
    net.apply(x, y)
    got = y.download()
    ref = gnn.forward(g, unflat(v, bs), r)
    jac = (r.reshape(n, bs) / g.diag).reshape(-1)
    err = np.linalg.norm((got - jac) - (ref - jac)) / np.linalg.norm(ref - jac)
    assert err <= 5e-2, err
    # Positive homogeneity, exactly.
    x2 = native.Vector(ctx, n, 0, bs).upload(2.0 * r)
    net.apply(x2, y)
    assert_bitwise(y.download(), 2.0 * got, "M(2r) = 2 M(r)")
    # Untrained decoder: the Jacobi step (FP32 reciprocal of the diagonal).
    v0 = v.copy()
    v0[1024 + 4 * 8192:] = 0.0
    net.set_parameters(v0)
    net.apply(x, y)
    np.testing.assert_allclose(y.download(), jac, rtol=2e-7)


def test_tma_and_register_gather_agree(native, ctx, monkeypatch):
    # Both layer kernels aggregate neighbours in edge order with the same FP32
    # operations (BF16 edge weights), so the training forward pass (separate
    # FP32 decoder) and the gradients are identical.  An inference pass of the
    # register path decodes on the tensor cores (BF16 decoder weights), so its
    # output agrees to BF16 level with the TMA path's FP32 decoder.
    c, m, net, g = setup(native, ctx, side=40, seed=37)
    n, bs = c["owned"], c["bs"]
    assert not net.uses_tma
    monkeypatch.setenv("OWTK_GNN_TMA", "1")
    net2 = native.Learned(m, seed=3)
    monkeypatch.delenv("OWTK_GNN_TMA")
    assert net2.uses_tma
    v = bf16_weights(bs, 5)
    net.set_parameters(v)
    net2.set_parameters(v)
    rng = np.random.default_rng(3)
    r = native.Vector(ctx, n, 0, bs).upload(rng.uniform(-1, 1, n * bs))
    e = native.Vector(ctx, n, 0, bs).upload(rng.uniform(-1, 1, n * bs))
    y1, y2 = native.Vector(ctx, n, 0, bs), native.Vector(ctx, n, 0, bs)
    net.apply(r, y1)
    net2.apply(r, y2)
    a, b = y1.download(), y2.download()
    assert np.linalg.norm(a - b) <= 1e-2 * np.linalg.norm(b), np.linalg.norm(a - b) / np.linalg.norm(b)
    l1, g1 = net.loss_grad(r, e, want_grads=True)
    l2, g2 = net2.loss_grad(r, e, want_grads=True)
    assert l1 == l2 and np.array_equal(g1, g2)


@pytest.mark.parametrize("weights,loss_tol,cos_min,rel_max", [((1.0, 0.0), 5e-2, 0.99, 0.1),
                                                             ((0.1, 1.0), 0.15, 0.98, 0.2)])
def test_gradients_match_restatement(native, ctx, weights, loss_tol, cos_min, rel_max):
    # The residual term multiplies the network output by A, which roughly
    # doubles the relative BF16 error of the loss and its gradient.
    from oracle import gnn
    c, m, net, g = setup(native, ctx, side=20)
    n, bs = c["owned"], c["bs"]
    v = bf16_weights(bs, 11)
    net.set_parameters(v)
    net.set_loss_weights(*weights)
    rng = np.random.default_rng(13)
    r = rng.uniform(-1, 1, n * bs)
    e = rng.uniform(-1, 1, n * bs)
    loss, grads = net.loss_grad(native.Vector(ctx, n, 0, bs).upload(r), native.Vector(ctx, n, 0, bs).upload(e),
                                want_grads=True)
    rl, rg = gnn.loss_and_grad(g, unflat(v, bs), r, e, we=weights[0], wr=weights[1])
    assert abs(loss - rl) <= loss_tol * rl, (loss, rl)
    got = unflat(grads, bs)
    pairs = [("we", got["we"], rg["we"]), ("wd", got["wd"], rg["wd"])]
    pairs += [(f"wl{l}", got["wl"][l], rg["wl"][l]) for l in range(4)]
    for name, a, b in pairs:
        a, b = a.reshape(-1), b.reshape(-1)
        cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert cos >= cos_min and rel <= rel_max, (name, cos, rel)


def test_training_reduces_the_loss(native, ctx):
    c, m, net, g = setup(native, ctx, side=20, seed=23)
    n, bs = c["owned"], c["bs"]
    rng = np.random.default_rng(17)
    r = native.Vector(ctx, n, 0, bs).upload(rng.uniform(-1, 1, n * bs))
    e = native.Vector(ctx, n, 0, bs).upload(rng.uniform(-1, 1, n * bs))
    first = net.loss_grad(r, e)
    for _ in range(40):
        net.loss_grad(r, e)
        net.adam_step(3e-3)
    last = net.loss_grad(r, e)
    assert last < 0.8 * first, (first, last)


def test_fallback_takes_every_failed_step(native, ctx):
    # A network scaled to be useless fails every step: each one is handed to
    # ILU(0), so FGMRES reproduces ILU(0)-FGMRES bit for bit.
    c, m, net, g = setup(native, ctx, side=16, seed=29)
    n, bs = c["owned"], c["bs"]
    v = net.parameters()
    v[1024 + 4 * 8192:] = 1e6
    net.set_parameters(v)
    ilu = native.Preconditioner(m, native.PC_ILU, 0)
    pc = native.LearnedPreconditioner(net, ilu)
    b = native.Vector(ctx, n, 0, bs).upload(c["rhs"][: n * bs])
    x1, x2 = native.Vector(ctx, n, 0, bs), native.Vector(ctx, n, 0, bs)
    r1 = native.solve(native.FGMRES, m, pc, b, x1)
    r2 = native.solve(native.FGMRES, m, ilu, b, x2)
    apps, falls = pc.counts()
    assert apps == r1.preconditioner_applications and falls == apps
    assert r1.iterations == r2.iterations and r1.status == 0
    assert_bitwise(x1.download(), x2.download(), "fallback solution")


def test_fgmres_reuses_the_check_product(native, ctx):
    # FGMRES takes the network's residual-check product A z as its Arnoldi
    # vector when the network is bound to the solver's own operator.  The
    # same solve against a second Matrix holding the same values (no reuse:
    # FGMRES applies the operator itself) must give the same bits, the same
    # iterations and the same counted operator applications.
    c, m, net, g = setup(native, ctx, side=20, seed=31)
    n, bs = c["owned"], c["bs"]
    net.set_parameters(bf16_weights(bs, 9))
    m2 = native.Matrix(ctx, "bsr", n, 0, bs, c["rowptr"], c["cols"], c["vals"])
    ilu = native.Preconditioner(m, native.PC_ILU, 0)
    pc = native.LearnedPreconditioner(net, ilu)
    b = native.Vector(ctx, n, 0, bs).upload(c["rhs"][: n * bs])
    x1, x2 = native.Vector(ctx, n, 0, bs), native.Vector(ctx, n, 0, bs)
    r1 = native.solve(native.FGMRES, m, pc, b, x1)
    r2 = native.solve(native.FGMRES, m2, pc, b, x2)
    assert r1.status == 0 and r1.iterations == r2.iterations
    assert r1.operator_applications == r2.operator_applications
    assert r1.preconditioner_applications == r2.preconditioner_applications
    assert_bitwise(x1.download(), x2.download(), "solution with and without the reused product")


def test_trained_network_beats_untrained(native, ctx):
    # Train on residual/error pairs of ILU(0)-GMRES solves over a few
    # coefficient draws of an anisotropic mesh, then compare FGMRES
    # iterations with the trained network against the untrained one (the
    # Jacobi preconditioner) on a held-out draw.
    from owtk_b200 import learned
    systems = [learned.training_system(3000, seed=41, draw=d) for d in range(8)]
    held = learned.training_system(3000, seed=41, draw=99)
    s0 = systems[0]
    m0 = native.Matrix(ctx, "bsr", s0.owned, 0, s0.bs, s0.rowptr, s0.cols, s0.vals)
    net = native.Learned(m0, seed=1)
    hist = learned.train(ctx, net, systems, epochs=10, learning_rate=1e-3, pairs_per_system=6)
    assert hist[-1] < hist[0]
    mh = native.Matrix(ctx, "bsr", held.owned, 0, held.bs, held.rowptr, held.cols, held.vals)
    net.update_matrix(mh)
    trained = learned.fgmres_iterations(ctx, mh, native.LearnedPreconditioner(net), held.rhs)
    net.set_parameters(np.where(np.arange(net.parameter_count()) >= 1024 + 4 * 8192, 0.0, net.parameters()))
    untrained = learned.fgmres_iterations(ctx, mh, native.LearnedPreconditioner(net), held.rhs)
    assert trained < untrained, (trained, untrained)
    ilu = learned.fgmres_iterations(ctx, mh, native.Preconditioner(mh, native.PC_ILU, 0), held.rhs)
    assert trained <= ilu + 2, (trained, ilu)   # as good as ILU(0) in iterations
