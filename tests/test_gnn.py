"""The FP64 network restatement (oracle/gnn.py) pinned by finite differences,
homogeneity and a descending Adam run — the checker the device kernels of the
learned preconditioner are held to."""
import numpy as np

import cases


def tiny_graph(bs=3, side=6, seed=4):
    from oracle import gnn
    c = cases.lattice_case(side=side, bs=bs, seed=seed)
    return gnn.Graph(c["owned"], bs, c["rowptr"], c["cols"], c["vals"]), c


def random_weights(bs, seed):
    from oracle import gnn
    p = gnn.init_weights(bs, seed)
    p["wd"] = np.random.default_rng(seed + 1).normal(0, 0.2, size=p["wd"].shape)
    return p


def test_gradients_match_finite_differences():
    from oracle import gnn
    g, c = tiny_graph()
    p = random_weights(3, 5)
    rng = np.random.default_rng(9)
    r = rng.uniform(-1, 1, g.n * 3)
    e = rng.uniform(-1, 1, g.n * 3)
    loss, grads = gnn.loss_and_grad(g, p, r, e)
    assert loss > 0
    checks = [("we", None, (0, 1)), ("we", None, (7, 4)), ("wd", None, (2, 11)), ("wl", 0, (3, 70)),
              ("wl", 3, (60, 5)), ("wl", 2, (10, 100))]
    for name, layer, idx in checks:
        arr = p[name] if layer is None else p[name][layer]
        gr = grads[name] if layer is None else grads[name][layer]
        h = 1e-6
        old = arr[idx]
        arr[idx] = old + h
        lp, _ = gnn.loss_and_grad(g, p, r, e)
        arr[idx] = old - h
        lm, _ = gnn.loss_and_grad(g, p, r, e)
        arr[idx] = old
        fd = (lp - lm) / (2 * h)
        assert abs(fd - gr[idx]) <= 1e-6 * max(1.0, abs(fd)), (name, layer, idx, fd, gr[idx])


def test_network_is_positively_homogeneous_and_starts_as_jacobi():
    from oracle import gnn
    g, c = tiny_graph(bs=2, seed=8)
    r = np.random.default_rng(2).uniform(-1, 1, g.n * 2)
    p0 = gnn.init_weights(2, 0)
    # Zero decoder: the untrained network is the Jacobi preconditioner.
    np.testing.assert_allclose(gnn.forward(g, p0, r), (r.reshape(-1, 2) / g.diag).reshape(-1), rtol=1e-14)
    p = random_weights(2, 3)
    np.testing.assert_allclose(gnn.forward(g, p, 3.5 * r), 3.5 * gnn.forward(g, p, r), rtol=1e-12)
    assert not gnn.forward(g, p, np.zeros_like(r)).any()


def test_adam_reduces_the_loss():
    from oracle import gnn
    g, c = tiny_graph(seed=12)
    p = random_weights(3, 7)
    rng = np.random.default_rng(1)
    r = rng.uniform(-1, 1, g.n * 3)
    e = rng.uniform(-1, 1, g.n * 3)
    first, _ = gnn.loss_and_grad(g, p, r, e)
    state = {}
    for _ in range(60):
        _, grads = gnn.loss_and_grad(g, p, r, e)
        gnn.adam_step(p, grads, state, lr=3e-3)
    last, _ = gnn.loss_and_grad(g, p, r, e)
    assert last < 0.7 * first
