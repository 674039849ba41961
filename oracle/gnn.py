"""FP64 restatement of the learned preconditioner network (test infrastructure).

This is the checker for the device forward, backward and Adam kernels of the
learned preconditioner (owt-krylov_b200/csrc/gnn.cu); it is never part of the
product path.  The reference has no learned preconditioner, so this file
states the network itself; parity is pinned by its own finite-difference
check (tests/test_gnn.py) and the device kernels are held to it within
BF16 tolerances.

Network (hidden H = 64, L = 4 layers, block size bs <= 8, no biases, so
M(alpha r) = alpha M(r) for alpha > 0):

  q      = r / diag                        the Jacobi step, per vertex and component
  sr, sq = rms(r), rms(q)                  (M(0) = 0)
  x_v    = [r_v / sr, q_v / sq, 0 ...]     16 input features
  h0     = x W_e^T                         W_e: H x 16
  layer  m_v = sum_{u in N(v), u != v} w_vu h_u,   w_vu = -mean_c a_vu,c / d_v,c
         y   = [h | m] W_l^T               W_l: H x 2H
         h   = h + relu(y)
  out    = q + sq (h W_d^T)                W_d: bs x H

The correction lives in the scale of the Jacobi step, so the weights stay of
order one whatever the magnitude of the diagonal.

Training loss of one (r, e) pair, with e the error that the residual r leaves
(A e = r):  we ||M(r) - e||^2 / ||e||^2 + wr ||r - A M(r)||^2 / ||r||^2  — the
error term and the residual term (how far one preconditioner step reduces the
residual); the device default weights are (0.1, 1).
"""
from __future__ import annotations

import numpy as np

HIDDEN = 64
LAYERS = 4
FEATURES = 16


class Graph:
    """Off-diagonal edges of a component-diagonal BSR matrix with the
    aggregation weights w_vu, plus the diagonal."""

    def __init__(self, owned, bs, rowptr, cols, vals):
        rowptr = np.asarray(rowptr, np.int64)
        cols = np.asarray(cols, np.int64)
        v = np.asarray(vals, np.float64).reshape(-1, bs)
        rows = np.repeat(np.arange(owned), np.diff(rowptr))
        diag_mask = cols == rows
        self.n, self.bs = owned, bs
        self.diag = np.zeros((owned, bs))
        self.diag[rows[diag_mask]] = v[diag_mask]
        off = ~diag_mask
        self.dst = rows[off]            # v (receiving vertex)
        self.src = cols[off]            # u (neighbour)
        self.w = -(v[off] / self.diag[self.dst]).mean(axis=1)
        self.a = v[off]                 # a_vu per component

    def matvec(self, x):
        """(A x)_v = d_v x_v + sum_u a_vu x_u."""
        y = self.diag * x
        np.add.at(y, self.dst, self.a * x[self.src])
        return y

    def matvec_t(self, x):
        y = self.diag * x
        np.add.at(y, self.src, self.a * x[self.dst])
        return y

    def aggregate(self, h):
        out = np.zeros_like(h)
        np.add.at(out, self.dst, self.w[:, None] * h[self.src])
        return out

    def aggregate_t(self, g):
        out = np.zeros_like(g)
        np.add.at(out, self.src, self.w[:, None] * g[self.dst])
        return out


def init_weights(bs: int, seed: int = 0, hidden: int = HIDDEN, layers: int = LAYERS):
    """Seeded initial weights (the device initialiser draws the same values
    from the same generator on the host)."""
    rng = np.random.default_rng(seed)
    we = rng.normal(0.0, 1.0 / np.sqrt(2 * bs), size=(hidden, FEATURES))
    we[:, 2 * bs:] = 0.0
    wl = [rng.normal(0.0, 0.5 / np.sqrt(2 * hidden), size=(hidden, 2 * hidden)) for _ in range(layers)]
    wd = np.zeros((bs, hidden))
    return {"we": we, "wl": wl, "wd": wd}


def forward(g: Graph, p, r, cache: bool = False):
    n, bs = g.n, g.bs
    r = np.asarray(r, np.float64).reshape(n, bs)
    q = r / g.diag
    sr, s = np.sqrt(np.mean(r * r)), np.sqrt(np.mean(q * q))
    if sr == 0.0:
        out = np.zeros_like(r)
        return (out.reshape(-1), None) if cache else out.reshape(-1)
    x = np.zeros((n, FEATURES))
    x[:, :bs] = r / sr
    x[:, bs:2 * bs] = q / s
    h = x @ p["we"].T
    hs, ms, ys = [h], [], []
    for w in p["wl"]:
        m = g.aggregate(h)
        y = np.concatenate([h, m], axis=1) @ w.T
        h = h + np.maximum(y, 0.0)
        ms.append(m)
        ys.append(y)
        hs.append(h)
    out = q + s * (h @ p["wd"].T)
    if cache:
        return out.reshape(-1), dict(s=s, x=x, hs=hs, ms=ms, ys=ys)
    return out.reshape(-1)


def loss_and_grad(g: Graph, p, r, e, we: float = 1.0, wr: float = 1.0):
    out, c = forward(g, p, r, cache=True)
    e = np.asarray(e, np.float64).reshape(-1)
    r = np.asarray(r, np.float64).reshape(-1)
    ee, rr = float(e @ e), float(r @ r)
    diff = out - e
    res = r - g.matvec(out.reshape(g.n, g.bs)).reshape(-1)
    loss = we * float(diff @ diff) / ee + wr * float(res @ res) / rr
    if c is None:
        return loss, {"we": np.zeros_like(p["we"]), "wl": [np.zeros_like(w) for w in p["wl"]],
                      "wd": np.zeros_like(p["wd"])}
    n, bs = g.n, g.bs
    dout = (2.0 * we / ee) * diff.reshape(n, bs) - (2.0 * wr / rr) * g.matvec_t(res.reshape(n, bs))
    dz = c["s"] * dout
    grads = {"wd": dz.T @ c["hs"][-1], "wl": [None] * len(p["wl"])}
    dh = dz @ p["wd"]
    for l in range(len(p["wl"]) - 1, -1, -1):
        h_in, m, y = c["hs"][l], c["ms"][l], c["ys"][l]
        dy = dh * (y > 0.0)
        grads["wl"][l] = dy.T @ np.concatenate([h_in, m], axis=1)
        dcat = dy @ p["wl"][l]
        dh = dh + dcat[:, :HIDDEN] + g.aggregate_t(dcat[:, HIDDEN:])
    grads["we"] = dh.T @ c["x"]
    return loss, grads


def adam_step(p, grads, state, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam step (bias-corrected) on every weight array, in place."""
    state["t"] = state.get("t", 0) + 1
    t = state["t"]
    flat_p = [p["we"]] + p["wl"] + [p["wd"]]
    flat_g = [grads["we"]] + grads["wl"] + [grads["wd"]]
    if "m" not in state:
        state["m"] = [np.zeros_like(a) for a in flat_p]
        state["v"] = [np.zeros_like(a) for a in flat_p]
    for a, gr, m, v in zip(flat_p, flat_g, state["m"], state["v"]):
        m *= beta1
        m += (1 - beta1) * gr
        v *= beta2
        v += (1 - beta2) * gr * gr
        mh = m / (1 - beta1 ** t)
        vh = v / (1 - beta2 ** t)
        a -= lr * mh / (np.sqrt(vh) + eps)
