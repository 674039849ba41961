"""Training of the learned preconditioner (owtk_learned_* in include/owtk.h).

Training pairs come from the plain ILU(0)-preconditioned GMRES solver: for a
coefficient draw of the anisotropic mesh, x* is the solve to rtol 1e-10 and
x_k the iterate after k iterations; each pair is (r_k = b - A x_k,
e_k = x* - x_k) — the residuals ILU(0)-GMRES leaves and the errors behind
them.  The loss and gradients (forward and backward kernels) and the Adam
step run on the GPU; this module only orchestrates.
"""
from __future__ import annotations

import numpy as np

from . import native, problems

ITERATES = (0, 1, 2, 4, 6, 8, 12, 16)


def training_system(n_target: int, seed: int = 41, draw: int = 0, bs: int = 3):
    """Coefficient draw `draw` of the anisotropic unit-square mesh."""
    return problems.config4(n_target, seed=seed, bs=bs, draw=draw)


def make_pairs(ctx, matrix, rhs: np.ndarray, pairs: int, rng=None):
    """(r_k, e_k) device vector pairs from ILU(0)-GMRES iterates."""
    n, bs = matrix.owned, matrix.bs
    ilu = native.Preconditioner(matrix, native.PC_ILU, 0)
    b = native.Vector(ctx, n, 0, bs).upload(rhs)
    xs = native.Vector(ctx, n, 0, bs)
    r = native.solve(native.FGMRES, matrix, ilu, b, xs, native.default_options(relative_tolerance=1e-10))
    if r.status != 0:
        raise RuntimeError(f"training solve did not converge: {r.as_dict()}")
    xstar = xs.download()
    ks = ITERATES[:pairs] if rng is None else sorted(rng.choice(ITERATES, size=pairs, replace=False))
    out = []
    for k in ks:
        xk = native.Vector(ctx, n, 0, bs)
        if k > 0:
            native.solve(native.FGMRES, matrix, ilu, b, xk, native.default_options(maximum_iterations=int(k),
                                                                                   relative_tolerance=0.0))
        xkh = xk.download()
        ax = native.Vector(ctx, n, 0, bs)
        matrix.apply(xk, ax)
        rk = rhs - ax.download()
        ek = xstar - xkh
        if not np.any(ek):
            continue
        out.append((native.Vector(ctx, n, 0, bs).upload(rk), native.Vector(ctx, n, 0, bs).upload(ek)))
    return out


def train(ctx, net, systems, epochs: int = 4, learning_rate: float = 1e-3, pairs_per_system: int = 4,
          seed: int = 0, final_learning_rate=None, log=None):
    """Adam over all pairs of all systems for `epochs` passes; returns the
    mean loss of each epoch (the first is the untrained loss).  With
    `final_learning_rate` the rate decays geometrically from `learning_rate`
    to it over the epochs.  `systems` may be a generator: only the device
    copies (matrix and pairs) of each system are kept."""
    rng = np.random.default_rng(seed)
    data = []
    for s in systems:
        m = native.Matrix(ctx, "bsr", s.owned, 0, s.bs, s.rowptr, s.cols, s.vals)
        data.append((m, make_pairs(ctx, m, s.rhs, pairs_per_system)))
        del s
    history = []
    for ep in range(epochs + 1):
        lr = learning_rate
        if final_learning_rate is not None and epochs > 1 and ep > 0:
            lr = learning_rate * (final_learning_rate / learning_rate) ** ((ep - 1) / (epochs - 1))
        losses = []
        order = rng.permutation(len(data))
        for i in order:
            m, pairs = data[i]
            net.update_matrix(m)
            for r, e in pairs:
                loss = net.loss_grad(r, e)
                if not np.isfinite(loss):
                    raise FloatingPointError(f"training loss is {loss} (epoch {ep})")
                losses.append(loss)
                if ep > 0:
                    net.adam_step(lr)
        history.append(float(np.mean(losses)))
        if log is not None:
            log(f"epoch {ep}/{epochs}: rate {lr:.2e} mean loss {history[-1]:.5f}")
    return history


def fgmres_iterations(ctx, matrix, pc, rhs: np.ndarray, rtol: float = 1e-8, restart: int = 30) -> int:
    n, bs = matrix.owned, matrix.bs
    b = native.Vector(ctx, n, 0, bs).upload(rhs)
    x = native.Vector(ctx, n, 0, bs)
    r = native.solve(native.FGMRES, matrix, pc, b, x, native.default_options(relative_tolerance=rtol,
                                                                            restart=restart))
    return int(r.iterations) if r.status == 0 else 10 ** 9
