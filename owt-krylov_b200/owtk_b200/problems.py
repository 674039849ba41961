"""Seeded synthetic linear systems with the shapes of the benchmark configurations.

Every system is a vertex graph of a triangle mesh with a ``bs``-component
block per vertex.  The component-diagonal block-CSR matrix is built per
component ``c`` and undirected edge ``(i, j)`` as

    a_ij = -w_ij (1 + s_ij),   a_ji = -w_ij (1 - s_ij),
    w ~ U(0.5, 1.5),  s ~ U(-0.3, 0.3),
    a_ii = 1.05 * sum_j |a_ij| + U(0, 0.1),

with rows stored in ascending column order, the diagonal included.  RNG
streams are numpy PCG64 generators drawn in a fixed order (points, w, s,
diagonal noise, right-hand side), so a seed pins the system on any machine.
Point sets: jittered triangulated lattices, or Poisson-disk samples (the
stand-alone program lib/owtk_meshgen, run as a child process) triangulated
with Delaunay (scipy's Qhull).

Orderings: "rcm" relabels by reverse Cuthill-McKee, "hilbert" by the Hilbert
curve.  The builders take an optional ``rcm`` callable ``(n, rowptr, cols) ->
new_to_old`` that computes the RCM permutation; by default it is this
library's ``owtk_rcm_order``.  The reference's own ordering can be passed
instead, so a process that must not load this library (the CPU reference
timing) builds the same system.
"""
from __future__ import annotations

import math
import os
import subprocess
import tempfile
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_DIR = os.path.join(os.path.dirname(_HERE), "lib")


@dataclass
class BlockSystem:
    """Host arrays of one system: CSR pattern (int64), values, rhs, coordinates."""

    owned: int
    bs: int
    rowptr: np.ndarray
    cols: np.ndarray
    vals: np.ndarray            # component-diagonal: nnz*bs ; dense: nnz*bs*bs
    rhs: np.ndarray
    xy: np.ndarray | None = None
    ghost: int = 0
    kind: str = "bsr"           # "bsr" or "dense"
    meta: dict = field(default_factory=dict)

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1])

    def split(self):
        """Split diagonal/edge view arrays: (off_rowptr, off_cols, diag, off)."""
        bs = self.bs
        rows = np.repeat(np.arange(self.owned), np.diff(self.rowptr))
        is_diag = self.cols == rows
        diag = self.vals.reshape(-1, bs)[is_diag].reshape(-1).copy()
        off_mask = ~is_diag
        off_cols = self.cols[off_mask].copy()
        off = self.vals.reshape(-1, bs)[off_mask].reshape(-1).copy()
        counts = np.bincount(rows[off_mask], minlength=self.owned)
        off_rowptr = np.zeros(self.owned + 1, dtype=np.int64)
        np.cumsum(counts, out=off_rowptr[1:])
        return off_rowptr, off_cols, diag, off


MESHGEN = os.path.join(_LIB_DIR, "owtk_meshgen")


def poisson_disk(target: int, domain: str, seed: int) -> np.ndarray:
    """About ``target`` Poisson-disk points in the unit disk or the unit square
    (Bridson sampling by the program lib/owtk_meshgen in a child process)."""
    if not os.path.exists(MESHGEN):
        raise FileNotFoundError(f"mesh point generator not built: {MESHGEN} (run `make -C owt-krylov_b200`)")
    area = math.pi if domain == "disk" else 1.0
    radius = math.sqrt(0.616 * area / target)
    cap = int(target * 1.5) + 1024
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "points.f64")
        rc = subprocess.run([MESHGEN, repr(radius), "1" if domain == "disk" else "0", str(int(seed)), str(cap), out],
                            check=False).returncode
        if rc == 2:
            raise RuntimeError("Poisson-disk point buffer overflow")
        if rc != 0:
            raise RuntimeError(f"owtk_meshgen failed with exit code {rc}")
        return np.fromfile(out, dtype="<f8").reshape(-1, 2)


def delaunay_edges(xy: np.ndarray) -> np.ndarray:
    from scipy.spatial import Delaunay

    tri = Delaunay(xy).simplices.astype(np.int64)
    e = np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]])
    e.sort(axis=1)
    key = np.unique(e[:, 0] * xy.shape[0] + e[:, 1])
    return np.stack([key // xy.shape[0], key % xy.shape[0]], axis=1)


def lattice(nx: int, ny: int, jitter: float, rng, aspect: float = 1.0):
    """Jittered nx*ny lattice, every cell split along the same diagonal."""
    hx, hy = aspect / max(nx - 1, 1), 1.0 / max(ny - 1, 1)
    gx, gy = np.meshgrid(np.arange(nx) * hx, np.arange(ny) * hy)
    xy = np.stack([gx.ravel(), gy.ravel()], axis=1)
    xy += rng.uniform(-jitter, jitter, size=xy.shape) * np.array([hx, hy])
    idx = np.arange(nx * ny).reshape(ny, nx)
    horiz = np.stack([idx[:, :-1].ravel(), idx[:, 1:].ravel()], axis=1)
    vert = np.stack([idx[:-1, :].ravel(), idx[1:, :].ravel()], axis=1)
    diag = np.stack([idx[:-1, :-1].ravel(), idx[1:, 1:].ravel()], axis=1)
    edges = np.concatenate([horiz, vert, diag]).astype(np.int64)
    return xy, edges


def _assemble(n: int, edges: np.ndarray, bs: int, a_fwd, a_bwd, diag):
    """CSR (rows sorted by column) from edge coefficients and the diagonal."""
    i, j = edges[:, 0], edges[:, 1]
    rows = np.concatenate([np.arange(n), i, j])
    cols = np.concatenate([np.arange(n), j, i])
    order = np.argsort(rows * np.int64(n) + cols, kind="stable")
    rows, cols = rows[order], cols[order]
    if bs is None:
        vals = None
    else:
        vals = np.concatenate([diag, a_fwd, a_bwd])[order]
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=n), out=rowptr[1:])
    return rowptr, cols.astype(np.int64), vals


def pattern(n: int, edges: np.ndarray):
    rowptr, cols, _ = _assemble(n, edges, None, None, None, None)
    return rowptr, cols


def _coefficients(n: int, edges: np.ndarray, bs: int, rng):
    e = edges.shape[0]
    w = rng.uniform(0.5, 1.5, size=(e, bs))
    s = rng.uniform(-0.3, 0.3, size=(e, bs))
    a_fwd = -w * (1.0 + s)
    a_bwd = -w * (1.0 - s)
    absum = np.empty((n, bs))
    for c in range(bs):
        absum[:, c] = (np.bincount(edges[:, 0], weights=np.abs(a_fwd[:, c]), minlength=n)
                       + np.bincount(edges[:, 1], weights=np.abs(a_bwd[:, c]), minlength=n))
    diag = 1.05 * absum + rng.uniform(0.0, 0.1, size=(n, bs))
    return a_fwd, a_bwd, diag


def _relabel(edges: np.ndarray, new_to_old: np.ndarray):
    old_to_new = np.empty_like(new_to_old)
    old_to_new[new_to_old] = np.arange(new_to_old.shape[0])
    e = old_to_new[edges]
    return e


def component_diagonal_system(xy, edges, bs, rng, order="natural", rcm=None) -> BlockSystem:
    """Coefficients as documented above; optional RCM or Hilbert relabelling
    (``order`` may also be a precomputed new_to_old permutation)."""
    n = xy.shape[0]
    a_fwd, a_bwd, diag = _coefficients(n, edges, bs, rng)
    rhs = rng.uniform(-1.0, 1.0, size=n * bs)
    return _ordered_system(xy, edges, bs, a_fwd, a_bwd, diag, rhs, order, rcm)


def ordering(xy, edges, order: str, rcm=None) -> np.ndarray | None:
    """new_to_old of the named vertex order of a mesh (None for "natural")."""
    n = xy.shape[0]
    if order == "natural":
        return None
    if order == "rcm":
        rp, cp = pattern(n, edges)
        if rcm is None:
            from . import native
            rcm = native.rcm_order
        return np.asarray(rcm(n, rp, cp), dtype=np.int64)
    if order == "hilbert":
        from . import native
        return np.asarray(native.hilbert_order(xy), dtype=np.int64)
    raise ValueError(order)


def _ordered_system(xy, edges, bs, a_fwd, a_bwd, diag, rhs, order, rcm=None) -> BlockSystem:
    n = xy.shape[0]
    if isinstance(order, np.ndarray):
        new_to_old, name = order, "given"
    else:
        new_to_old, name = ordering(xy, edges, order, rcm), order
    meta = {"order": name}
    if new_to_old is not None:
        edges = _relabel(edges, new_to_old)
        flip = edges[:, 0] > edges[:, 1]
        a_fwd, a_bwd = np.where(flip[:, None], a_bwd, a_fwd), np.where(flip[:, None], a_fwd, a_bwd)
        edges = np.sort(edges, axis=1)
        diag = diag[new_to_old]
        rhs = rhs.reshape(n, bs)[new_to_old].reshape(-1)
        xy = xy[new_to_old]
    rowptr, cols, vals = _assemble(n, edges, bs, a_fwd, a_bwd, diag)
    return BlockSystem(n, bs, rowptr, cols, np.ascontiguousarray(vals).reshape(-1), rhs, xy,
                       meta=meta)


def angle_field(xy: np.ndarray, rng, modes: int = 6) -> np.ndarray:
    """Smooth random angle field: pi * sum of `modes` low-frequency sine modes
    with N(0, 1)/modes amplitudes, integer wave numbers in [-3, 3]."""
    k = rng.integers(-3, 4, size=(modes, 2))
    amp = rng.normal(0.0, 1.0, size=modes) / modes
    phase = rng.uniform(0.0, 2.0 * np.pi, size=modes)
    theta = np.zeros(xy.shape[0])
    for (kx, ky), a, ph in zip(k, amp, phase):
        theta += a * np.sin(2.0 * np.pi * (kx * xy[:, 0] + ky * xy[:, 1]) + ph)
    return np.pi * theta


def anisotropic_system(xy, edges, bs, rng, strength: float = 1e4, order="rcm", rcm=None) -> BlockSystem:
    """w_ij = 1 + strength (e_ij . d(x_ij))^2 per edge, with e_ij the unit edge
    vector and d the unit direction rotated by the smooth angle field at the
    edge midpoint; per component a skew s ~ U(-0.3, 0.3) (s_ji = -s_ij),
    a_ij = -w (1 + s); diagonal 1.05 sum |a| + U(0, 0.1); rhs U(-1, 1)."""
    n = xy.shape[0]
    i, j = edges[:, 0], edges[:, 1]
    mid = 0.5 * (xy[i] + xy[j])
    theta = angle_field(mid, rng)
    d = np.stack([np.cos(theta), np.sin(theta)], axis=1)
    ev = xy[j] - xy[i]
    ev /= np.linalg.norm(ev, axis=1, keepdims=True)
    w = 1.0 + strength * np.einsum("ij,ij->i", ev, d) ** 2
    s = rng.uniform(-0.3, 0.3, size=(edges.shape[0], bs))
    a_fwd = -w[:, None] * (1.0 + s)
    a_bwd = -w[:, None] * (1.0 - s)
    absum = np.empty((n, bs))
    for c in range(bs):
        absum[:, c] = (np.bincount(i, weights=np.abs(a_fwd[:, c]), minlength=n)
                       + np.bincount(j, weights=np.abs(a_bwd[:, c]), minlength=n))
    diag = 1.05 * absum + rng.uniform(0.0, 0.1, size=(n, bs))
    rhs = rng.uniform(-1.0, 1.0, size=n * bs)
    return _ordered_system(xy, edges, bs, a_fwd, a_bwd, diag, rhs, order, rcm)


def config4(n_target: int = 8_000_000, seed: int = 4, bs: int = 3, draw: int = 0,
            order: str = "rcm", rcm=None) -> BlockSystem:
    """Poisson-disk points in the unit square, Delaunay, anisotropic
    coefficients (draw `draw` of the coefficient stream), RCM-ordered, bs 3."""
    def build():
        xy, edges = disk_mesh(n_target, seed, domain="square")
        rng = np.random.default_rng([seed, draw])
        return anisotropic_system(xy, edges, bs, rng, order=order, rcm=rcm)

    sysm = _cached(f"square-{n_target}-{seed}-{bs}-{draw}-{order}", build)
    sysm.meta.update(config=f"poisson-square-{sysm.owned}-delaunay-anisotropic-{order}-bs{bs}", seed=seed, draw=draw)
    return sysm


def config0(seed: int = 0, side: int = 64, bs: int = 3) -> BlockSystem:
    """64x64 jittered triangulated lattice (4096 vertices), bs 3."""
    rng = np.random.default_rng(seed)
    xy, edges = lattice(side, side, 0.2, rng)
    sysm = component_diagonal_system(xy, edges, bs, rng)
    sysm.meta.update(config="lattice-64x64-bs3", seed=seed)
    return sysm


def batch_systems(count: int = 256, seed: int = 3, n_min: int = 5_000, n_max: int = 200_000,
                  block_sizes=(1, 2, 3, 4)) -> list:
    """The batching workload: `count` independent systems with vertex counts
    log-uniform in [n_min, n_max] on jittered triangulated lattices of aspect
    ratio U(1, 4), block sizes drawn from `block_sizes`, coefficients and
    right-hand sides as config0.  System i draws from its own stream
    (seed, i), so any subset regenerates identically."""
    rng = np.random.default_rng(seed)
    spec = []
    for _ in range(count):
        n = float(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
        aspect = float(rng.uniform(1.0, 4.0))
        bs = int(rng.choice(block_sizes))
        spec.append((n, aspect, bs))
    out = []
    for i, (n, aspect, bs) in enumerate(spec):
        ny = max(2, int(round(np.sqrt(n / aspect))))
        nx = max(2, int(round(n / ny)))
        srng = np.random.default_rng([seed, i])
        xy, edges = lattice(nx, ny, 0.2, srng, aspect)
        s = component_diagonal_system(xy, edges, bs, srng)
        s.meta.update(index=i, aspect=aspect, config=f"batch-{count}-{seed}")
        out.append(s)
    return out


def disk_mesh(n_target: int, seed: int, domain: str = "disk"):
    xy = poisson_disk(n_target, domain, seed)
    return xy, delaunay_edges(xy)


def _cached(key: str, build):
    """Optional on-disk cache (directory in OWTK_CACHE_DIR) for large systems."""
    root = os.environ.get("OWTK_CACHE_DIR")
    if not root:
        return build()
    path = os.path.join(root, key + ".npz")
    if os.path.exists(path):
        d = np.load(path)
        return BlockSystem(int(d["owned"]), int(d["bs"]), d["rowptr"], d["cols"], d["vals"], d["rhs"], d["xy"],
                           meta={"cached": path})
    s = build()
    os.makedirs(root, exist_ok=True)
    np.savez(path, owned=s.owned, bs=s.bs, rowptr=s.rowptr, cols=s.cols, vals=s.vals, rhs=s.rhs, xy=s.xy)
    return s


def config1(n_target: int = 2_000_000, seed: int = 1, bs: int = 3, order: str = "rcm", rcm=None) -> BlockSystem:
    """Poisson-disk points in the unit disk, Delaunay, RCM-ordered, bs 3."""
    def build():
        xy, edges = disk_mesh(n_target, seed)
        rng = np.random.default_rng(seed)
        return component_diagonal_system(xy, edges, bs, rng, order=order, rcm=rcm)

    sysm = _cached(f"disk-{n_target}-{seed}-{bs}-{order}", build)
    sysm.meta.update(config=f"poisson-disk-{sysm.owned}-delaunay-{order}-bs{bs}", seed=seed)
    return sysm


def config2(n_target: int = 2_000_000, seed: int = 1, bs: int = 3, order: str = "rcm", rcm=None) -> BlockSystem:
    """The config-1 disk mesh with dense bs x bs blocks (see dense_block_system)."""
    def build():
        xy, edges = disk_mesh(n_target, seed)
        rng = np.random.default_rng([seed, 2])
        return dense_block_system(xy, edges, bs, rng, order=order, rcm=rcm)

    sysm = _cached(f"disk-dense-{n_target}-{seed}-{bs}-{order}", build)
    sysm.kind = "dense"
    sysm.meta.update(config=f"poisson-disk-{sysm.owned}-delaunay-{order}-dense{bs}x{bs}", seed=seed)
    return sysm


def anisotropic_draws(n_target: int, seed: int, draws, bs: int = 3, order: str = "rcm", rcm=None):
    """Coefficient draws of one anisotropic unit-square mesh (mesh and
    ordering built once); yields (draw, BlockSystem)."""
    xy, edges = disk_mesh(n_target, seed, domain="square")
    perm = ordering(xy, edges, order, rcm)
    for d in draws:
        rng = np.random.default_rng([seed, d])
        s = anisotropic_system(xy, edges, bs, rng, order=perm if perm is not None else "natural")
        s.meta.update(draw=d, order=order)
        yield d, s


def dense_block_system(xy, edges, bs: int, rng, order: str = "natural", rcm=None) -> BlockSystem:
    """Dense bs x bs blocks: off-diagonal -w_ij (I + 0.3 R_ij), R ~ N(0,1)/3 drawn
    per direction; diagonal 1.1 * sum ||off||_1 * I + 0.05 N(0,1)."""
    n = xy.shape[0]
    new_to_old = ordering(xy, edges, order, rcm)
    if new_to_old is not None:
        edges = np.sort(_relabel(edges, new_to_old), axis=1)
        xy = xy[new_to_old]
    e = edges.shape[0]
    eye = np.eye(bs)
    w = rng.uniform(0.5, 1.5, size=e)
    r_fwd = rng.normal(0.0, 1.0, size=(e, bs, bs)) / 3.0
    r_bwd = rng.normal(0.0, 1.0, size=(e, bs, bs)) / 3.0
    b_fwd = -w[:, None, None] * (eye + 0.3 * r_fwd)
    b_bwd = -w[:, None, None] * (eye + 0.3 * r_bwd)
    norm1 = lambda b: np.abs(b).sum(axis=1).max(axis=1)   # induced 1-norm: max column sum
    acc = np.zeros(n)
    np.add.at(acc, edges[:, 0], norm1(b_fwd))
    np.add.at(acc, edges[:, 1], norm1(b_bwd))
    diag = 1.1 * acc[:, None, None] * eye + 0.05 * rng.normal(0.0, 1.0, size=(n, bs, bs))
    rhs = rng.uniform(-1.0, 1.0, size=n * bs)
    i, j = edges[:, 0], edges[:, 1]
    rows = np.concatenate([np.arange(n), i, j])
    cols = np.concatenate([np.arange(n), j, i])
    blocks = np.concatenate([diag, b_fwd, b_bwd])
    o = np.lexsort((cols, rows))
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=n), out=rowptr[1:])
    return BlockSystem(n, bs, rowptr, cols[o].astype(np.int64), blocks[o].reshape(-1), rhs, xy,
                       kind="dense", meta={"order": order})
