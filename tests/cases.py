"""Small seeded systems shared by the golden generator and the tests."""
import numpy as np

from owtk_b200 import problems


def lattice_case(side, bs, seed, ghosts=0):
    """Jittered triangulated lattice; the last `ghosts` vertices become ghost
    nodes (their rows are dropped, their columns stay as ghost columns)."""
    rng = np.random.default_rng(seed)
    xy, edges = problems.lattice(side, side, 0.2, rng)
    s = problems.component_diagonal_system(xy, edges, bs, rng)
    n = s.owned - ghosts
    rowptr = s.rowptr[: n + 1].copy()
    nnz = int(rowptr[-1])
    x = rng.uniform(-1.0, 1.0, size=s.owned * bs)
    return dict(owned=n, ghost=ghosts, bs=bs, rowptr=rowptr, cols=s.cols[:nnz].copy(),
                vals=s.vals[: nnz * bs].copy(), rhs=s.rhs[: (n + ghosts) * bs].copy(), x=x,
                xy=s.xy)


def unsorted_case(n, bs, seed, ghosts=0, duplicates=False, extra=4):
    """Random rows in random column order with a dominant diagonal, optional
    ghost columns and (for SpMV/SSOR, not ILU) duplicate columns."""
    rng = np.random.default_rng(seed)
    rowptr = [0]
    cols, vals = [], []
    for r in range(n):
        cand = set(rng.integers(0, n + ghosts, size=extra).tolist()) - {r}
        row = [r] + sorted(cand)
        if duplicates and r % 3 == 0 and len(row) > 1:
            row.append(row[1])
        rng.shuffle(row)
        for c in row:
            cols.append(c)
            if c == r:
                vals.append(4.0 + 0.5 * extra + rng.uniform(0.0, 0.5, size=bs))
            else:
                vals.append(-rng.uniform(0.05, 0.6, size=bs))
        rowptr.append(len(cols))
    x = rng.uniform(-1.0, 1.0, size=(n + ghosts) * bs)
    return dict(owned=n, ghost=ghosts, bs=bs, rowptr=np.array(rowptr, np.int64),
                cols=np.array(cols, np.int64), vals=np.concatenate(vals), x=x,
                rhs=rng.uniform(-1.0, 1.0, size=(n + ghosts) * bs))


def split_of(case):
    """Split diagonal/edge arrays of a case whose rows hold exactly one diagonal."""
    n, bs = case["owned"], case["bs"]
    rp, ci, v = case["rowptr"], case["cols"], case["vals"].reshape(-1, bs)
    rows = np.repeat(np.arange(n), np.diff(rp))
    is_diag = ci == rows
    diag = np.zeros((n, bs))
    diag[rows[is_diag]] = v[is_diag]
    off_rows = rows[~is_diag]
    off_rp = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(off_rows, minlength=n), out=off_rp[1:])
    return off_rp, ci[~is_diag].copy(), diag.reshape(-1), v[~is_diag].reshape(-1).copy()


def dense_case(side, bs, seed, hub=0):
    """Dense bs x bs blocks on a side x side lattice, or with hub > 0 on a
    star plus a path over `hub` vertices: row 0 couples to every row, so its
    block row (hub * bs * bs values) is longer than one SpMV tile stages."""
    rng = np.random.default_rng(seed)
    if hub:
        xy = rng.uniform(0.0, 1.0, size=(hub, 2))
        star = np.stack([np.zeros(hub - 1, np.int64), np.arange(1, hub)], axis=1)
        path = np.stack([np.arange(1, hub - 1), np.arange(2, hub)], axis=1)
        edges = np.concatenate([star, path])
    else:
        xy, edges = problems.lattice(side, side, 0.2, rng)
    s = problems.dense_block_system(xy, edges, bs, rng)
    x = rng.uniform(-1.0, 1.0, size=s.owned * bs)
    return dict(owned=s.owned, ghost=0, bs=bs, rowptr=s.rowptr, cols=s.cols, vals=s.vals, x=x, rhs=s.rhs)


# name -> (builder, kwargs)
SPMV_CASES = {
    "lattice8_bs3": (lattice_case, dict(side=8, bs=3, seed=11)),
    "lattice7_bs1_ghost": (lattice_case, dict(side=7, bs=1, seed=12, ghosts=5)),
    "lattice6_bs5_ghost": (lattice_case, dict(side=6, bs=5, seed=13, ghosts=4)),
    "unsorted40_bs2_dup": (unsorted_case, dict(n=40, bs=2, seed=14, ghosts=3, duplicates=True)),
    "unsorted30_bs33": (unsorted_case, dict(n=30, bs=33, seed=15, ghosts=2)),
    "unsorted6_bs1296": (unsorted_case, dict(n=6, bs=1296, seed=16, extra=3)),
    "long_rows_bs4": (unsorted_case, dict(n=600, bs=4, seed=17, ghosts=0, extra=1500)),
}
ILU_CASES = ["lattice8_bs3", "lattice7_bs1_ghost", "lattice6_bs5_ghost", "unsorted30_bs33"]
DENSE_CASES = {"dense5_bs3": dict(side=5, bs=3, seed=18), "dense4_bs2": dict(side=4, bs=2, seed=19),
               "dense4_bs4": dict(side=4, bs=4, seed=20), "dense4_bs5": dict(side=4, bs=5, seed=22),
               "dense_hub300_bs3": dict(side=0, bs=3, seed=23, hub=300)}


def build(name):
    fn, kw = SPMV_CASES[name]
    return fn(**kw)
