"""Product library on the CPU host: ABI exports, host setup (orderings, level
sets), option defaults and argument validation.  No kernel is launched here."""
import ctypes
import os
import re

import numpy as np
import pytest

import cases
from conftest import REPO


def declared_symbols():
    text = open(os.path.join(REPO, "include", "owtk.h")).read()
    return sorted(set(re.findall(r"\b(owtk_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(native):
    syms = declared_symbols()
    assert len(syms) > 40
    lib = ctypes.CDLL(native.LIB_PATH)
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_abi_version(native):
    assert native.lib().owtk_abi_version() == 1


def test_default_options_match_reference_defaults(native):
    # core.hpp:88-111
    o = native.default_options()
    assert o.relative_tolerance == 1e-8 and o.absolute_tolerance == 0
    assert o.breakdown_tolerance == 64 * np.finfo(np.float64).eps
    assert (o.maximum_iterations, o.convergence_check_interval, o.restart) == (1000, 10, 30)
    assert (o.residual_replacement_interval, o.idr_shadow_space) == (50, 4)
    assert o.gmres_orthogonalization == 0


def test_rcm_matches_reference(native, golden, problems, restatement):
    c0 = problems.config0()
    got = native.rcm_order(c0.owned, c0.rowptr, c0.cols)
    np.testing.assert_array_equal(got, golden["cfg0/rcm"])
    lat = cases.build("lattice8_bs3")
    np.testing.assert_array_equal(native.rcm_order(lat["owned"], lat["rowptr"], lat["cols"]),
                                  golden["lattice8_bs3/rcm"])
    # Random graphs with ghosts and several components.
    for seed in range(4):
        c = cases.unsorted_case(n=120, bs=1, seed=seed, ghosts=6, extra=2)
        np.testing.assert_array_equal(native.rcm_order(c["owned"], c["rowptr"], c["cols"], ghost=6),
                                      restatement.rcm(c["owned"], c["rowptr"], c["cols"]))


def test_rcm_disconnected_and_isolated_nodes(native, restatement):
    # Two components plus an isolated vertex: every component is seeded at
    # its minimum-degree vertex (ordering.hpp:146-154).
    rp = np.array([0, 2, 4, 5, 7, 9, 10, 11])
    ci = np.array([0, 1, 0, 1, 2, 3, 4, 3, 4, 5, 6])
    got = native.rcm_order(7, rp, ci)
    np.testing.assert_array_equal(got, restatement.rcm(7, rp, ci))
    assert sorted(got.tolist()) == list(range(7))


def test_hilbert_matches_reference(native, golden, problems):
    c0 = problems.config0()
    np.testing.assert_array_equal(native.hilbert_order(c0.xy), golden["cfg0/hilbert"])
    # Degenerate extent (all points on a line) keeps a valid permutation.
    xy = np.stack([np.linspace(0, 1, 50), np.zeros(50)], axis=1)
    assert sorted(native.hilbert_order(xy).tolist()) == list(range(50))


def test_inverse_permutation(native):
    p = np.random.default_rng(0).permutation(1000)
    inv = native.inverse_permutation(p)
    np.testing.assert_array_equal(inv[p], np.arange(1000))
    with pytest.raises(native.OwtkError) as e:
        native.inverse_permutation([0, 0, 1])
    assert e.value.kind == "invalid_argument"
    with pytest.raises(native.OwtkError):
        native.inverse_permutation([0, 5])


@pytest.mark.parametrize("name", ["lattice8_bs3", "lattice7_bs1_ghost", "unsorted40_bs2_dup", "long_rows_bs4"])
def test_level_sets_match_oracle(native, restatement, name):
    c = cases.build(name)
    lo, up, dl, du = native.level_sets(c["owned"], c["rowptr"], c["cols"])
    rlo, rup = restatement.levels(c["owned"], c["rowptr"], c["cols"])
    np.testing.assert_array_equal(lo, rlo)
    np.testing.assert_array_equal(up, rup)
    assert dl == rlo.max() + 1 and du == rup.max() + 1


def test_level_sets_are_valid_schedules(native, problems):
    c0 = problems.config0()
    lo, up, _, _ = native.level_sets(c0.owned, c0.rowptr, c0.cols)
    rows = np.repeat(np.arange(c0.owned), np.diff(c0.rowptr))
    low = c0.cols < rows
    assert (lo[rows[low]] > lo[c0.cols[low]]).all()
    high = c0.cols > rows
    assert (up[rows[high]] > up[c0.cols[high]]).all()


def test_context_without_device_reports_no_device(native):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    with pytest.raises(native.OwtkError) as e:
        native.Context(0)
    assert e.value.kind in ("no_device", "cuda_error")


def test_bindings_marshal_with_null_handles(native):
    # Every binding of the batching, tensor-core and learned entry points
    # converts its arguments and reaches the library, which rejects the null
    # handle with a status (no GPU needed).
    b = native.Batch.__new__(native.Batch)
    b.h, b.count = None, 2
    net = native.Learned.__new__(native.Learned)
    net.h = None
    ctx = native.Context.__new__(native.Context)
    ctx.h = None
    v = native.Vector.__new__(native.Vector)
    v.h = None
    calls = [b.layout, b.config, lambda: b.set_config(1, 3, 4), b.autotune, lambda: b.use_graph(True),
             b.graph_counts, lambda: b.solve_host(0, 0), lambda: native.Batch(ctx, [(2, 1, [0, 1, 2], [0, 1], [1.0, 1.0])]),
             net.parameters, lambda: net.set_parameters(np.zeros(native.Learned.parameter_count())),
             lambda: net.loss_grad(v, v, want_grads=True), lambda: net.adam_step(1e-3), lambda: net.apply(v, v),
             lambda: native.bf16_gemm_nt(ctx, 0, 0, 0, 128, 64, 64)]
    for call in calls:
        with pytest.raises(native.OwtkError):
            call()
    assert native.Learned.parameter_count() == 64 * 16 + 4 * 64 * 128 + 8 * 64
    b.h = net.h = None


def test_mesh_points_program_is_deterministic(problems):
    """lib/owtk_meshgen (a child process, so a reader maps no project library)
    gives the same Poisson-disk points for a seed, inside the domain and at
    least the sampling radius apart."""
    a = problems.poisson_disk(3000, "square", 11)
    b = problems.poisson_disk(3000, "square", 11)
    np.testing.assert_array_equal(a, b)
    assert 2000 < a.shape[0] < 4000
    assert np.all((a >= 0) & (a < 1))
    from scipy.spatial import cKDTree
    radius = np.sqrt(0.616 / 3000)
    d, _ = cKDTree(a).query(a, k=2)
    assert d[:, 1].min() >= radius * (1 - 1e-12)
    disk = problems.poisson_disk(2000, "disk", 3)
    assert np.all(np.hypot(disk[:, 0], disk[:, 1]) < 1)
    assert not np.array_equal(problems.poisson_disk(3000, "square", 12), a)
