"""Checkpoints of the learned preconditioner (owtk_b200/checkpoint.py) on
the CPU: the binary format round-trips weights, Adam moments, step and
metadata; corruption, truncation and a wrong parameter count are rejected;
the committed trained network loads and records its training command."""
import os
import struct

import numpy as np
import pytest

from conftest import PKG

from owtk_b200 import checkpoint

P = 64 * 16 + 4 * 64 * 128 + 8 * 64   # encoder, 4 layers, decoder


def _arrays(seed=0):
    rng = np.random.default_rng(seed)
    return [rng.normal(size=P).astype(np.float32) for _ in range(3)]


def test_round_trip(tmp_path):
    p, m, v = _arrays()
    path = str(tmp_path / "net.owtkgnn")
    checkpoint.save(path, p, m, v, 1234, {"draws": 500, "loss_history": [1.0, 0.5]})
    ck = checkpoint.load(path, P)
    assert ck["step"] == 1234 and ck["metadata"] == {"draws": 500, "loss_history": [1.0, 0.5]}
    for a, b in zip((p, m, v), (ck["parameters"], ck["first_moment"], ck["second_moment"])):
        np.testing.assert_array_equal(a, b)
    # Little-endian header: magic, version, count, step, metadata length.
    head = open(path, "rb").read(32)
    assert head[:8] == b"OWTKGNN\x01"
    assert struct.unpack_from("<IIQ", head, 8) == (1, P, 1234)


def test_rejects_damage(tmp_path):
    p, m, v = _arrays(1)
    path = str(tmp_path / "net.owtkgnn")
    checkpoint.save(path, p, m, v, 7)
    data = bytearray(open(path, "rb").read())
    bad = tmp_path / "bad.owtkgnn"
    flipped = bytearray(data)
    flipped[100] ^= 0x01
    bad.write_bytes(bytes(flipped))
    with pytest.raises(ValueError, match="CRC"):
        checkpoint.load(str(bad))
    bad.write_bytes(bytes(data[:-9]))
    with pytest.raises(ValueError):
        checkpoint.load(str(bad))
    with pytest.raises(ValueError, match="parameters"):
        checkpoint.load(path, P + 1)
    bad.write_bytes(b"NOTAFILE" + bytes(data[8:]))
    with pytest.raises(ValueError, match="checkpoint"):
        checkpoint.load(str(bad))
    with pytest.raises(ValueError):
        checkpoint.save(path, p, m[:-1], v, 0)


def test_committed_network():
    path = os.path.join(PKG, "weights", "learned_anisotropic_bs3.owtkgnn")
    ck = checkpoint.load(path, P)
    meta = ck["metadata"]
    assert meta["draws"] == 500 and meta["train_vertices"] >= 190_000 and meta["epochs"] == 20
    assert "train_learned.py" in meta["command"]
    assert ck["step"] == meta["epochs"] * meta["draws"] * meta["pairs_per_draw"]
    hist = meta["loss_history"]
    assert hist[-1] < 0.2 * hist[0]
    assert np.all(np.isfinite(ck["parameters"])) and np.any(ck["parameters"] != 0)
