"""Checkpoints of the learned preconditioner: weights and Adam state.

One little-endian binary file, so training can stop and resume:

    offset  size      field
    0       8         magic b"OWTKGNN\\x01"
    8       u32       format version (1)
    12      u32       parameter count P (owtk_learned_parameter_count())
    16      u64       Adam step t (its bias correction)
    24      u32       metadata length L in bytes
    28      u32       0 (reserved)
    32      f32[P]    parameters: encoder 64x16, 4 layers 64x128, decoder 8x64
            f32[P]    Adam first moment
            f32[P]    Adam second moment
            u8[L]     metadata, UTF-8 JSON (training command, data, loss history)
            u32       CRC-32 of every byte before it

Loading checks the magic, the version, the parameter count, the sizes and
the CRC, and raises ValueError on any mismatch.
"""
from __future__ import annotations

import json
import struct
import zlib

import numpy as np

MAGIC = b"OWTKGNN\x01"
VERSION = 1
_HEADER = struct.Struct("<8sIIQII")


def save(path: str, parameters, first_moment, second_moment, step: int, metadata: dict | None = None) -> None:
    p = np.ascontiguousarray(parameters, dtype="<f4")
    m = np.ascontiguousarray(first_moment, dtype="<f4")
    v = np.ascontiguousarray(second_moment, dtype="<f4")
    if not (p.ndim == m.ndim == v.ndim == 1 and p.size == m.size == v.size):
        raise ValueError("parameters and Adam moments must be flat arrays of one length")
    meta = json.dumps(metadata or {}, sort_keys=True).encode()
    body = _HEADER.pack(MAGIC, VERSION, p.size, int(step), len(meta), 0) + p.tobytes() + m.tobytes() + v.tobytes() + meta
    with open(path, "wb") as f:
        f.write(body)
        f.write(struct.pack("<I", zlib.crc32(body) & 0xFFFFFFFF))


def load(path: str, parameter_count: int | None = None) -> dict:
    """{"parameters", "first_moment", "second_moment", "step", "metadata"}."""
    with open(path, "rb") as f:
        data = f.read()
    if len(data) < _HEADER.size + 4:
        raise ValueError(f"{path}: truncated checkpoint")
    magic, version, count, step, meta_len, _ = _HEADER.unpack_from(data, 0)
    if magic != MAGIC or version != VERSION:
        raise ValueError(f"{path}: not a version-{VERSION} learned-preconditioner checkpoint")
    if parameter_count is not None and count != parameter_count:
        raise ValueError(f"{path}: {count} parameters, the network has {parameter_count}")
    want = _HEADER.size + 3 * 4 * count + meta_len + 4
    if len(data) != want:
        raise ValueError(f"{path}: {len(data)} bytes, expected {want}")
    (crc,) = struct.unpack_from("<I", data, want - 4)
    if zlib.crc32(data[: want - 4]) & 0xFFFFFFFF != crc:
        raise ValueError(f"{path}: CRC mismatch")
    off = _HEADER.size
    arrays = []
    for _ in range(3):
        arrays.append(np.frombuffer(data, dtype="<f4", count=count, offset=off).astype(np.float32))
        off += 4 * count
    meta = json.loads(data[off: off + meta_len].decode()) if meta_len else {}
    return {"parameters": arrays[0], "first_moment": arrays[1], "second_moment": arrays[2], "step": int(step),
            "metadata": meta}


def save_network(path: str, net, metadata: dict | None = None) -> None:
    """Weights and Adam state of a native.Learned network."""
    m, v, t = net.adam_state()
    save(path, net.parameters(), m, v, t, metadata)


def load_network(path: str, net, with_optimizer: bool = True) -> dict:
    """Load weights (and the Adam state) into a native.Learned network."""
    ck = load(path, net.parameter_count())
    net.set_parameters(ck["parameters"])
    if with_optimizer:
        net.set_adam_state(ck["first_moment"], ck["second_moment"], ck["step"])
    return ck
