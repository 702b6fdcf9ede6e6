"""Weights file of the learned-split MLP (fkd_mlp_* in include/fkdtree_b200.h).

No reference counterpart (the reference has no learned part).  A trained
network is saved once and loaded by later processes instead of being
retrained.  Layout, little-endian:

    offset  size  field
    0       8     magic b"FKDMLP\\0\\1"
    8       4     format version (1)
    12      4     parameter count P
    16      4     storage: 0 = float32, 1 = bfloat16 (round to nearest even)
    20      16    layer widths: inputs 40, hidden 64, hidden 64, outputs 1
    36      28    zero
    64      P*4 or P*2   the parameters in fkd_mlp_get_params order:
                  W1[48][64] (rows 40..47 zero), b1[64], W2[64][64], b2[64], w3[64], b3

float32 storage round-trips exactly; bfloat16 halves the file and rounds
every parameter to the nearest bfloat16 (the precision the forward pass feeds
its tensor cores with, except for the float32 biases and output layer).
"""
from __future__ import annotations

import struct

import numpy as np

MAGIC = b"FKDMLP\x00\x01"
VERSION = 1
HEADER = 64
LAYERS = (40, 64, 64, 1)
STORAGE = {"f32": 0, "bf16": 1}


def param_count() -> int:
    return 48 * 64 + 64 + 64 * 64 + 64 + 64 + 1


def to_bf16_bits(x: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 bit patterns, round to nearest even (NaN kept NaN)."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    nan = (b & 0x7FFFFFFF) > 0x7F800000
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16).astype(np.uint16)
    r[nan] = ((b[nan] >> 16) | 0x40).astype(np.uint16)
    return r


def from_bf16_bits(h: np.ndarray) -> np.ndarray:
    return (np.asarray(h, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


def save_params(path, params, storage: str = "f32") -> None:
    p = np.ascontiguousarray(params, dtype=np.float32).reshape(-1)
    if p.size != param_count():
        raise ValueError(f"expected {param_count()} parameters, got {p.size}")
    if storage not in STORAGE:
        raise ValueError("storage must be 'f32' or 'bf16'")
    head = MAGIC + struct.pack("<III4I", VERSION, p.size, STORAGE[storage], *LAYERS)
    head += b"\x00" * (HEADER - len(head))
    body = p.astype("<f4").tobytes() if storage == "f32" else to_bf16_bits(p).astype("<u2").tobytes()
    with open(path, "wb") as f:
        f.write(head)
        f.write(body)


def load_params(path) -> np.ndarray:
    with open(path, "rb") as f:
        data = f.read()
    if len(data) < HEADER or data[:8] != MAGIC:
        raise ValueError(f"{path}: not an FKDTree MLP weights file")
    version, count, storage, *layers = struct.unpack("<III4I", data[8:36])
    if version != VERSION:
        raise ValueError(f"{path}: format version {version}, this library reads {VERSION}")
    if tuple(layers) != LAYERS or count != param_count():
        raise ValueError(f"{path}: network {tuple(layers)} with {count} parameters does not match {LAYERS}")
    width = {0: 4, 1: 2}.get(storage)
    if width is None:
        raise ValueError(f"{path}: unknown storage code {storage}")
    body = data[HEADER:]
    if len(body) != count * width:
        raise ValueError(f"{path}: truncated ({len(body)} of {count * width} bytes)")
    if storage == 0:
        return np.frombuffer(body, dtype="<f4").astype(np.float32)
    return from_bf16_bits(np.frombuffer(body, dtype="<u2"))
