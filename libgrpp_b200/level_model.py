"""Learned grid-level model: host side.

The model predicts, per radial task (shell pair x centre with semilocal
potentials), the nested-grid level (0..8) at which libgrpp's adaptive type 2
quadrature stops (libgrpp/radial_type2_integral.c:285-315). The engine runs it
in-kernel (BF16 weights, FP32 accumulation) to order the grid walk deepest
task first; see include/libgrpp_b200.h for the parameter layout.

This module initialises parameter vectors, stores them as a versioned binary
with a checksum, generates training pairs with the engine's plain walk
(``libgrpp_b200_level_samples``), and trains with the engine's CUDA training
kernels (``libgrpp_b200_mlp_train``).
"""
from __future__ import annotations

import os
import struct
import zlib

import numpy as np

N_FEAT, N_HID, N_OUT = 12, 64, 9
OFF_W1 = 2 * N_FEAT
OFF_B1 = OFF_W1 + N_HID * N_FEAT
OFF_W2 = OFF_B1 + N_HID
OFF_B2 = OFF_W2 + N_HID * N_HID
OFF_W3 = OFF_B2 + N_HID
OFF_B3 = OFF_W3 + N_HID * N_HID
OFF_W4 = OFF_B3 + N_HID
OFF_B4 = OFF_W4 + N_OUT * N_HID
N_PARAMS = OFF_B4 + N_OUT  # 9761 (LIBGRPP_B200_LEVEL_MODEL_PARAMS)

MAGIC = b"GRPPLVL1"
MODEL_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "level_model.bin")


def init_params(X: np.ndarray, seed: int = 0) -> np.ndarray:
    """Parameter vector with the feature normalisation of X (mean, std; constant
    features get std 1) and He-initialised weights, zero biases."""
    X = np.asarray(X, dtype=np.float64)
    p = np.zeros(N_PARAMS, dtype=np.float32)
    mean = X.mean(axis=0)
    std = X.std(axis=0)
    std[std < 1e-6] = 1.0
    p[:N_FEAT] = mean
    p[N_FEAT:2 * N_FEAT] = std
    rng = np.random.default_rng(seed)
    for off, nout, nin in ((OFF_W1, N_HID, N_FEAT), (OFF_W2, N_HID, N_HID), (OFF_W3, N_HID, N_HID), (OFF_W4, N_OUT, N_HID)):
        p[off:off + nout * nin] = rng.normal(0.0, np.sqrt(2.0 / nin), nout * nin)
    return p


def save(params: np.ndarray, path: str = MODEL_FILE, meta: dict | None = None) -> None:
    """Binary: magic, parameter count (u32), CRC-32 of the payload (u32), metadata length
    (u32) + UTF-8 JSON metadata, then the FP32 parameters (little endian)."""
    import json
    payload = np.asarray(params, dtype="<f4").tobytes()
    m = json.dumps(meta or {}, sort_keys=True).encode()
    with open(path, "wb") as f:
        f.write(MAGIC + struct.pack("<III", N_PARAMS, zlib.crc32(payload), len(m)) + m + payload)


def load(path: str = MODEL_FILE):
    """(params, metadata); raises ValueError on a wrong magic, size or checksum."""
    import json
    with open(path, "rb") as f:
        data = f.read()
    if data[:8] != MAGIC:
        raise ValueError(f"{path}: not a level model file")
    n, crc, lm = struct.unpack("<III", data[8:20])
    meta = json.loads(data[20:20 + lm].decode())
    payload = data[20 + lm:]
    if n != N_PARAMS or len(payload) != 4 * N_PARAMS:
        raise ValueError(f"{path}: expected {N_PARAMS} parameters")
    if zlib.crc32(payload) != crc:
        raise ValueError(f"{path}: checksum mismatch")
    return np.frombuffer(payload, dtype="<f4").astype(np.float32), meta


def samples(lib, systems, max_tasks_per_batch: int = 200_000, seed: int = 0, per_system: int | None = None):
    """Training pairs from the engine's plain walk: for each system, its task list (or a
    seeded sample of per_system tasks), in batches; returns (X [n, 12], levels [n]) of the
    tasks that walked the grid."""
    rng = np.random.default_rng(seed)
    Xs, ys = [], []
    for S in systems:
        a, b, c = S.all_tasks()
        if per_system is not None and per_system < len(a):
            sel = np.sort(rng.choice(len(a), per_system, replace=False))
            a, b, c = a[sel], b[sel], c[sel]
        for s0 in range(0, len(a), max_tasks_per_batch):
            sl = slice(s0, s0 + max_tasks_per_batch)
            X, y = lib.level_samples(S.batch(a[sl], b[sl], c[sl]))
            keep = y >= 0
            Xs.append(X[keep])
            ys.append(y[keep])
    return np.concatenate(Xs), np.concatenate(ys)


def train(lib, X, y, epochs: int = 6, batch: int = 2048, lr: float = 2e-3, seed: int = 0):
    """Initialise from X and train on the GPU; returns (params, per-epoch mean loss)."""
    p0 = init_params(X, seed)
    return lib.mlp_train(p0, X, y, epochs=epochs, batch=batch, lr=lr, seed=seed)
