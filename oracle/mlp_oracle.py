"""ORACLE — test infrastructure only.

CPU restatement (numpy) of the learned grid-level model's forward and backward
pass, the checker for the engine's CUDA training kernels
(libgrpp_b200/csrc/level_model.cuh: mlp_train_kernel). libgrpp has no
counterpart: the model is this project's addition; its layout is the one
documented in include/libgrpp_b200.h (LIBGRPP_B200_LEVEL_MODEL_PARAMS).

Semantics pinned here, as the kernels implement them:
  * features are normalised in FP32 as (x - mean) / std;
  * every weight and bias is rounded to BF16 (round to nearest even) before use;
  * 12 -> 64 -> 64 -> 64 with ReLU, 9 logits, softmax cross-entropy averaged over
    the samples; the gradient is taken w.r.t. the BF16-rounded values.
``grad(..., dtype=np.float64)`` evaluates the same in double precision, which
the tests use to pin this restatement with central finite differences.
"""
from __future__ import annotations

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
N_PARAMS = OFF_B4 + N_OUT

LAYERS = ((OFF_W1, OFF_B1, N_HID, N_FEAT), (OFF_W2, OFF_B2, N_HID, N_HID), (OFF_W3, OFF_B3, N_HID, N_HID),
          (OFF_W4, OFF_B4, N_OUT, N_HID))


def bf16_round(x: np.ndarray) -> np.ndarray:
    """float32 -> nearest BF16 value (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def _unpack(p, dtype, round_bf16):
    w = bf16_round(p) if round_bf16 else np.asarray(p, dtype=np.float32)
    w = w.astype(dtype)
    return [(w[o:o + no * ni].reshape(no, ni), w[b:b + no]) for o, b, no, ni in LAYERS]


def forward(params, X, dtype=np.float32, round_bf16=True):
    """Logits and the activations of every layer (input normalised first)."""
    p = np.asarray(params, dtype=np.float32)
    X = np.asarray(X, dtype=np.float32)
    x = ((X - p[:N_FEAT]) / p[N_FEAT:2 * N_FEAT]).astype(dtype)
    acts = [x]
    layers = _unpack(p, dtype, round_bf16)
    for k, (W, b) in enumerate(layers):
        z = acts[-1] @ W.T + b
        acts.append(np.maximum(z, 0) if k < 3 else z)
    return acts[-1], acts, layers


def grad(params, X, y, dtype=np.float32, round_bf16=True):
    """(mean cross-entropy, gradient in the parameter layout; normalisation slots 0)."""
    logits, acts, layers = forward(params, X, dtype, round_bf16)
    y = np.asarray(y, dtype=np.int64)
    n = len(y)
    m = logits.max(axis=1, keepdims=True)
    e = np.exp(logits - m)
    z = e.sum(axis=1, keepdims=True)
    loss = float(np.mean(-(logits[np.arange(n), y] - m[:, 0] - np.log(z[:, 0]))))
    d = e / z
    d[np.arange(n), y] -= 1.0
    d /= n
    g = np.zeros(N_PARAMS, dtype=np.float64)
    for k in range(3, -1, -1):
        o, b, no, ni = LAYERS[k]
        W, _ = layers[k]
        g[o:o + no * ni] = (d.T @ acts[k]).ravel()
        g[b:b + no] = d.sum(axis=0)
        if k > 0:
            d = (d @ W) * (acts[k] > 0)
    return loss, g


def predict(params, X):
    logits, _, _ = forward(params, X)
    return np.argmax(logits, axis=1).astype(np.int8)
