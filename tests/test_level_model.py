"""Learned grid-level model: the numpy oracle (oracle/mlp_oracle.py) pinned by finite
differences; the model file format; the CUDA training and inference kernels against the
oracle; the learned walk against the plain walk; and what the trained model gains over
the model-free prediction (the most frequent level)."""
import os
import sys

import numpy as np
import pytest

from libgrpp_b200 import level_model, synthetic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import mlp_oracle  # noqa: E402


def _random_problem(n=48, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, 12)).astype(np.float32) * 2 + 1
    y = rng.integers(0, 9, n).astype(np.int8)
    p = level_model.init_params(X, seed)
    p[level_model.OFF_B1:level_model.OFF_B1 + 64] = rng.normal(0, 0.1, 64)  # non-zero biases
    return p, X, y


def test_layout_constants_agree():
    assert level_model.N_PARAMS == mlp_oracle.N_PARAMS == 9761
    with open(os.path.join(ROOT, "include", "libgrpp_b200.h")) as f:
        assert "#define LIBGRPP_B200_LEVEL_MODEL_PARAMS 9761" in f.read()


def test_oracle_gradient_matches_finite_differences():
    p, X, y = _random_problem()
    loss, g = mlp_oracle.grad(p, X, y, dtype=np.float64, round_bf16=False)
    rng = np.random.default_rng(1)
    idx = np.concatenate([rng.integers(mlp_oracle.OFF_W1, mlp_oracle.N_PARAMS, 60),
                          np.arange(mlp_oracle.OFF_B4, mlp_oracle.N_PARAMS)])
    h = 1e-6  # small enough that no ReLU changes side
    for i in idx:
        pp, pm = p.astype(np.float64), p.astype(np.float64)
        pp = pp.copy()
        pm = pm.copy()
        pp[i] += h
        pm[i] -= h
        # the oracle reads float32 parameters: evaluate the perturbed loss in float64 directly
        lp = _loss64(pp, X, y)
        lm = _loss64(pm, X, y)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * abs(g[i]) + 1e-8, (i, fd, g[i])
    assert abs(_loss64(p.astype(np.float64), X, y) - loss) < 1e-12


def _loss64(p64, X, y):
    """Cross-entropy with float64 parameters (no BF16 rounding), for finite differences."""
    p32 = p64.astype(np.float32)
    a = ((X - p32[:12]) / p32[12:24]).astype(np.float64)  # normalised in FP32, as the model does
    for k, (o, b, no, ni) in enumerate(mlp_oracle.LAYERS):
        z = a @ p64[o:o + no * ni].reshape(no, ni).T + p64[b:b + no]
        a = np.maximum(z, 0) if k < 3 else z
    m = a.max(axis=1, keepdims=True)
    lz = np.log(np.exp(a - m).sum(axis=1)) + m[:, 0]
    return float(np.mean(lz - a[np.arange(len(y)), y.astype(int)]))


def test_bf16_rounding():
    # BF16 keeps 7 mantissa bits: the spacing at 1.0 is 2^-7
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.14159265], dtype=np.float32)
    r = mlp_oracle.bf16_round(x)
    assert r[0] == 1.0
    assert r[1] == 1.0  # exactly halfway: ties to the even neighbour
    assert r[2] == np.float32(1.0078125)
    assert r[3] == np.float32(-2.5)
    assert r[4] == np.float32(3.140625)


def test_model_file_roundtrip(tmp_path):
    p, X, _ = _random_problem()
    f = str(tmp_path / "m.bin")
    level_model.save(p, f, {"note": "test"})
    q, meta = level_model.load(f)
    assert np.array_equal(p, q) and meta["note"] == "test"
    raw = bytearray(open(f, "rb").read())
    raw[-5] ^= 0x10
    open(f, "wb").write(bytes(raw))
    with pytest.raises(ValueError, match="checksum"):
        level_model.load(f)


def test_committed_model_is_valid():
    if not os.path.exists(level_model.MODEL_FILE):
        pytest.skip("no trained model committed")
    p, meta = level_model.load()
    assert np.all(np.isfinite(p)) and np.all(p[12:24] > 0)
    assert meta["held_out_mean_abs_error"] < meta["majority_mean_abs_error"]


# ------------------------------------------------------------------------------ GPU
@pytest.mark.gpu
def test_cuda_gradient_matches_oracle(gpu_lib):
    p, X, y = _random_problem(n=100, seed=3)
    g_gpu, l_gpu = gpu_lib.mlp_grad(p, X, y)
    l_orc, g_orc = mlp_oracle.grad(p, X, y)
    assert abs(l_gpu - l_orc) <= 1e-5 * abs(l_orc)
    scale = np.abs(g_orc).max()
    err = np.abs(g_gpu - g_orc).max()
    print(f"mlp gradient: max |gpu - oracle| = {err:.2e} (max |grad| {scale:.2e}), loss {l_gpu:.6f} vs {l_orc:.6f}")
    assert err <= 1e-4 * scale


@pytest.mark.gpu
def test_cuda_inference_matches_oracle(gpu_lib):
    p, X, _ = _random_problem(n=4000, seed=4)
    got = gpu_lib.mlp_predict(p, X)
    want = mlp_oracle.predict(p, X)
    logits, _, _ = mlp_oracle.forward(p, X)
    top2 = np.sort(logits, axis=1)[:, -2:]
    clear = (top2[:, 1] - top2[:, 0]) > 1e-4 * np.abs(top2[:, 1]).clip(1.0)
    assert np.array_equal(got[clear], want[clear])


@pytest.mark.gpu
def test_cuda_training_learns(gpu_lib):
    """Labels that are a fixed function of two features: training must beat the majority."""
    rng = np.random.default_rng(5)
    X = rng.normal(size=(20000, 12)).astype(np.float32)
    y = np.clip(np.round(2 * X[:, 0] + X[:, 3] + 4), 0, 8).astype(np.int8)
    p0 = level_model.init_params(X, 0)
    p, losses = gpu_lib.mlp_train(p0, X, y, epochs=8, batch=512, lr=3e-3)
    assert losses[-1] < 0.5 * losses[0]
    acc = np.mean(gpu_lib.mlp_predict(p, X) == y)
    assert acc > 0.85 > np.mean(y == np.bincount(y).argmax())


def _model_or_skip():
    if not os.path.exists(level_model.MODEL_FILE):
        pytest.skip("no trained model committed")
    return level_model.load()[0]


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["config1", "config2"])
def test_learned_walk_equals_plain(gpu_lib, name):
    from tests.util import load_fixture
    gpu_lib.set_level_model(_model_or_skip())
    batch, _ = load_fixture(name)
    plain = gpu_lib.plan(batch, 0)
    learned = gpu_lib.plan(batch, 1)
    plain.execute()
    learned.execute()
    for x, y in zip(plain.outputs(), learned.outputs()):
        assert np.array_equal(x, y)
    st = learned.learned_stats()
    assert st["fallbacks"] >= 0
    plain.close()
    learned.close()


@pytest.mark.gpu
def test_trained_model_gain(gpu_lib):
    """On tasks outside the training set, the committed model predicts the stop level
    better than the model-free guess (the most frequent level of its training data)."""
    p = _model_or_skip()
    _, meta = level_model.load()
    S = synthetic.config1(seed=123)
    X, y = level_model.samples(gpu_lib, [S], per_system=20000, seed=9)
    pred = gpu_lib.mlp_predict(p, X).astype(int)
    maj = meta["majority_level"]
    mae_model = np.mean(np.abs(pred - y))
    mae_major = np.mean(np.abs(maj - y.astype(int)))
    acc_model, acc_major = np.mean(pred == y), np.mean(y == maj)
    print(f"level model on {len(y)} unseen tasks: accuracy {acc_model:.3f} (majority {acc_major:.3f}), "
          f"mean |level error| {mae_model:.3f} (majority {mae_major:.3f})")
    assert mae_model < mae_major and acc_model > acc_major
