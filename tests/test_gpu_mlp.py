"""Learned-correction MLP: tensor-core forward pass and FP32 training
gradients against an FP64 CPU restatement (oracle/mlp_oracle.py), and Adam
training on a fixed regression task."""
import numpy as np
import pytest

import mlp_oracle as MO

pytestmark = pytest.mark.gpu


def test_param_count(sim):
    import amk
    assert amk.lib().amk_mlp_num_params() == MO.NUM_PARAMS


def test_tensor_core_forward_matches_fp64(sim):
    p = MO.init_params(3)
    sim.set_mlp_params(p)
    assert np.array_equal(sim.mlp_params(), p)
    rng = np.random.default_rng(4)
    for n in (1, 127, 128, 129, 1000, 5000):
        x = rng.normal(0, 1, (n, MO.IN)).astype(np.float32)
        y = sim.mlp_forward(x)
        ref = MO.forward(p, x, act_bf16=True)   # BF16 operands, FP32 accumulation
        scale = np.max(np.abs(ref)) + 1e-30
        assert np.max(np.abs(y - ref)) < 2e-2 * scale, n
        ref32 = MO.forward(p, x)
        assert np.max(np.abs(y - ref32)) < 5e-2 * scale, n


def test_gradients_match_fp64(sim):
    p = MO.init_params(5)
    sim.set_mlp_params(p)
    rng = np.random.default_rng(6)
    x = rng.normal(0, 1, (300, MO.IN)).astype(np.float32)
    t = rng.normal(0, 1, (300, 3)).astype(np.float32)
    loss, g, yhat = sim.mlp_gradients(x, t)
    rloss, rg = MO.gradients(p, x, t)
    assert abs(loss - rloss) <= 1e-5 * abs(rloss)
    assert np.max(np.abs(yhat - MO.forward(p, x))) < 1e-4 * (np.max(np.abs(yhat)) + 1e-30)
    for name, off, size in _blocks():
        a, b = g[off:off + size], rg[off:off + size]
        assert np.max(np.abs(a - b)) <= 1e-4 * (np.max(np.abs(b)) + 1e-30), name


def _blocks():
    off = 0
    for name, shape in MO.SHAPES:
        size = int(np.prod(shape))
        yield name, off, size
        off += size


def test_adam_training_fits_a_smooth_map(sim):
    rng = np.random.default_rng(7)
    x = rng.uniform(-1, 1, (8192, MO.IN)).astype(np.float32)
    t = np.stack([np.sin(2 * x[:, 0]) * x[:, 1], x[:, 2] ** 2 - x[:, 3], np.tanh(x[:, 4] + x[:, 5])], 1)
    t = t.astype(np.float32)
    sim.set_mlp_params(MO.init_params(8))
    l0, _, _ = sim.mlp_gradients(x, t)
    l1 = sim.mlp_train(x, t, steps=600, batch=1024, lr=2e-3)
    assert l1 < 0.1 * l0, (l0, l1)
    # the trained network on the tensor cores agrees with its FP32 evaluation
    p = sim.mlp_params()
    y = sim.mlp_forward(x[:2048])
    assert np.max(np.abs(y - MO.forward(p, x[:2048], act_bf16=True))) < 2e-2 * np.max(np.abs(t))
