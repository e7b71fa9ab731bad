"""Tensor-core kernels of the opacity-surrogate network against the NumPy
reference (tests/mlp_ref.py): the operand layout of one tcgen05 product, the
forward pass, the gradient of one batch, and a short training run."""
import numpy as np
import pytest

import mlp_ref as R

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N", [256, 32, 64])
def test_tensor_core_product_layout(ctx, N):
    rng = np.random.default_rng(N)
    a = rng.normal(0, 1, (128, 256)).astype(np.float32)
    b = rng.normal(0, 1, (N, 256)).astype(np.float32)
    d = ctx.mlp_gemm_check(R.bf16_bits(a), R.bf16_bits(b))
    ref = R.bf16(a).astype(np.float64) @ R.bf16(b).astype(np.float64).T
    # FP32 accumulation of exact BF16 products: only summation order differs
    assert np.max(np.abs(d - ref)) < 1e-4 * np.max(np.abs(ref)), np.max(np.abs(d - ref))


# 1000 rows: one tile per CTA; 40063 rows: 313 tiles, two per CTA step,
# the last step with a second tile past the end
@pytest.mark.parametrize("n", [1000, 40063])
def test_forward_matches_reference(ctx, n):
    rng = np.random.default_rng(1)
    p = R.init(seed=2)
    x = rng.uniform(-1, 1, (n, R.IN)).astype(np.float32)
    ctx.mlp_set_params(p)
    y = ctx.mlp_forward(x)
    ref, _, _ = R.forward(p, x)
    scale = np.max(np.abs(ref))
    # same roundings; a BF16 tie flipped by a different FP32 summation order
    # moves an output by at most a few BF16 ulps of one activation
    assert np.max(np.abs(y - ref)) < 2e-2 * scale
    assert np.mean(np.abs(y - ref)) < 1e-3 * scale


@pytest.mark.parametrize("n", [2000, 40063])
def test_gradient_matches_reference(ctx, n):
    rng = np.random.default_rng(7)
    p = R.init(seed=4)
    x = rng.uniform(-1, 1, (n, R.IN)).astype(np.float32)
    t = rng.normal(0, 1, (n, R.OUT)).astype(np.float32)
    w = rng.uniform(0.5, 1.5, R.OUT).astype(np.float32)
    ctx.mlp_set_params(p)
    g, loss = ctx.mlp_gradient(x, t, w)
    gr, lr = R.gradient(p, x, t, w)
    assert abs(loss / lr - 1) < 1e-3
    blocks = dict(zip(("W0", "b0", "W123", "b123", "W4", "b4"),
                      [np.asarray(a).ravel() for a in R.unpack(g)]))
    refs = dict(zip(("W0", "b0", "W123", "b123", "W4", "b4"),
                    [np.asarray(a).ravel() for a in R.unpack(gr)]))
    for k in blocks:
        err = np.linalg.norm(blocks[k] - refs[k]) / np.linalg.norm(refs[k])
        assert err < 2e-2, (k, err)


def test_training_fits_a_smooth_function(ctx):
    rng = np.random.default_rng(11)
    x = rng.uniform(-1, 1, (65536, R.IN)).astype(np.float32)
    t = np.zeros((x.shape[0], R.OUT), np.float32)
    t[:, 0] = np.sin(2 * x[:, 0]) + x[:, 1] ** 2
    t[:, 1] = x[:, 2] * x[:, 3] - 0.5 * x[:, 4]
    t[:, 2] = np.tanh(3 * x[:, 5])
    w = np.zeros(R.OUT, np.float32)
    w[:3] = 1.0
    ctx.mlp_set_params(R.init(seed=9, scale=0.5))
    _, l0 = ctx.mlp_gradient(x[:4096], t[:4096], w)
    rep = ctx.mlp_train(x, t, w, epochs=12, batch=4096, lr=2e-3, lr_min=1e-4, seed=3)
    _, l1 = ctx.mlp_gradient(x[:4096], t[:4096], w)
    assert l1 < 0.05 * l0, (l0, l1, rep["epoch_loss"])
