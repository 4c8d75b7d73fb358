"""Training convolutions of the closure network on the tensor cores (forward, data and weight
gradients as tcgen05 GEMMs over bf16 im2col operands, FP32 accumulation) against the FP32 SIMT
path and the FP64 oracle: the forward output, the loss and every parameter gradient agree to the
bf16 rounding of the operands, the gradients are deterministic, and Adam training converges."""
import numpy as np
import pytest

from oracle import cnn_oracle as CO

pytestmark = pytest.mark.gpu


def P():
    import optimizec_b200 as mod

    return mod


def per_layer_errors(g, g_ref, layers, ch):
    """Relative L2 error of each layer's gradient (weights and bias together: a bias gradient
    alone is a sum over every pixel whose cancellation makes its relative error meaningless)."""
    out, off = [], 0
    for ci, co in CO.layer_shapes(layers, ch):
        n = co * ci * 9 + co
        a, r = g[off:off + n], g_ref[off:off + n]
        out.append(float(np.linalg.norm(a - r) / (np.linalg.norm(r) + 1e-30)))
        off += n
    return out


@pytest.mark.parametrize("layers,ch,H,W,B", [
    (6, 32, 48, 48, 4),   # the closure's N = 32 training images
    (6, 32, 12, 20, 1),   # 240 pixels: the last 128-pixel tile is partly padding
    (4, 8, 16, 16, 2),    # 8 channels: 72-row weight gradient, 5 K steps
])
def test_tensor_core_training_matches_fp32(layers, ch, H, W, B):
    rng = np.random.default_rng(layers * 7 + H)
    net = P().CNN(layers, ch, seed=11)
    x = rng.standard_normal((B, 3, H, W)).astype(np.float32)
    t = rng.standard_normal((B, 1, H, W)).astype(np.float32)
    y32 = net.forward(x)
    l32, g32 = net.loss_grad(x, t)
    net.set_train_tc(True)
    ytc = net.forward(x)
    ltc, gtc = net.loss_grad(x, t)
    # bf16 operands, FP32 accumulation: the forward within 1 %, the loss within 2 %
    assert np.linalg.norm(ytc - y32) <= 1e-2 * np.linalg.norm(y32)
    assert ltc == pytest.approx(l32, rel=2e-2)
    errs = per_layer_errors(gtc, g32, layers, ch)
    assert max(errs) <= 5e-2, errs
    assert np.linalg.norm(gtc - g32) <= 2e-2 * np.linalg.norm(g32)
    # fixed partition and fixed-order sums: the same bits call after call
    _, gtc2 = net.loss_grad(x, t)
    np.testing.assert_array_equal(gtc2, gtc)
    net.close()


def test_tensor_core_gradients_match_oracle():
    """FP64 oracle at 24 x 24 (B = 2): every layer's gradient within the bf16 tolerance."""
    layers, ch, H, W, B = 6, 32, 24, 24, 2
    rng = np.random.default_rng(5)
    net = P().CNN(layers, ch, seed=7)
    p = net.params()
    x = rng.standard_normal((B, 3, H, W)).astype(np.float32)
    t = rng.standard_normal((B, 1, H, W)).astype(np.float32)
    net.set_train_tc(True)
    loss, g = net.loss_grad(x, t)
    loss_ref, g_ref = CO.loss_grad(p.astype(np.float64), layers, ch, x, t)
    assert loss == pytest.approx(loss_ref, rel=2e-2)
    errs = per_layer_errors(g, g_ref, layers, ch)
    assert max(errs) <= 5e-2, errs
    net.close()


def test_tensor_core_adam_training_fits_a_local_map():
    """The FP32 path's convergence test with the convolutions on the tensor cores."""
    rng = np.random.default_rng(3)
    H = W = 32
    x = rng.standard_normal((64, 3, H, W)).astype(np.float32)
    wt = rng.standard_normal((1, 3, 3, 3)) * 0.3
    t = CO.conv3x3(x.astype(np.float64), wt, np.zeros(1)).astype(np.float32)
    net = P().CNN(4, 16, seed=1)
    net.set_train_tc(True)
    net.set_dataset(x, t)
    losses = net.train(300, 16, 2e-3, seed=5)
    assert losses[-20:].mean() < losses[:5].mean() / 20, (losses[:5].mean(), losses[-20:].mean())
    net.close()


def test_tensor_core_training_rejects_wide_networks():
    net = P().CNN(3, 48, seed=1)
    with pytest.raises(P().Dns2dError):
        net.set_train_tc(True)
    net.close()
