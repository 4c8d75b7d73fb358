"""GPU tests of the closure network kernels against the FP64 numpy oracle: forward output,
loss and every parameter gradient, and that Adam training on the device fits a known map."""
import numpy as np
import pytest

from oracle import cnn_oracle as CO

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("layers,ch,H,W,B", [(6, 32, 24, 24, 2), (3, 8, 17, 33, 3), (6, 32, 96, 96, 1)])
def test_forward_and_gradients_match_oracle(layers, ch, H, W, B):
    import optimizec_b200 as P
    rng = np.random.default_rng(layers * 100 + H)
    net = P.CNN(layers, ch, seed=7)
    p = net.params()
    x = rng.standard_normal((B, 3, H, W)).astype(np.float32)
    t = rng.standard_normal((B, 1, H, W)).astype(np.float32)
    y = net.forward(x)
    y_ref, _ = CO.forward(p.astype(np.float64), layers, ch, x)
    assert np.linalg.norm(y - y_ref) <= 1e-5 * np.linalg.norm(y_ref)
    loss, g = net.loss_grad(x, t)
    loss_ref, g_ref = CO.loss_grad(p.astype(np.float64), layers, ch, x, t)
    assert loss == pytest.approx(loss_ref, rel=1e-5)
    # per layer: relative L2 of the weight and bias gradients (FP32 accumulation over B*H*W)
    off = 0
    for ci, co in CO.layer_shapes(layers, ch):
        for n in (co * ci * 9, co):
            a, r = g[off:off + n], g_ref[off:off + n]
            assert np.linalg.norm(a - r) <= 1e-4 * np.linalg.norm(r) + 1e-9, (ci, co, n)
            off += n
    net.close()


def test_adam_training_fits_a_local_map():
    """Target = a fixed random 3x3 periodic linear map of the inputs: the loss must fall 20x."""
    import optimizec_b200 as P
    rng = np.random.default_rng(3)
    H = W = 32
    x = rng.standard_normal((64, 3, H, W)).astype(np.float32)
    wt = rng.standard_normal((1, 3, 3, 3)) * 0.3
    t = CO.conv3x3(x.astype(np.float64), wt, np.zeros(1)).astype(np.float32)
    net = P.CNN(4, 16, seed=1)
    net.set_dataset(x, t)
    losses = net.train(300, 16, 2e-3, seed=5)
    assert losses[-20:].mean() < losses[:5].mean() / 20, (losses[:5].mean(), losses[-20:].mean())
    net.close()
