"""BF16 tensor-core (tcgen05) forward of the closure network against the FP64 restatement with
the same bf16 roundings (inputs, weights and every hidden activation rounded to bf16, round to
nearest even; exact erf GELU), and against the FP32 network.  Every layer runs as an implicit
GEMM on the tensor cores with FP32 accumulation and the tanh form of GELU."""
import numpy as np
import pytest

from oracle import cnn_oracle as CO

pytestmark = pytest.mark.gpu


def P():
    import optimizec_b200 as mod

    return mod


def bf16(a):
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward_bf16(params, layers, x):
    ps = CO.unpack(params, layers, 32)
    a = bf16(x)
    for l, (w, b) in enumerate(ps):
        w = bf16(w)
        z = CO.conv3x3(a, w, b)
        a = bf16(CO.gelu(z)) if l < layers - 1 else z
    return a


@pytest.mark.parametrize("B,H,W,layers", [(1, 16, 128, 4), (2, 8, 256, 6), (1, 384, 384, 6)])
def test_tensor_core_forward_matches_bf16_oracle(B, H, W, layers):
    rng = np.random.default_rng(3)
    net = P().CNN(layers, 32, seed=5)
    x = rng.standard_normal((B, 3, H, W)).astype(np.float32)
    y_tc = net.forward_tc(x).astype(np.float64)
    y_32 = net.forward(x).astype(np.float64)
    y_bf = forward_bf16(net.params(), layers, x)
    nrm = np.linalg.norm(y_bf)
    assert np.linalg.norm(y_tc - y_bf) <= 5e-3 * nrm, np.linalg.norm(y_tc - y_bf) / nrm
    # bf16 weights/activations against the FP32 network: within the bf16 rounding
    assert np.linalg.norm(y_tc - y_32) <= 3e-2 * np.linalg.norm(y_32)
    # repeated call (weights already packed) gives the same bits
    np.testing.assert_array_equal(net.forward_tc(x), y_tc.astype(np.float32))
    net.close()


def test_tensor_core_path_rejects_unsupported_width():
    net = P().CNN(4, 32, seed=1)
    with pytest.raises(P().Dns2dError):
        net.forward_tc(np.zeros((1, 3, 8, 96), np.float32))
    net.close()
