"""Warm-start network kernels (csrc/cnn.cu) against the FP64 CPU oracle.

The device keeps the features, the weights it multiplies and the hidden
activations in BF16 and accumulates in FP32; the oracle forward applies the
same BF16 roundings in FP64, so the forward output must agree to FP32
accumulation error (1e-3 relative).  The backward pass also rounds the
propagated gradients to BF16 where they enter a tensor-core convolution, so
gradients are compared by relative L2 (2e-2) and direction (cosine > 0.999).
"""

import numpy as np
import pytest

from gpu_util import need_gpu, rel_l2

torch = pytest.importorskip("torch")

from oracle import cnn_oracle as C  # noqa: E402

GRID = (32, 48)


def _flat_to_dict(p):
    from fbme_b200.learned import HIDDEN

    h = HIDDEN
    o, d = 0, {}
    for name, shape in (("W1", (3, 3, 2, h)), ("b1", (h,)), ("W2", (3, 3, h, h)), ("b2", (h,)),
                        ("W3", (3, 3, h, 1)), ("b3", (1,))):
        n = int(np.prod(shape))
        d[name] = p[o:o + n].astype(np.float64).reshape(shape)
        o += n
    return d


def _rounded_forward(params, x):
    """Oracle forward with the device's BF16 roundings."""
    q = {k: (C.bf16_round(v) if k.startswith("W") else v) for k, v in params.items()}
    xb = C.bf16_round(x)
    h1 = C.bf16_round(np.maximum(C.conv3x3(xb, q["W1"], q["b1"]), 0.0))
    h2 = C.bf16_round(np.maximum(C.conv3x3(h1, q["W2"], q["b2"]), 0.0))
    return C.conv3x3(h2, q["W3"], q["b3"])[..., 0], q, xb


def _net(seed=3):
    from fbme_b200.learned import WarmStartNet, init_params

    p = init_params(seed)
    p[-1] = 0.3  # nonzero output bias
    return WarmStartNet(torch.device("cuda", 0), p), p


def _bp(b, seed=0):
    rng = np.random.default_rng(seed)
    n = GRID[0] * GRID[1]
    amp = rng.normal(size=(b, n)) + 1j * rng.normal(size=(b, n))
    amp[:, rng.choice(n, 20, replace=False)] *= 30.0  # a few bright scatterers
    return amp.astype(np.complex64)


@pytest.mark.gpu
def test_cnn_forward_matches_oracle():
    need_gpu()
    net, p = _net()
    bp = _bp(2)
    out = net.predict(torch.from_numpy(bp).cuda(), *GRID).cpu().numpy().reshape(2, *GRID)
    x = C.features(bp, GRID)
    ref, _, _ = _rounded_forward(_flat_to_dict(p), x)
    assert rel_l2(out, ref) < 1e-3
    # the features themselves: f1 is the mean of f0
    assert np.allclose(x[..., 1], x[..., 0].mean(axis=(1, 2), keepdims=True))


@pytest.mark.gpu
def test_cnn_gradients_match_oracle():
    need_gpu()
    net, p = _net(5)
    bp = _bp(2, 1)
    rng = np.random.default_rng(2)
    target = rng.normal(size=(2, *GRID)).astype(np.float32)
    net.features(torch.from_numpy(bp).cuda(), *GRID)
    net.forward(2, *GRID)
    loss = float(net.backward(torch.from_numpy(target.reshape(2, -1)).cuda(), 2, *GRID))
    g = net.grad.cpu().numpy()
    params = _flat_to_dict(p)
    x = C.features(bp, GRID)
    _, q, xb = _rounded_forward(params, x)
    ref_loss, _, ref = C.loss_and_grads(q, xb, target.astype(np.float64))
    assert abs(loss - ref_loss) / ref_loss < 1e-3
    gd = _flat_to_dict(g)
    for k in ("W1", "b1", "W2", "b2", "W3", "b3"):
        a, b = gd[k].ravel(), ref[k].ravel()
        cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))
        assert rel_l2(a, b) < 2e-2, k
        assert cos > 0.999, k


@pytest.mark.gpu
def test_cnn_adam_reduces_loss_on_a_batch():
    need_gpu()
    net, _ = _net(7)
    bp = torch.from_numpy(_bp(4, 9)).cuda()
    x = C.features(_bp(4, 9), GRID)[..., 0]
    target = torch.from_numpy((0.5 * x - 1.0).reshape(4, -1).astype(np.float32)).cuda()
    losses = []
    for _ in range(60):
        net.features(bp, *GRID)
        net.forward(4, *GRID)
        losses.append(float(net.backward(target, 4, *GRID)))
        net.adam(3e-3)
    assert losses[-1] < 0.2 * losses[0]
