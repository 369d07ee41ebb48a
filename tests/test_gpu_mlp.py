"""The warm-start network's tensor-core kernels against an FP32 reference of
the same operation (torch on the same bf16 inputs)."""
from __future__ import annotations

import pytest

torch = pytest.importorskip("torch")

from bowshock_b200 import _native  # noqa: E402

pytestmark = pytest.mark.gpu


def _gemm(a, b, c, splits=1, accumulate=False):
    lib = _native.load()
    m, k = a.shape
    n = b.shape[0]
    _native.check(lib.bs_gemm_bf16(a.data_ptr(), b.data_ptr(), c.data_ptr(), m, n, k, splits,
                                   1 if accumulate else 0, torch.cuda.current_stream().cuda_stream), lib)


@pytest.mark.parametrize("m,n,k", [(128, 64, 64), (256, 256, 128), (200, 128, 256), (384, 256, 512),
                                   (1000, 256, 256)])
def test_gemm_matches_fp32_reference(m, n, k):
    g = torch.Generator(device="cuda").manual_seed(m * 7 + n * 3 + k)
    a = torch.randn(m, k, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(n, k, device="cuda", generator=g).to(torch.bfloat16)
    c = torch.full((m, n), float("nan"), device="cuda")
    _gemm(a, b, c)
    ref = a.double() @ b.double().T
    err = (c.double() - ref).abs().max().item()
    # Exact bf16 products, FP32 sums in a different order: ~1e-6 of sqrt(k).
    assert err <= 1e-4 * k ** 0.5, err


def test_split_k_accumulates():
    g = torch.Generator(device="cuda").manual_seed(5)
    m, n, k = 256, 256, 1024
    a = torch.randn(m, k, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(n, k, device="cuda", generator=g).to(torch.bfloat16)
    c = torch.ones(m, n, device="cuda")
    _gemm(a, b, c, splits=4, accumulate=True)
    ref = 1.0 + a.double() @ b.double().T
    assert (c.double() - ref).abs().max().item() <= 1e-4 * k ** 0.5


# ---- the warm-start network ------------------------------------------------------

import math  # noqa: E402

import numpy as np  # noqa: E402

from bowshock_b200.mlp import WarmStartNet  # noqa: E402


def _bf16(t):
    return t.to(torch.bfloat16).to(t.dtype)


def _ste(t):
    """bf16 rounding in the forward pass, identity in the backward pass."""
    return t + (_bf16(t) - t).detach()


def _features(s):
    x = s[:, 0] * 0.125
    r = s[:, 1] * 0.25
    cols = [x, r] + [s[:, 2 + k] for k in range(8)]
    for k in range(16):
        w = math.pi * 2.0 ** (7 * k / 15)
        cols += [torch.sin(w * x), torch.cos(w * x), torch.sin(w * r), torch.cos(w * r)]
    f = torch.stack(cols, 1)
    f = torch.cat([f, torch.zeros(len(s), 128 - f.shape[1], dtype=f.dtype, device=f.device)], 1)
    return _bf16(f.float()).double()


def _reference(net, params, samples, targets):
    """Loss, gradients and outputs of the same network in float64, rounding
    to bf16 where the kernels store bf16 (weights, features, activations)."""
    s = torch.tensor(samples, dtype=torch.float64, device="cuda")
    t = torch.tensor(targets, dtype=torch.float64, device="cuda")
    p = torch.tensor(params, dtype=torch.float64, device="cuda")
    tensors, k = [], 0
    for out, inp in net.layer_shapes():
        w = p[k:k + out * inp].reshape(out, inp).clone().requires_grad_(True)
        k += out * inp
        b = p[k:k + out].clone().requires_grad_(True)
        k += out
        tensors.append((w, b))
    h = _features(s)
    for li, (w, b) in enumerate(tensors):
        z = h @ _ste(w).T + b
        if li < len(tensors) - 1:
            h = _ste(torch.nn.functional.gelu(z))
        else:
            y = z
    loss = ((y[:, :4] - t) ** 2).mean()
    loss.backward()
    grads = torch.cat([torch.cat([w.grad.ravel(), b.grad]) for w, b in tensors]).cpu().numpy()
    return loss.item(), grads, y[:, :4].detach().cpu().numpy()


def _samples(n, seed):
    rng = np.random.default_rng(seed)
    s = np.zeros((n, 10), np.float32)
    s[:, 0] = rng.uniform(-1.0, 8.0, n)
    s[:, 1] = rng.uniform(0.0, 3.0, n)
    s[np.arange(n), 2 + rng.integers(0, 5, n)] = 1.0
    s[:, 7:10] = rng.uniform(0.2, 1.0, (n, 3))
    t = np.stack([0.5 * np.sin(1.3 * s[:, 0]) + 0.3 * s[:, 1], np.cos(0.7 * s[:, 1]) * s[:, 9],
                  0.2 * s[:, 0] * s[:, 8], np.log1p(s[:, 1]) + s[:, 7]], 1).astype(np.float32)
    return s, t


def _layer_errors(net, g, ref):
    errs, k = [], 0
    for out, inp in net.layer_shapes():
        n = out * inp + out
        errs.append(np.linalg.norm(g[k:k + n] - ref[k:k + n]) / np.linalg.norm(ref[k:k + n]))
        k += n
    return errs


@pytest.mark.parametrize("hidden_layers", [3, 5])  # 5: the warm start's own network
def test_network_gradients_match_float64_reference(hidden_layers):
    net = WarmStartNet(hidden_layers=hidden_layers, batch=256, seed=3)
    samples, targets = _samples(200, 1)
    params = net.params()
    loss, grads = net.loss_grad(samples, targets)
    ref_loss, ref_grads, _ = _reference(net, params, samples, targets)
    assert abs(loss - ref_loss) <= 1e-2 * ref_loss
    # bf16 rounding of the output and hidden gradients: a few 1e-3 per layer.
    assert max(_layer_errors(net, grads, ref_grads)) < 2e-2
    net.destroy()


def test_network_predictions_match_reference_and_training_lowers_the_loss():
    net = WarmStartNet(hidden_layers=3, batch=1024, seed=5)
    samples, targets = _samples(20000, 2)
    pred = net.predict(samples[:3000])
    _, _, ref = _reference(net, net.params(), samples[:3000], targets[:3000])
    assert np.abs(pred - ref).max() <= 1e-2 * max(1.0, np.abs(ref).max())
    net.set_data(samples, targets)
    losses = net.train(400, 2e-3, seed=7)
    assert np.all(np.isfinite(losses))
    assert losses[-20:].mean() < 0.1 * losses[:5].mean()
    net.destroy()
