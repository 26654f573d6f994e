"""TEST INFRASTRUCTURE ONLY: a float64 NumPy restatement of the amortised encoder's training step,
the checker of the CUDA kernels in gaspacho2_b200/csrc/k_mlp.cu. The reference has no encoder (it
places every cell by L-BFGS, ggplvm.cu:1214-1301); the network is this project's own, so this
oracle restates the project's specification, not reference code.

The network: 2-hidden-layer MLP n_in -> H -> H -> 2Q with GELU (exact, erf form), output = mean
(first Q) and log-variance (last Q) of the latent coordinates. Loss per cell
    0.5 * sum_q [ logvar_q + (x_q - mean_q)^2 exp(-logvar_q) ],
averaged over the batch (the Gaussian negative log-likelihood up to a constant).

Mixed precision exactly as the kernels: every matrix-multiply input (features, weights, hidden
activations, back-propagated output and pre-activation gradients) is rounded to BF16 (round to
nearest even); products are accumulated at high precision (float64 here, FP32 on the GPU); the
biases, the GELU and its derivative, the loss and the bias gradients work on the unrounded values.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf


def bf16(a) -> np.ndarray:
    """Rounds to the nearest BF16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(a, np.float64).astype(np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def forward(params, F):
    """params: dict W1 (H x n_in), b1, W2 (H x H), b2, W3 (2Q x H), b3; F: B x n_in features.
    Returns (out B x 2Q, cache)."""
    Fq = bf16(F)
    a1 = Fq @ bf16(params["W1"]).T + params["b1"]
    h1 = bf16(gelu(a1))
    a2 = h1 @ bf16(params["W2"]).T + params["b2"]
    h2 = bf16(gelu(a2))
    out = h2 @ bf16(params["W3"]).T + params["b3"]
    return out, dict(Fq=Fq, a1=a1, h1=h1, a2=a2, h2=h2)


def loss_and_dout(out, X):
    """Mean Gaussian NLL over the batch and its gradient with respect to the outputs."""
    B, Q2 = out.shape
    Q = Q2 // 2
    mu, lv = out[:, :Q], out[:, Q:]
    r = X - mu
    e = np.exp(-lv)
    loss = 0.5 * np.sum(lv + r * r * e) / B
    dout = np.concatenate([-r * e, 0.5 * (1.0 - r * r * e)], axis=1) / B
    return loss, dout


def backward(params, cache, dout):
    """Gradients of every parameter (float64)."""
    dq = bf16(dout)
    g = {"W3": dq.T @ cache["h2"], "b3": dout.sum(0)}
    dh2 = dq @ bf16(params["W3"])
    da2 = dh2 * gelu_grad(cache["a2"])
    da2q = bf16(da2)
    g["W2"] = da2q.T @ cache["h1"]
    g["b2"] = da2.sum(0)
    dh1 = da2q @ bf16(params["W2"])
    da1 = dh1 * gelu_grad(cache["a1"])
    da1q = bf16(da1)
    g["W1"] = da1q.T @ cache["Fq"]
    g["b1"] = da1.sum(0)
    return g


def loss_and_grads(params, F, X):
    out, cache = forward(params, F)
    loss, dout = loss_and_dout(out, X)
    return loss, backward(params, cache, dout), out


def init_params(n_in: int, H: int, Q: int, seed: int = 0) -> dict:
    """Seeded initialisation as the kernels' host side draws it: weights N(0, 1/fan_in) (FP32),
    biases zero."""
    rng = np.random.default_rng(seed)
    return {
        "W1": (rng.standard_normal((H, n_in)) / np.sqrt(n_in)).astype(np.float32).astype(np.float64),
        "b1": np.zeros(H),
        "W2": (rng.standard_normal((H, H)) / np.sqrt(H)).astype(np.float32).astype(np.float64),
        "b2": np.zeros(H),
        "W3": (rng.standard_normal((2 * Q, H)) / np.sqrt(H)).astype(np.float32).astype(np.float64),
        "b3": np.zeros(2 * Q),
    }
