"""CPU oracle of the learned auxiliary-field proposal: test infrastructure, not product code.

The proposal has no counterpart in the reference (MPSQMC2.cpp:551-588 samples the exact grid
PDF).  This file restates, in numpy and FP64, what the engine's proposal kernels compute, so the
tests can check the device forward pass, loss and gradients against it:

  features f (32) -> h1 = relu(f W1 + b1) (128) -> h2 = relu(h1 W2 + b2) (128) -> z = h2 W3 + b3 (G)
  q = softmax(z);  loss = mean over the batch of KL(p || q) = sum_x p (log p - log q)

Parameters are one flat vector in the engine's order and layout: W1 (32 x 128, input-major,
W1[i * 128 + o]), b1 (128), W2 (128 x 128), b2, W3 (128 x G), b3 (G).
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID = 32, 128


def n_params(G: int) -> int:
    return N_IN * N_HID + N_HID + N_HID * N_HID + N_HID + N_HID * G + G


def unpack(theta: np.ndarray, G: int):
    o = 0
    out = []
    for shape in ((N_IN, N_HID), (N_HID,), (N_HID, N_HID), (N_HID,), (N_HID, G), (G,)):
        n = int(np.prod(shape))
        out.append(np.asarray(theta[o:o + n], dtype=np.float64).reshape(shape))
        o += n
    return out


def forward(theta: np.ndarray, X: np.ndarray, G: int):
    W1, b1, W2, b2, W3, b3 = unpack(theta, G)
    h1 = np.maximum(X @ W1 + b1, 0.0)
    h2 = np.maximum(h1 @ W2 + b2, 0.0)
    z = h2 @ W3 + b3
    return h1, h2, z


def softmax(z: np.ndarray) -> np.ndarray:
    e = np.exp(z - z.max(axis=-1, keepdims=True))
    return e / e.sum(axis=-1, keepdims=True)


def loss_grad(theta: np.ndarray, X: np.ndarray, P: np.ndarray, G: int):
    """Mean KL(p || q) over the batch and its gradient with respect to theta."""
    W1, b1, W2, b2, W3, b3 = unpack(theta, G)
    X = np.asarray(X, np.float64)
    P = np.asarray(P, np.float64)
    B = X.shape[0]
    h1, h2, z = forward(theta, X, G)
    q = softmax(z)
    with np.errstate(divide="ignore", invalid="ignore"):
        plogp = np.where(P > 0, P * np.log(np.where(P > 0, P, 1.0)), 0.0)
    logq = z - z.max(axis=1, keepdims=True)
    logq = logq - np.log(np.exp(logq).sum(axis=1, keepdims=True))
    loss = float(np.sum(plogp - P * logq) / B)
    dz = (q - P) / B
    gW3 = h2.T @ dz
    gb3 = dz.sum(0)
    dh2 = (dz @ W3.T) * (h2 > 0)
    gW2 = h1.T @ dh2
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ W2.T) * (h1 > 0)
    gW1 = X.T @ dh1
    gb1 = dh1.sum(0)
    grad = np.concatenate([g.ravel() for g in (gW1, gb1, gW2, gb2, gW3, gb3)])
    return loss, grad


def init_params(G: int, seed: int) -> np.ndarray:
    """He-uniform weights, zero biases (the engine's initialisation with the same seed is its
    own; tests pass parameters explicitly)."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_in, fan_out in ((N_IN, N_HID), (N_HID, N_HID), (N_HID, G)):
        lim = np.sqrt(6.0 / fan_in)
        parts.append(rng.uniform(-lim, lim, size=(fan_in, fan_out)).ravel())
        parts.append(np.zeros(fan_out))
    return np.concatenate(parts)


def features(C: np.ndarray, M: np.ndarray, ov: float) -> np.ndarray:
    """The proposal's 32 inputs for one coupling: 4 C_kl / ov (the coefficients of the overlap
    ratio rho(x) = sum_kl f_kl x_k x_l) and 4 M / ov (the 16 closures of the left and right
    environment branches), both in the engine's index order."""
    return np.concatenate([4.0 * np.asarray(C).ravel() / ov, 4.0 * np.asarray(M).ravel() / ov])
