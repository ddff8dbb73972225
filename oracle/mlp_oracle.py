"""numpy FP64 restatement of the learned-bound MLP (TEST INFRASTRUCTURE ONLY).

Forward and backward of x -> Fourier features (sin, cos of 2*pi*B x_hat)
-> 3 ReLU layers -> linear head with the weighted squared loss used in
training (weight under_weight where the prediction is below the target).
Used to check the GPU training kernels' gradients.  With ``act_round``
(a rounding function, BF16 in the tests) the oracle rounds the tensors the
training kernels store in BF16 between their GEMMs: the features, the three
activations and the three masked activation gradients; everything else
stays FP64.
"""

import numpy as np


def features(x, norm, freq):
    xh = (np.asarray(x, np.float64) - np.asarray(norm[:3])) * norm[3]
    t = 2 * np.pi * xh @ np.asarray(freq, np.float64).T
    f = np.empty((x.shape[0], 2 * freq.shape[0]))
    f[:, 0::2] = np.sin(t)
    f[:, 1::2] = np.cos(t)
    return f


def forward_backward(x, target, P, norm, freq, under_weight=4.0, act_round=None):
    """P: dict W1 [64,128], W2, W3 [128,128], b1, b2, b3, w4 [128], b4 [1]."""
    r = act_round if act_round is not None else (lambda a: a)
    f = r(features(x, norm, freq))
    z1 = f @ P["W1"] + P["b1"]
    h1 = r(np.maximum(z1, 0))
    z2 = h1 @ P["W2"] + P["b2"]
    h2 = r(np.maximum(z2, 0))
    z3 = h2 @ P["W3"] + P["b3"]
    h3 = r(np.maximum(z3, 0))
    y = h3 @ P["w4"] + P["b4"][0]
    n = x.shape[0]
    e = y - target
    w = np.where(e < 0, under_weight, 1.0)
    loss = float((w * e * e).sum() / n)
    dy = w * 2 * e / n
    G = {"w4": h3.T @ dy, "b4": np.array([dy.sum()])}
    dz3 = r(np.outer(dy, P["w4"]) * (h3 > 0))
    G["W3"] = h2.T @ dz3
    G["b3"] = dz3.sum(0)
    dz2 = r((dz3 @ P["W3"].T) * (h2 > 0))
    G["W2"] = h1.T @ dz2
    G["b2"] = dz2.sum(0)
    dz1 = r((dz2 @ P["W2"].T) * (h1 > 0))
    G["W1"] = f.T @ dz1
    G["b1"] = dz1.sum(0)
    return y, loss, G
