"""The FP64 learned-bound oracle against central differences of its own
loss (pins the oracle the GPU training kernels are checked against), and
its BF16-rounding mode against the plain one."""

import numpy as np

from oracle import mlp_oracle as O


def _params(rng):
    s = 0.2
    return {"W1": rng.normal(0, s, (64, 128)), "W2": rng.normal(0, s, (128, 128)), "W3": rng.normal(0, s, (128, 128)),
            "b1": rng.normal(0, 0.05, 128), "b2": rng.normal(0, 0.05, 128), "b3": rng.normal(0, 0.05, 128),
            "w4": rng.normal(0, s, 128), "b4": np.array([0.1])}


def test_gradients_match_central_differences():
    rng = np.random.default_rng(0)
    P = _params(rng)
    x = rng.uniform(-1.5, 1.5, (24, 3))
    t = rng.uniform(0, 0.5, 24)
    norm = [0.0, 0.0, 0.0, 1 / 1.5]
    freq = rng.normal(0, 1, (32, 3))
    _, _, G = O.forward_backward(x, t, P, norm, freq)
    h = 1e-6
    for name in ("W1", "W2", "W3", "b1", "b2", "b3", "w4", "b4"):
        flat = P[name].reshape(-1)
        for j in rng.choice(flat.size, size=min(6, flat.size), replace=False):
            old = flat[j]
            flat[j] = old + h
            lp = O.forward_backward(x, t, P, norm, freq)[1]
            flat[j] = old - h
            lm = O.forward_backward(x, t, P, norm, freq)[1]
            flat[j] = old
            fd = (lp - lm) / (2 * h)
            g = G[name].reshape(-1)[j]
            assert abs(fd - g) <= 1e-6 + 1e-5 * abs(g), (name, j, fd, g)


def test_bf16_rounding_mode_stays_close_to_fp64():
    rng = np.random.default_rng(1)
    P = _params(rng)
    x = rng.uniform(-1.5, 1.5, (256, 3))
    t = rng.uniform(0, 0.5, 256)
    norm = [0.0, 0.0, 0.0, 1 / 1.5]
    freq = rng.normal(0, 1, (32, 3))

    def bf16(a):
        # round to nearest even on the upper 16 bits of the FP32 pattern
        u = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
        u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
        return u.astype(np.uint32).view(np.float32).astype(np.float64)

    y0, l0, G0 = O.forward_backward(x, t, P, norm, freq)
    y1, l1, G1 = O.forward_backward(x, t, P, norm, freq, act_round=bf16)
    assert np.abs(y1 - y0).max() <= 0.02 * np.abs(y0).max()
    for name in G0:
        assert np.abs(G1[name] - G0[name]).max() <= 0.05 * (np.abs(G0[name]).max() + 1e-12), name
    # the rounding is real: the two modes differ
    assert not np.array_equal(y0, y1)
