"""Learned bound: training-kernel gradients vs the FP64 CPU oracle,
inference kernel vs training forward, conservativeness, and the gain of the
trained network over the traversal without it (results identical)."""

import math

import numpy as np
import pytest
import torch

from atom3d_b200 import MeshBVH, synthetic
from atom3d_b200.learned import LearnedBound, train_for_mesh

pytestmark = pytest.mark.gpu


def bf16_round(a):
    return torch.from_numpy(np.asarray(a, np.float32)).bfloat16().float().numpy().astype(np.float64)


def test_training_gradients_match_fp64_oracle():
    from oracle import mlp_oracle as O

    lb = LearnedBound([-1.5] * 3, [1.5] * 3, seed=3)
    g = torch.Generator().manual_seed(0)
    x = (torch.rand(512, 3, generator=g) * 3 - 1.5).cuda()
    t = (torch.rand(512, generator=g) * 0.5).cuda()
    y, loss = lb.forward_backward(x, t)
    torch.cuda.synchronize()
    P = {k: bf16_round(v.detach().cpu().numpy()) if k in ("W1", "W2", "W3") else v.detach().cpu().double().numpy()
         for k, v in lb.views.items()}
    xs, ts, fq = x.cpu().numpy(), t.cpu().numpy(), lb.freq.cpu().numpy()
    # the oracle with the kernels' BF16 roundings (features, activations,
    # activation gradients): only FP32 summation order and the odd rounding
    # flip differ, so the bounds are tight
    yr, lr_, G = O.forward_backward(xs, ts, P, lb.norm, fq, act_round=bf16_round)
    err = {"y": np.abs(y.cpu().numpy() - yr).max() / max(1.0, np.abs(yr).max()),
           "loss": abs(float(loss) - lr_) / (lr_ + 1e-6)}
    assert err["y"] <= 1e-2 and err["loss"] <= 1e-3, err
    # and the plain FP64 model, with the BF16 error budget
    y64, l64, G64 = O.forward_backward(xs, ts, P, lb.norm, fq)
    assert np.abs(y.cpu().numpy() - y64).max() <= 0.03 * max(1.0, np.abs(y64).max())
    off = 0
    for name in ("W1", "W2", "W3", "b1", "b2", "b3", "w4", "b4"):
        gg = lb.grads[off:off + G[name].size].view(G[name].shape).cpu().double().numpy()
        off += G[name].size
        scale = np.abs(G[name]).max() + 1e-12
        err[name] = np.abs(gg - G[name]).max() / scale
        assert err[name] <= 3e-3, (name, err)
        assert np.abs(gg - G64[name]).max() <= 0.06 * (np.abs(G64[name]).max() + 1e-12), name
    print("relative errors against the BF16-rounding oracle:", {k: float(f"{v:.2e}") for k, v in err.items()})


def test_inference_kernel_matches_training_forward():
    lb = LearnedBound([-1.5] * 3, [1.5] * 3, seed=5)
    x = (torch.rand(10000, 3, generator=torch.Generator().manual_seed(1)) * 3 - 1.5).cuda()
    y = lb.predict(x)
    b = lb(x)
    assert lb.status() == 0
    assert torch.allclose(b, torch.clamp(y, min=0), atol=2e-3, rtol=2e-2)


@pytest.mark.parametrize("n,log_space", [(1, False), (127, False), (128, True), (129, False), (4096 + 77, True),
                                         (600_000, False)])
def test_tensor_core_inference_matches_training_kernels(n, log_space):
    """The tcgen05 inference kernel (tensor-memory accumulators, swizzled
    shared-memory operands) against the training path's mma.sync GEMMs on the
    same BF16 weights and features: the same roundings, so only the FP32
    summation order differs; ragged tails, many tiles per warpgroup, both
    output spaces."""
    lb = LearnedBound([-1.5] * 3, [1.5] * 3, seed=7, log_space=log_space)
    g = torch.Generator().manual_seed(3)
    xt = (torch.rand(8192, 3, generator=g) * 3 - 1.5).cuda()
    lb.fit(xt, xt.norm(dim=1) * 0.5, epochs=2, batch=1024)  # a trained spread of weights
    x = (torch.rand(n, 3, generator=g) * 3 - 1.5).cuda()
    y = lb.predict(x)
    y = torch.exp(y) if log_space else torch.clamp(y, min=0)
    b = lb(x)
    assert lb.status() == 0
    d = (b - y).abs()
    scale = float(y.abs().max()) + 1e-6
    assert float(d.max()) <= 2e-2 * scale, float(d.max())
    assert float(d.median()) <= 1e-3 * scale, float(d.median())
    # every query written (no tile skipped), deterministically
    out = torch.full((n,), float("nan"), device="cuda")
    lb(x, out=out)
    assert torch.equal(out, b)


def test_trained_bound_against_the_plain_method():
    """The learned bound judged against the plain method the bench times (the
    neighbour seed on): results identical in every mode; node + triangle
    tests per query and time of the learned cap beside plain, and beside an
    exact bound (a perfect network: the ceiling of any bound-seeded radius).
    The learned cap must not add more than 10% tests per query (a bound that
    excludes every triangle restarts the query in the traversal kernel);
    the times are reported, not asserted."""
    from atom3d_b200 import _lib

    v, f = synthetic.displaced_sphere(5, 16, 0.05, 3)
    mesh = MeshBVH(v.cuda(), f.cuda())
    g = torch.Generator().manual_seed(2)
    train = synthetic.mixed_queries(v, f, 1 << 18, g)
    lb = train_for_mesh(mesh, train, epochs=12)
    q = synthetic.mixed_queries(v, f, 1 << 20, g).cuda()
    b = lb(q)
    ref = mesh._bvh.query(q)
    cover = (ref[0] <= b).float().mean().item()
    assert cover > 0.95
    exact = torch.nextafter(ref[0], torch.full_like(ref[0], float("inf"))) * (1 + 1e-6)
    modes = {
        "plain": (None, 0),
        "learned_cap": (b, 0),
        "learned_seeds": (b, _lib.A3D_UDF_NO_REUSE | _lib.A3D_UDF_BOUND_SEEDS),
        "exact_cap": (exact, 0),
        "plain_without_neighbour_seed": (None, _lib.A3D_UDF_NO_REUSE),
    }
    tests, ms = {}, {}
    for name, (bound, flags) in modes.items():
        st = torch.zeros(4, dtype=torch.int64, device="cuda")
        r = mesh._bvh.query(q, bound=bound, stats=st, seeding=flags)
        for a, c in zip(ref, r):
            assert torch.equal(a, c), name  # identical distances, ids, points, uvw
        tests[name] = (int(st[0]) + int(st[1])) / q.shape[0]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            mesh._bvh.query(q, bound=bound, seeding=flags)
        e1.record()
        torch.cuda.synchronize()
        ms[name] = e0.elapsed_time(e1) / 3
    print("tests per query:", {k: round(x, 1) for k, x in tests.items()})
    print("ms per call:", {k: round(x, 3) for k, x in ms.items()})
    assert tests["exact_cap"] <= tests["plain"]
    assert tests["learned_cap"] <= 1.10 * tests["plain"]
    assert tests["learned_seeds"] < tests["plain_without_neighbour_seed"]
