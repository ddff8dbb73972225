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
    yr, lr_, G = O.forward_backward(x.cpu().numpy(), t.cpu().numpy(), P, lb.norm, lb.freq.cpu().numpy())
    # BF16 activations on the GPU: compare with relative tolerances
    assert np.abs(y.cpu().numpy() - yr).max() <= 0.03 * max(1.0, np.abs(yr).max())
    assert abs(float(loss) - lr_) <= 0.05 * lr_ + 1e-6
    off = 0
    for name in ("W1", "W2", "W3", "b1", "b2", "b3", "w4", "b4"):
        gg = lb.grads[off:off + G[name].size].view(G[name].shape).cpu().double().numpy()
        off += G[name].size
        ref = G[name]
        scale = np.abs(ref).max() + 1e-12
        assert np.abs(gg - ref).max() <= 0.06 * scale, (name, np.abs(gg - ref).max(), scale)


def test_inference_kernel_matches_training_forward():
    lb = LearnedBound([-1.5] * 3, [1.5] * 3, seed=5)
    x = (torch.rand(10000, 3, generator=torch.Generator().manual_seed(1)) * 3 - 1.5).cuda()
    y = lb.predict(x)
    b = lb(x)
    assert torch.allclose(b, torch.clamp(y, min=0), atol=2e-3, rtol=2e-2)


def test_trained_bound_is_conservative_and_results_identical():
    from atom3d_b200 import _lib

    v, f = synthetic.displaced_sphere(5, 16, 0.05, 3)
    mesh = MeshBVH(v.cuda(), f.cuda())
    g = torch.Generator().manual_seed(2)
    train = synthetic.mixed_queries(v, f, 1 << 18, g)
    lb = train_for_mesh(mesh, train, epochs=12)
    q = synthetic.mixed_queries(v, f, 1 << 17, g).cuda()
    b = lb(q)
    ref = mesh._bvh.query(q)
    cover = (ref[0] <= b).float().mean().item()
    assert cover > 0.95
    visits = {}
    modes = {
        "plain": (None, _lib.A3D_UDF_NO_REUSE),
        "learned_cap": (b, _lib.A3D_UDF_NO_REUSE),
        "learned_seeds": (b, _lib.A3D_UDF_NO_REUSE | _lib.A3D_UDF_BOUND_SEEDS),
        "reuse": (None, 0),
        "reuse+learned_cap": (b, 0),
    }
    for name, (bound, flags) in modes.items():
        st = torch.zeros(4, dtype=torch.int64, device="cuda")
        r = mesh._bvh.query(q, bound=bound, stats=st, seeding=flags)
        for a, c in zip(ref, r):
            assert torch.equal(a, c), name  # identical distances, ids, points, uvw
        visits[name] = (int(st[0]) + int(st[1])) / q.shape[0]
    # what the trained network gains over the method without it: node +
    # triangle tests per query when the learned bound replaces the greedy
    # descent that seeds the plain method's radius (a too-small bound costs a
    # re-run, so a cap on an already tight radius may add a little work)
    print("tests per query:", {k: round(x, 1) for k, x in visits.items()})
    assert visits["learned_seeds"] < visits["plain"]
