"""Parity of the native SparseDiffDMC (training mode) with the reference's
golden outputs/gradients and the numpy oracle; adjoint vs FP64 central
differences.  Topology (faces) bit-exact; vertices, L_dev, p_alpha, n_alpha
within 1e-6 of the bounding-box diagonal of the grid ([-1, 1]^3: 2*sqrt(3))."""

import numpy as np
import pytest
import torch

from atom3d_b200 import SparseDiffDMC, synthetic

pytestmark = pytest.mark.gpu

TOL = 1e-6 * 2 * np.sqrt(3)


def run(g, **kw):
    dmc = SparseDiffDMC(device="cuda")
    s = torch.from_numpy(g["sdf"]).cuda().requires_grad_(True)
    args = {k: torch.from_numpy(v).cuda().requires_grad_(True) for k, v in kw.items()}
    o = dmc(torch.from_numpy(g["vox"]).cuda(), s, torch.from_numpy(g["cidx"]).cuda(), int(g["res"]), **args)
    (o.vertices ** 2).sum().backward()
    return o, s.grad, {k: v.grad for k, v in args.items()}


def test_dmc_forward_matches_reference_golden(golden):
    g = golden("dmc_small.npz")
    o, gs, ga = run(g, deform=g["deform"])
    assert np.array_equal(o.faces.cpu().numpy(), g["train_faces"])
    for k in ("vertices", "L_dev", "p_alpha", "n_alpha"):
        a, b = getattr(o, k).detach().cpu().numpy(), g["train_" + k]
        assert a.shape == b.shape, k
        assert np.abs(a - b).max() <= TOL, (k, np.abs(a - b).max())
    # reference autograd gradients (loss = sum |v|^2)
    assert np.abs(gs.cpu().numpy() - g["train_grad_sdf"]).max() <= 1e-4 * max(1.0, np.abs(g["train_grad_sdf"]).max())
    gd = ga["deform"].cpu().numpy()
    assert np.abs(gd - g["train_grad_deform"]).max() <= 1e-4 * max(1.0, np.abs(g["train_grad_deform"]).max())


def test_dmc_alpha_beta_matches_reference_golden(golden):
    g = golden("dmc_small.npz")
    o, gs, _ = run(g, alpha=g["alpha"], beta=g["beta"])
    assert np.array_equal(o.faces.cpu().numpy(), g["ab_faces"])
    assert np.abs(o.vertices.detach().cpu().numpy() - g["ab_vertices"]).max() <= TOL
    assert np.abs(o.L_dev.detach().cpu().numpy() - g["ab_L_dev"]).max() <= TOL
    assert np.abs(gs.cpu().numpy() - g["ab_grad_sdf"]).max() <= 1e-4 * max(1.0, np.abs(g["ab_grad_sdf"]).max())


def test_dmc_matches_numpy_oracle_medium():
    from oracle import dmc_oracle as D

    vox, sdf, cidx, _ = synthetic.dmc_spheres(res=96, seed=7, n_spheres=10)
    o = SparseDiffDMC(device="cuda")(vox.cuda(), sdf.cuda(), cidx.cuda(), 96)
    r = D.forward(vox.numpy(), sdf.numpy(), cidx.numpy(), 96)
    assert np.array_equal(o.faces.cpu().numpy(), r["faces"])
    for k in ("vertices", "L_dev", "p_alpha", "n_alpha"):
        assert np.abs(getattr(o, k).cpu().numpy() - r[k]).max() <= TOL, k


def test_dmc_grad_vs_fp64_central_differences():
    from oracle import dmc_oracle as D

    vox, sdf, cidx, _ = synthetic.dmc_spheres(res=24, seed=3, n_spheres=3, noise=0.0)
    s = sdf.double().numpy()
    rng = np.random.default_rng(0)
    deform = rng.normal(0, 1e-3, (s.shape[0], 3))
    o = SparseDiffDMC(device="cuda")
    st = torch.from_numpy(s).float().cuda().requires_grad_(True)
    dt = torch.from_numpy(deform).float().cuda().requires_grad_(True)
    out = o(vox.cuda(), st, cidx.cuda(), 24, deform=dt)
    (out.vertices ** 2).sum().backward()
    gs, gd = st.grad.cpu().double().numpy(), dt.grad.cpu().double().numpy()
    active = np.nonzero(np.abs(gs) > 1e-6)[0]
    pick = rng.choice(active, size=min(40, active.shape[0]), replace=False)
    h = 1e-6
    for i in pick:
        sp, sm = s.copy(), s.copy()
        sp[i] += h
        sm[i] -= h
        fp = D.loss_vertices_sq(vox.numpy(), sp, cidx.numpy(), 24, deform=deform, dtype=np.float64)
        fm = D.loss_vertices_sq(vox.numpy(), sm, cidx.numpy(), 24, deform=deform, dtype=np.float64)
        fdv = (fp - fm) / (2 * h)
        assert abs(fdv - gs[i]) <= 2e-3 * max(1.0, abs(fdv)), (i, fdv, gs[i])
    for i in pick[:15]:
        for a in range(3):
            dp, dm = deform.copy(), deform.copy()
            dp[i, a] += h
            dm[i, a] -= h
            fp = D.loss_vertices_sq(vox.numpy(), s, cidx.numpy(), 24, deform=dp, dtype=np.float64)
            fm = D.loss_vertices_sq(vox.numpy(), s, cidx.numpy(), 24, deform=dm, dtype=np.float64)
            fdv = (fp - fm) / (2 * h)
            assert abs(fdv - gd[i, a]) <= 2e-3 * max(1.0, abs(fdv)), (i, a, fdv, gd[i, a])


def test_dmc_empty_surface():
    vox = torch.tensor([[0, 0, 0]], device="cuda")
    cidx = torch.arange(8, device="cuda").view(1, 8)
    out = SparseDiffDMC(device="cuda")(vox, torch.ones(8, device="cuda"), cidx, 4)
    assert out.vertices.shape == (0, 3) and out.faces.shape == (0, 3)


def _eval(g, **kw):
    dmc = SparseDiffDMC(device="cuda").eval()
    args = {k: torch.from_numpy(v).cuda() for k, v in kw.items()}
    return dmc(torch.from_numpy(g["vox"]).cuda(), torch.from_numpy(g["sdf"]).cuda(),
               torch.from_numpy(g["cidx"]).cuda(), int(g["res"]), **args)


def test_dmc_qef_mode_matches_reference_golden(golden):
    g = golden("dmc_small.npz")
    o = _eval(g, deform=g["deform"])
    assert np.array_equal(o.faces.cpu().numpy(), g["eval_faces"])
    # the reference solves each vertex's least squares in FP32 (QR): its
    # vertices sit up to ~4.4e-6 from the FP64 solution of the same system
    for k, tol in (("vertices", 1e-5), ("L_dev", 1e-5), ("p_alpha", TOL), ("n_alpha", TOL)):
        a, b = getattr(o, k).cpu().numpy(), g["eval_" + k]
        assert a.shape == b.shape, k
        assert np.abs(a - b).max() <= tol, (k, np.abs(a - b).max())


def test_dmc_qef_mode_matches_numpy_oracle_medium():
    from oracle import dmc_oracle as D

    vox, sdf, cidx, _ = synthetic.dmc_spheres(res=96, seed=7, n_spheres=10)
    gd = torch.Generator().manual_seed(4)
    deform = (torch.randn(sdf.shape[0], 3, generator=gd) * 0.003).float()
    o = SparseDiffDMC(device="cuda").eval()(vox.cuda(), sdf.cuda(), cidx.cuda(), 96, deform=deform.cuda())
    r = D.forward(vox.numpy(), sdf.numpy(), cidx.numpy(), 96, deform=deform.numpy(), mode="qef")
    assert np.array_equal(o.faces.cpu().numpy(), r["faces"])
    for k in ("vertices", "L_dev", "p_alpha", "n_alpha"):
        assert np.abs(getattr(o, k).cpu().numpy() - r[k]).max() <= TOL, (k, np.abs(getattr(o, k).cpu().numpy() - r[k]).max())


def test_dmc_corner_gradients_and_given_gradients():
    from oracle import dmc_oracle as D
    from atom3d_b200.mesh_extractor import sparse_diffdmc as M

    vox, sdf, cidx, _ = synthetic.dmc_spheres(res=64, seed=8, n_spheres=6)
    x = D.CUBE_CORNERS
    # oracle corner gradients on the undeformed grid
    pos = np.zeros((sdf.shape[0], 3), np.float32)
    pos[cidx.numpy().reshape(-1)] = (vox.numpy()[:, None, :] + x[None]).reshape(-1, 3)
    world = pos * np.float32(2.0 / 64) - np.float32(1.0)
    G = D.corner_gradients(world, sdf.numpy(), cidx.numpy())
    c = M._DmcContext(vox.cuda(), sdf.cuda(), cidx.cuda(), 64, None, None, None, 0.0, 0.99)
    got = torch.empty(sdf.shape[0], 3, device="cuda")
    lib = M._bind()
    from atom3d_b200 import _lib

    ws = _lib.workspace(lib.a3d_dmc_corner_gradients_workspace_bytes(vox.shape[0], sdf.shape[0]), "cuda")
    _lib.check("a3d_dmc_corner_gradients", lib.a3d_dmc_corner_gradients(
        __import__("ctypes").byref(c.inp), ws.data_ptr(), ws.numel(), got.data_ptr(), c.stream))
    assert np.allclose(got.cpu().numpy(), G, rtol=1e-5, atol=1e-5)
    # caller-supplied gradients are used as given
    Gs = (G * np.float32(0.5)).astype(np.float32)
    o = SparseDiffDMC(device="cuda").eval()(vox.cuda(), sdf.cuda(), cidx.cuda(), 64,
                                            corner_gradients=torch.from_numpy(Gs).cuda())
    r = D.forward(vox.numpy(), sdf.numpy(), cidx.numpy(), 64, mode="qef", corner_grads=Gs)
    assert np.array_equal(o.faces.cpu().numpy(), r["faces"])
    assert np.abs(o.vertices.cpu().numpy() - r["vertices"]).max() <= TOL


def test_dmc_qef_grad_matches_reference_autograd(golden):
    """QEF (eval) mode gradients of sum |v|^2 w.r.t. sdf and deform against
    the reference's own autograd (torch.linalg.lstsq in FP32 QR; this build
    solves the same system through FP64 normal equations, so the vertices
    differ by up to ~4.4e-6 and the gradients by a few 1e-4 of their scale)."""
    g = golden("dmc_small.npz")
    dmc = SparseDiffDMC(device="cuda").eval()
    s = torch.from_numpy(g["sdf"]).cuda().requires_grad_(True)
    de = torch.from_numpy(g["deform"]).cuda().requires_grad_(True)
    o = dmc(torch.from_numpy(g["vox"]).cuda(), s, torch.from_numpy(g["cidx"]).cuda(), int(g["res"]), deform=de)
    (o.vertices ** 2).sum().backward()
    for got, ref in ((s.grad, g["eval_grad_sdf"]), (de.grad, g["eval_grad_deform"])):
        got = got.cpu().numpy()
        scale = max(1.0, np.abs(ref).max())
        err = np.abs(got - ref)
        assert err.max() <= 2e-3 * scale, (err.max(), scale)
        assert np.median(err[np.abs(ref) > 0]) <= 1e-5 * scale


def _qef_loss(out, w):
    return ((out["vertices"] ** 2).sum() + (w["L_dev"] * out["L_dev"]).sum() + (w["p_alpha"] * out["p_alpha"]).sum()
            + (w["n_alpha"] * out["n_alpha"]).sum())


def test_dmc_qef_grad_vs_fp64_central_differences():
    """Every output of the QEF mode (vertices, L_dev, p_alpha, n_alpha) in one
    seeded linear functional; its gradient w.r.t. sdf, deform and caller-given
    corner gradients against FP64 central differences of the oracle's QEF
    forward (the corner gradients held fixed, as the reference's are)."""
    from oracle import dmc_oracle as D

    vox, sdf, cidx, _ = synthetic.dmc_spheres(res=24, seed=3, n_spheres=3, noise=0.0)
    s = sdf.double().numpy()
    rng = np.random.default_rng(1)
    deform = rng.normal(0, 1e-3, (s.shape[0], 3))
    G = D.corner_gradients(_corner_positions(vox.numpy(), cidx.numpy(), 24, deform), s, cidx.numpy(),
                           dtype=np.float64)
    ref0 = D.forward(vox.numpy(), s, cidx.numpy(), 24, deform=deform, dtype=np.float64, mode="qef", corner_grads=G)
    w = {k: rng.normal(0, 1, ref0[k].shape) for k in ("L_dev", "p_alpha", "n_alpha")}

    st = torch.from_numpy(s).float().cuda().requires_grad_(True)
    dt = torch.from_numpy(deform).float().cuda().requires_grad_(True)
    gt = torch.from_numpy(G).float().cuda().requires_grad_(True)
    o = SparseDiffDMC(device="cuda").eval()(vox.cuda(), st, cidx.cuda(), 24, deform=dt, corner_gradients=gt)
    assert np.array_equal(o.faces.cpu().numpy(), ref0["faces"])
    wt = {k: torch.from_numpy(v).float().cuda() for k, v in w.items()}
    loss = ((o.vertices ** 2).sum() + (wt["L_dev"] * o.L_dev).sum() + (wt["p_alpha"] * o.p_alpha).sum()
            + (wt["n_alpha"] * o.n_alpha).sum())
    loss.backward()
    gs, gd, gg = (t.grad.cpu().double().numpy() for t in (st, dt, gt))

    def f(ss=s, dd=deform, gg_=G):
        return _qef_loss(D.forward(vox.numpy(), ss, cidx.numpy(), 24, deform=dd, dtype=np.float64, mode="qef",
                                   corner_grads=gg_), w)

    h = 1e-6
    active = np.nonzero(np.abs(gs) > 1e-6)[0]
    pick = rng.choice(active, size=min(30, active.shape[0]), replace=False)
    for i in pick:
        sp, sm = s.copy(), s.copy()
        sp[i] += h
        sm[i] -= h
        fdv = (f(ss=sp) - f(ss=sm)) / (2 * h)
        assert abs(fdv - gs[i]) <= 2e-3 * max(1.0, abs(fdv)), ("sdf", i, fdv, gs[i])
    for i in pick[:10]:
        for a in range(3):
            dp, dm = deform.copy(), deform.copy()
            dp[i, a] += h
            dm[i, a] -= h
            fdv = (f(dd=dp) - f(dd=dm)) / (2 * h)
            assert abs(fdv - gd[i, a]) <= 2e-3 * max(1.0, abs(fdv)), ("deform", i, a, fdv, gd[i, a])
    gact = np.nonzero(np.abs(gg).sum(1) > 1e-6)[0]
    for i in rng.choice(gact, size=min(10, gact.shape[0]), replace=False):
        for a in range(3):
            gp, gm = G.copy(), G.copy()
            gp[i, a] += h
            gm[i, a] -= h
            fdv = (f(gg_=gp) - f(gg_=gm)) / (2 * h)
            assert abs(fdv - gg[i, a]) <= 2e-3 * max(1.0, abs(fdv)), ("corner gradient", i, a, fdv, gg[i, a])


def _corner_positions(vox, cidx, res, deform):
    from oracle import dmc_oracle as D

    M = deform.shape[0]
    pos = np.zeros((M, 3))
    pos[cidx.reshape(-1)] = (vox[:, None, :] + D.CUBE_CORNERS[None]).reshape(-1, 3)
    return pos * (2.0 / res) - 1.0 + deform


@pytest.mark.parametrize("mode", ["train", "eval"])
def test_dmc_cube_idx_out_of_range_raises(golden, mode):
    """A cube_idx entry outside [0, M) is an argument error: every kernel reads
    such an entry as corner 0 and the topology pass reports it at its first
    host read, before any output is written."""
    g = golden("dmc_small.npz")
    dmc = SparseDiffDMC(device="cuda")
    if mode == "eval":
        dmc = dmc.eval()
    vox, sdf = torch.from_numpy(g["vox"]).cuda(), torch.from_numpy(g["sdf"]).cuda()
    deform = torch.from_numpy(g["deform"]).cuda()
    for bad in (sdf.shape[0], -1):
        cidx = torch.from_numpy(g["cidx"]).cuda().clone()
        cidx[cidx.shape[0] // 2, 5] = bad
        with pytest.raises(RuntimeError, match="outside"):
            dmc(vox, sdf, cidx, int(g["res"]), deform=deform)
    # the next valid call is unaffected
    o = dmc(vox, sdf, torch.from_numpy(g["cidx"]).cuda(), int(g["res"]), deform=deform)
    key = "train_faces" if mode == "train" else "eval_faces"
    assert np.array_equal(o.faces.cpu().numpy(), g[key])


def test_dmc_corner_gradients_non_grid_indices():
    """Cube indices that are not one grid's (a corner with two different +x
    neighbours: one cube uses a duplicate of a shared corner) take the
    adjacency-list gather; it matches the oracle like the grid gather."""
    import ctypes

    from oracle import dmc_oracle as D
    from atom3d_b200 import _lib
    from atom3d_b200.mesh_extractor import sparse_diffdmc as M

    vox, sdf, cidx, _ = synthetic.dmc_spheres(res=64, seed=8, n_spheres=6)
    ci = cidx.numpy().copy()
    # an x-edge (corner slots (0,1), (2,3), (4,5) or (6,7)) held by two cubes
    pairs = [(0, 1), (2, 3), (4, 5), (6, 7)]
    keys = np.concatenate([ci[:, p] for p in pairs])
    _, first, counts = np.unique(keys, axis=0, return_index=True, return_counts=True)
    k = int(first[np.argmax(counts >= 2)])
    assert counts.max() >= 2
    cube, (p0, p1) = k % ci.shape[0], pairs[k // ci.shape[0]]
    m = sdf.shape[0]
    b = int(ci[cube, p1])
    ci[cube, p1] = m  # this cube's copy of corner b
    sdf2 = np.concatenate([sdf.numpy(), sdf.numpy()[b:b + 1]])
    x = D.CUBE_CORNERS
    pos = np.zeros((m + 1, 3), np.float32)
    pos[ci.reshape(-1)] = (vox.numpy()[:, None, :] + x[None]).reshape(-1, 3)
    world = pos * np.float32(2.0 / 64) - np.float32(1.0)
    G = D.corner_gradients(world, sdf2, ci)
    c = M._DmcContext(vox.cuda(), torch.from_numpy(sdf2).cuda(), torch.from_numpy(ci).cuda(), 64, None, None, None,
                      0.0, 0.99)
    got = torch.empty(m + 1, 3, device="cuda")
    lib = M._bind()
    ws = _lib.workspace(lib.a3d_dmc_corner_gradients_workspace_bytes(vox.shape[0], m + 1), "cuda")
    _lib.check("a3d_dmc_corner_gradients", lib.a3d_dmc_corner_gradients(
        ctypes.byref(c.inp), ws.data_ptr(), ws.numel(), got.data_ptr(), c.stream))
    assert np.allclose(got.cpu().numpy(), G, rtol=1e-5, atol=1e-5)


def _features_case():
    import os
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_dmc_features_golden as G

    return G.inputs()


def test_dmc_vertex_features_train_mode_vs_reference(golden):
    g = golden("dmc_features.npz")
    vox, sdf, cidx, feat, alpha, beta = _features_case()
    s = sdf.cuda().requires_grad_(True)
    f = feat.cuda().requires_grad_(True)
    a = alpha.cuda().requires_grad_(True)
    b = beta.cuda().requires_grad_(True)
    o = SparseDiffDMC(device="cuda")(vox.cuda(), s, cidx.cuda(), int(g["res"]), alpha=a, beta=b, v_features=f)
    ((o.vertices ** 2).sum() + (o.v_features ** 2).sum()).backward()
    assert np.array_equal(o.faces.cpu().numpy(), g["train_faces"])
    assert np.abs(o.vertices.detach().cpu().numpy() - g["train_vertices"]).max() <= TOL
    vf = o.v_features.detach().cpu().numpy()
    assert vf.shape == g["train_v_features"].shape
    assert np.abs(vf - g["train_v_features"]).max() <= 1e-5 * max(1.0, np.abs(g["train_v_features"]).max())
    for name, t in (("grad_sdf", s), ("grad_feat", f), ("grad_alpha", a), ("grad_beta", b)):
        ref = g[name]
        got = t.grad.cpu().numpy()
        assert np.abs(got - ref).max() <= 1e-4 * max(1.0, np.abs(ref).max()), (name, np.abs(got - ref).max())


def test_dmc_qef_mode_alpha_and_features_vs_reference(golden):
    g = golden("dmc_features.npz")
    vox, sdf, cidx, feat, alpha, _ = _features_case()
    dmc = SparseDiffDMC(device="cuda")
    dmc.eval()
    o = dmc(vox.cuda(), sdf.cuda(), cidx.cuda(), int(g["res"]), alpha=alpha.cuda(), v_features=feat.cuda())
    assert np.array_equal(o.faces.cpu().numpy(), g["eval_faces"])
    assert np.abs(o.vertices.cpu().numpy() - g["eval_vertices"]).max() <= 1e-5
    assert np.abs(o.p_alpha.cpu().numpy() - g["eval_p_alpha"]).max() <= TOL
    ref = g["eval_v_features"]
    assert np.abs(o.v_features.cpu().numpy() - ref).max() <= 1e-5 * max(1.0, np.abs(ref).max())


def test_dmc_float64_inputs_need_an_explicit_dtype():
    vox, sdf, cidx, _ = synthetic.dmc_spheres(res=24, seed=3, n_spheres=3)
    with pytest.raises(TypeError):
        SparseDiffDMC(device="cuda")(vox.cuda(), sdf.double().cuda(), cidx.cuda(), 24)
    o = SparseDiffDMC(device="cuda")(vox.cuda(), sdf.double().cuda(), cidx.cuda(), 24, dtype=torch.float32)
    r = SparseDiffDMC(device="cuda")(vox.cuda(), sdf.cuda(), cidx.cuda(), 24)
    assert o.vertices.dtype == torch.float32 and torch.equal(o.vertices, r.vertices)
