"""Parity of the closest-point / signed-distance path on the GPU.

Oracle: FP64 brute force (oracle.c, Ericson regions) for distances and
closest points; the reference's FP32 triangle maths restated in C for uvw;
golden sign fixtures from the reference's own _compute_sign.

Tolerances (from the path's specification): distances and closest points
within 1e-6 of the mesh bounding-box diagonal; face ids bit-exact except at
ties, where a tie means the returned face is itself a closest face (its FP64
distance is within the same 1e-6 * diag of the FP64 minimum).
"""

import numpy as np
import pytest
import torch

from atom3d_b200 import MeshBVH, synthetic

pytestmark = pytest.mark.gpu


def diag_of(v):
    v = v.double()
    return float((v.max(0).values - v.min(0).values).norm())


def check_udf(orc, v, f, q, res, tol_scale=1e-6):
    dist = res.distances.cpu().numpy().astype(np.float64)
    fid = res.face_ids.cpu().numpy()
    cp = res.closest_points.cpu().numpy().astype(np.float64)
    d64, f64, cp64 = orc.udf_exact(v.numpy(), f.numpy(), q.numpy())
    tol = tol_scale * diag_of(v)
    err = np.abs(dist - d64)
    assert err.max() <= tol, f"max distance error {err.max():.3e} > {tol:.3e}"
    # face id: exact, or a tie (the returned face is itself closest)
    dmine = orc.tri_dist(v.numpy(), f.numpy(), q.numpy(), fid)
    exact = fid == f64
    tie = np.abs(dmine - d64) <= tol
    assert np.all(exact | tie), f"{np.sum(~(exact | tie))} face ids are neither exact nor ties"
    # closest point lies at the returned distance from the query
    cerr = np.abs(np.linalg.norm(cp - q.numpy().astype(np.float64), axis=1) - d64)
    assert cerr.max() <= tol
    return dict(max_err=float(err.max()), exact_frac=float(exact.mean()))


def test_udf_small_mesh_vs_fp64_oracle(orc):
    v, f, q = synthetic.udf_small(n_queries=20000)
    mesh = MeshBVH(v.cuda(), f.cuda())
    res = mesh.udf(q.cuda(), return_closest=True, return_face_ids=True, return_uvw=True)
    stats = check_udf(orc, v, f, q, res)
    # most uniform queries on this bumpy sphere are closest to a shared
    # vertex or edge, where every incident face ties
    assert stats["exact_frac"] > 0.1


def test_udf_uvw_matches_reference_formula(orc):
    v, f, q = synthetic.udf_small(n_queries=5000)
    mesh = MeshBVH(v.cuda(), f.cuda())
    res = mesh.udf(q.cuda(), return_closest=True, return_face_ids=True, return_uvw=True)
    d, fid, cp, uvw = orc.ref_udf_bruteforce(v.numpy(), f.numpy(), q.numpy())
    same = res.face_ids.cpu().numpy() == fid
    assert same.mean() > 0.1
    du = np.abs(res.uvw.cpu().numpy()[same] - uvw[same])
    assert du.max() < 1e-3
    assert np.abs(res.uvw.sum(1).cpu().numpy() - 1).max() < 1e-5


def test_udf_default_returns_tensor_and_filters():
    v, f, q = synthetic.udf_small(n_queries=1000)
    mesh = MeshBVH(v.cuda(), f.cuda())
    d = mesh.udf(q.cuda())
    assert isinstance(d, torch.Tensor) and d.shape == (1000,)
    r = mesh.udf(q.cuda(), return_closest=True)
    assert r.face_ids is None and r.uvw is None and r.closest_points.shape == (1000, 3)
    r = mesh.udf(q.cuda(), return_face_ids=True)
    assert r.face_ids.dtype == torch.int32 and r.closest_points is None


@pytest.mark.parametrize("level", [0, 1, 3, 6])
def test_udf_various_sizes(orc, level):
    v, f = synthetic.displaced_sphere(level, 8, 0.05, 7)
    g = torch.Generator().manual_seed(level)
    q = synthetic.mixed_queries(v, f, 3000, g)
    mesh = MeshBVH(v.cuda(), f.cuda())
    res = mesh.udf(q.cuda(), return_closest=True, return_face_ids=True)
    check_udf(orc, v, f, q, res)


def test_single_triangle_and_degenerate(orc):
    v = torch.tensor([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [2, 2, 2], [2.5, 2.5, 2.5], [3, 3, 3]])
    f = torch.tensor([[0, 1, 2], [3, 4, 5]], dtype=torch.int32)  # second face is degenerate (collinear)
    q = torch.tensor([[0.2, 0.2, 1.0], [2.5, 2.6, 2.5], [-1, -1, -1], [5, 5, 5], [0.5, 0.5, 0.0]])
    mesh = MeshBVH(v.cuda(), f.cuda())
    res = mesh.udf(q.cuda(), return_closest=True, return_face_ids=True)
    check_udf(orc, v, f, q, res)
    one = MeshBVH(v[:3].cuda(), f[:1].cuda())
    res = one.udf(q.cuda(), return_closest=True, return_face_ids=True)
    check_udf(orc, v[:3], f[:1], q, res)


def test_empty_query():
    v, f, _ = synthetic.udf_small(n_queries=1)
    mesh = MeshBVH(v.cuda(), f.cuda())
    d = mesh.udf(torch.zeros(0, 3, device="cuda"))
    assert d.shape == (0,)


def test_unsorted_and_sorted_queries_agree():
    v, f, q = synthetic.udf_small(n_queries=20000)
    mesh = MeshBVH(v.cuda(), f.cuda())
    a = mesh._bvh.query(q.cuda(), sort_queries=True)
    b = mesh._bvh.query(q.cuda(), sort_queries=False)
    for x, y in zip(a, b):
        assert torch.equal(x, y)


def test_bound_seeding_gives_identical_results():
    v, f, q = synthetic.udf_small(n_queries=20000)
    mesh = MeshBVH(v.cuda(), f.cuda())
    qd = q.cuda()
    plain = mesh._bvh.query(qd)
    d = plain[0]
    g = torch.Generator(device="cuda").manual_seed(3)
    # valid bounds (loose), exact bounds (equal: must re-run), invalid bounds (too small)
    for bound in (d * 1.5 + 0.01, d, d * 0.5, torch.full_like(d, float("inf"))):
        got = mesh._bvh.query(qd, bound=bound.contiguous())
        for x, y in zip(plain, got):
            assert torch.equal(x, y)
    mixed = torch.where(torch.rand(d.shape, generator=g, device="cuda") < 0.5, d * 0.9, d * 1.1 + 1e-3)
    got = mesh._bvh.query(qd, bound=mixed)
    for x, y in zip(plain, got):
        assert torch.equal(x, y)


def test_sdf_sign_matches_reference_compute_sign(golden, orc):
    gs = golden("sign.npz")
    gb = golden("bvh_small.npz")
    v, f, q = (torch.from_numpy(gb[k]) for k in ("vs", "fs", "qs"))
    mesh = MeshBVH(v.cuda(), f.cuda())
    sd = mesh.sdf(q.cuda()).cpu().numpy()
    d64, _, _ = orc.udf_exact(v.numpy(), f.numpy(), q.numpy())
    ref_sign = gs["signs"]
    mine = np.where(sd < 0, -1.0, 1.0)
    # the reference decides in FP32: disagreement is only allowed within 1e-6 * diag of the surface
    near = d64 <= 1e-6 * diag_of(v)
    assert np.all((mine == ref_sign) | near)
    assert np.abs(np.abs(sd) - d64).max() <= 1e-6 * diag_of(v)


def test_sdf_sign_inside_outside_sphere():
    v, f = synthetic.icosphere(5)
    mesh = MeshBVH(v.cuda(), f.cuda())
    g = torch.Generator().manual_seed(5)
    q = (torch.rand(50000, 3, generator=g) * 3 - 1.5)
    r = q.norm(dim=1)
    keep = (r - 1).abs() > 0.01
    sd = mesh.sdf(q[keep].cuda()).cpu()
    assert torch.all((sd < 0) == (r[keep] < 1))


def test_mesh_normals_match_reference(golden):
    gn = golden("normals.npz")
    gb = golden("bvh_small.npz")
    mesh = MeshBVH(torch.from_numpy(gb["vs"]).cuda(), torch.from_numpy(gb["fs"]).cuda())
    np.testing.assert_allclose(mesh._face_normals.cpu().numpy(), gn["face_normals"], atol=2e-6)
    np.testing.assert_allclose(mesh._face_angles.cpu().numpy(), gn["face_angles"], atol=2e-5)
    np.testing.assert_allclose(mesh._vertex_pn.cpu().numpy(), gn["vertex_pn"], atol=2e-6)
    np.testing.assert_allclose(mesh._edge_pn.cpu().numpy(), gn["edge_pn"], atol=2e-6)
    assert np.array_equal(mesh._he_edge_idx.cpu().numpy(), gn["he_edge_idx"])


def test_udf_matches_reference_tree_traversal(golden, orc):
    """bvh_udf_kernel restated over the reference's own SAH tree: same face
    ids except at ties, same distances within tolerance."""
    gb = golden("bvh_small.npz")
    v, f, q = gb["vs"], gb["fs"], gb["qs"]
    d_ref, f_ref, _, _ = orc.ref_bvh_udf(gb["nodes_s"], gb["tris_s"], q)
    mesh = MeshBVH(torch.from_numpy(v).cuda(), torch.from_numpy(f).cuda())
    r = mesh.udf(torch.from_numpy(q).cuda(), return_face_ids=True)
    fid = r.face_ids.cpu().numpy()
    tol = 1e-6 * diag_of(torch.from_numpy(v))
    assert np.abs(r.distances.cpu().numpy() - d_ref).max() <= tol
    dm = orc.tri_dist(v, f, q, fid)
    dr = orc.tri_dist(v, f, q, f_ref)
    assert np.all((fid == f_ref) | (np.abs(dm - dr) <= tol))


def test_udf_grad_points_and_vertices_fd(orc):
    v, f = synthetic.displaced_sphere(2, 4, 0.05, 9)
    g = torch.Generator().manual_seed(1)
    q = synthetic.mixed_queries(v, f, 64, g, sigma=0.05)
    mesh = MeshBVH(v.cuda(), f.cuda())
    p = q.cuda().requires_grad_(True)
    vv = mesh.vertices.requires_grad_(True)
    w = torch.rand(64, generator=g).cuda()
    d = mesh.udf(p, return_grad=True)
    (d * w).sum().backward()
    gp = p.grad.cpu().double().numpy()
    gv = vv.grad.cpu().double().numpy()
    # FP64 central differences of sum_i w_i * dist_i through the oracle (with
    # h = 1e-3 they agree with the analytic FP64 gradient to 2e-5 here)
    V = v.double().numpy()
    Fn = f.numpy()
    Q = q.double().numpy()
    W = w.cpu().double().numpy()

    def energy(Vx, Qx):
        d, _, _ = orc.udf_exact(Vx.astype(np.float32), Fn, Qx.astype(np.float32))
        return float((d * W).sum())

    h = 1e-3
    for i in range(0, 64, 9):
        for a in range(3):
            Qp, Qm = Q.copy(), Q.copy()
            Qp[i, a] += h
            Qm[i, a] -= h
            fd = (energy(V, Qp) - energy(V, Qm)) / (2 * h)
            assert abs(fd - gp[i, a]) < 1e-3 * max(1.0, abs(fd)), (i, a, fd, gp[i, a])
    touched = np.argsort(-np.abs(gv).sum(1))[:6]
    for vi in touched:
        for a in range(3):
            Vp, Vm = V.copy(), V.copy()
            Vp[vi, a] += h
            Vm[vi, a] -= h
            fd = (energy(Vp, Q) - energy(Vm, Q)) / (2 * h)
            assert abs(fd - gv[vi, a]) < 2e-3 * max(1.0, abs(fd)), (vi, a, fd, gv[vi, a])


def test_cpu_device_raises():
    v, f = synthetic.icosphere(1)
    with pytest.raises(RuntimeError):
        MeshBVH(v, f, device="cpu")


@pytest.mark.parametrize("bad", [-1, "nv"])
def test_face_index_out_of_range_raises(bad):
    """A face index outside [0, V) is an argument error (the normals pass and
    the build clamp it before any access), and the device stays usable."""
    v, f = synthetic.icosphere(2)
    fb = f.clone()
    fb[7, 1] = v.shape[0] if bad == "nv" else bad
    with pytest.raises(RuntimeError, match="face index"):
        MeshBVH(v.cuda(), fb.cuda())
    d = MeshBVH(v.cuda(), f.cuda()).udf(torch.zeros(4, 3, device="cuda"))
    assert bool(torch.isfinite(d).all()) and bool((d == d[0]).all()) and 0.5 < float(d[0]) <= 1.0
