"""CPU checks of the oracle itself: pinned against the reference's golden
fixtures, against independent small pure-Python computations, and against
scipy's connected-component labelling for the flood fill."""

import itertools

import numpy as np
import pytest
import torch

from atom3d_b200 import synthetic


def test_morton_oracle_matches_reference_golden(golden, orc):
    g = golden("morton.npz")
    assert np.array_equal(orc.morton_encode(g["ijk"]), g["morton"])


def test_exact_udf_against_python_projection(orc):
    # points above the interior of a single triangle: distance = height
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    f = np.array([[0, 1, 2]], np.int32)
    rng = np.random.default_rng(0)
    uv = rng.random((200, 2)) * 0.4
    h = rng.random(200) * 2 - 1
    p = np.stack([uv[:, 0], uv[:, 1], h], 1).astype(np.float32)
    d, fid, cp = orc.udf_exact(v, f, p)
    assert np.allclose(d, np.abs(p[:, 2].astype(np.float64)), atol=1e-7)
    # beyond a vertex: distance to the vertex
    p2 = np.array([[-1, -1, 0], [2, -0.5, 0.3], [-0.2, 3, 0]], np.float32)
    d2, _, _ = orc.udf_exact(v, f, p2)
    assert np.isclose(d2[0], np.sqrt(2), atol=1e-6)
    assert np.isclose(d2[1], np.linalg.norm([1, -0.5, 0.3]), atol=1e-6)
    assert np.isclose(d2[2], np.linalg.norm([-0.2, 2, 0]), atol=1e-6)


def test_reference_fp32_restatement_close_to_fp64(orc):
    v, f, q = synthetic.udf_small(n_queries=2000)
    d64, f64, _ = orc.udf_exact(v.numpy(), f.numpy(), q.numpy())
    d32, f32, cp, uvw = orc.ref_udf_bruteforce(v.numpy(), f.numpy(), q.numpy())
    diag = float((v.max(0).values - v.min(0).values).norm())
    assert np.abs(d32 - d64).max() < 1e-6 * diag
    assert np.abs(uvw.sum(1) - 1).max() < 1e-5


def test_reference_tree_traversal_equals_bruteforce(golden, orc):
    """bvh_udf_kernel over the reference SAH tree finds the brute-force
    minimum (face ids equal up to ties)."""
    gb = golden("bvh_small.npz")
    v, f, q = gb["vs"], gb["fs"], gb["qs"]
    dt, ft, _, _ = orc.ref_bvh_udf(gb["nodes_s"], gb["tris_s"], q)
    db, fb, _, _ = orc.ref_udf_bruteforce(v, f, q)
    assert np.array_equal(dt, db) or np.abs(dt - db).max() < 1e-7
    tie = np.abs(orc.tri_dist(v, f, q, ft) - orc.tri_dist(v, f, q, fb)) < 1e-7
    assert np.all((ft == fb) | tie)


def test_reference_tree_box_hits_vs_sat_semantics(golden, orc):
    """The reference's SAT over its own tree agrees with the tree-free SAT
    semantics (the product's) on grid boxes; differences could only come from
    triangles within sat_eps of a box that their leaf box misses."""
    gb = golden("bvh_small.npz")
    v, f = gb["v3"], gb["f3"]
    lo, hi = np.float32(-1.5), np.float32(1.5)
    res = 32
    cell = np.float32((hi - lo) / np.float32(res))
    ijk = np.array(list(itertools.product(range(res), repeat=3)), np.int64)
    mn = (ijk.astype(np.float32) * cell + lo).astype(np.float32)
    mx = (mn + cell).astype(np.float32)
    mine = orc.boxes_hit(v, f, mn, mx)
    ref = orc.ref_bvh_aabb_hit(gb["nodes3"], gb["tris3"], mn, mx)
    assert mine.sum() > 0
    assert not np.any(ref & ~mine)  # reference result is a subset
    assert np.sum(mine != ref) == 0


def test_octree_oracle_subset_of_reference_cpu_broadphase(golden, orc):
    g = golden("octree_cpu.npz")
    out = orc.octree_traverse(g["v"], g["f"], [-1.5] * 3, [1.5] * 3, 2, 5)
    sup = set(map(tuple, g["cand"].tolist()))
    got = set(map(tuple, out.tolist()))
    assert got <= sup and len(got) > 0


def test_octree_oracle_order_is_hierarchical(orc):
    v, f = synthetic.displaced_sphere(3, 8, 0.05, 2)
    out = orc.octree_traverse(v.numpy(), f.numpy(), [-1.5] * 3, [1.5] * 3, 1, 4)
    # parent keys (level 1 meshgrid order, then child corner order) are non-decreasing
    par = out >> 3
    lin = (par[:, 0] * 2 + par[:, 1]) * 2 + par[:, 2]
    assert np.all(np.diff(lin) >= 0)


def _closed_shell(n=24, r=8):
    ijk = np.array(list(itertools.product(range(n), repeat=3)))
    c = (n - 1) / 2
    d = np.linalg.norm(ijk - c, axis=1)
    return ijk[np.abs(d - r) < 0.9]


@pytest.mark.parametrize("conn", [6, 26])
def test_flood_fill_oracle_vs_scipy_labels(orc, conn):
    from scipy import ndimage

    dam = _closed_shell()
    res = 64
    water, dry, coll, tdam, dmask, ext = orc.flood_fill_3d_sparse(dam + 20, res, padding=10, connectivity=conn)
    # scipy: components of the free space of the same crop
    bmin = np.maximum(dam.min(0) + 20 - 10, 0)
    bmax = np.minimum(dam.max(0) + 20 + 10, res - 1)
    size = bmax - bmin + 1
    occ = np.zeros(size, bool)
    loc = dam + 20 - bmin
    occ[loc[:, 0], loc[:, 1], loc[:, 2]] = True
    lab, _ = ndimage.label(~occ, structure=ndimage.generate_binary_structure(3, 1 if conn == 6 else 3))
    reach = lab == lab[0, 0, 0]
    wet = np.zeros(size, bool)
    allw = np.concatenate([water, coll], 0) - bmin
    wet[allw[:, 0], allw[:, 1], allw[:, 2]] = True
    assert np.array_equal(wet, reach)
    # collision = wet voxels with an occupied neighbour (in the connectivity)
    st = ndimage.generate_binary_structure(3, 1 if conn == 6 else 3)
    near_occ = ndimage.binary_dilation(occ, structure=st)
    cm = np.zeros(size, bool)
    cc = coll - bmin
    cm[cc[:, 0], cc[:, 1], cc[:, 2]] = True
    assert np.array_equal(cm, reach & near_occ)
    dm = np.zeros(size, bool)
    dd = tdam - bmin
    dm[dd[:, 0], dd[:, 1], dd[:, 2]] = True
    assert np.array_equal(dm, occ & ndimage.binary_dilation(reach, structure=st))
    # lexicographic output order
    for arr in (water, dry, coll, tdam):
        lin = (arr[:, 0].astype(np.int64) * res + arr[:, 1]) * res + arr[:, 2]
        assert np.all(np.diff(lin) > 0)


def test_flood_fill_occupied_source_returns_empty(orc):
    dam = np.array([[0, 0, 0], [1, 1, 1]])
    out = orc.flood_fill_3d_sparse(dam, 16, source=(0, 0, 0), padding=2)
    assert all(len(x) == 0 for x in out)


def test_dam_neighbourhood_signs_oracle(orc):
    dam = _closed_shell(16, 5) + 10
    d = orc.sparse_flood_fill_from_dam(dam, 64)
    # neighbours of the dam are either outside water/tide (+1), inside (-1) or dam (0)
    nb = np.concatenate([d["extended_tide_ijk"], d["dry_adjacent_ijk"]], 0)
    assert len(d["dry_adjacent_ijk"]) > 0 and len(d["extended_tide_ijk"]) > 0
    c = np.array([17.5, 17.5, 17.5])
    r_in = np.linalg.norm(d["dry_adjacent_ijk"] - c, axis=1)
    r_out = np.linalg.norm(d["extended_tide_ijk"] - c, axis=1)
    assert r_in.max() < r_out.max()
    assert len(set(map(tuple, nb.tolist())) & set(map(tuple, d["dam_ijk"].tolist()))) == 0


def test_ray_oracle_matches_reference_cpu_path(golden, orc):
    """The oracle's restatement of the reference's ray maths against the
    reference's own CPU nearest-hit results (it rejects t <= 1e-6 where the
    GPU kernel rejects t <= 1e-8, and rounds u, v in FP32 first)."""
    g = golden("ray_small.npz")
    hit, t, fid, hp, _ = orc.ray_nearest(g["v"], g["f"], g["o"], g["d"])
    ok = (g["t"] > 1e-5) | ~g["hit"]
    assert ((hit == g["hit"]) | ~ok).mean() > 0.999
    both = hit & g["hit"]
    # same formula; torch's reductions order the dot products differently and
    # the determinant's cancellation amplifies that: up to ~5e-6 relative
    assert np.allclose(t[both], g["t"][both], rtol=1e-5, atol=0)
    assert (fid[both] == g["face_ids"][both]).mean() > 0.99
    assert np.allclose(hp[both], g["hit_points"][both], atol=1e-5)


@pytest.mark.parametrize("mode", ["train", "ab", "eval"])
def test_dmc_oracle_matches_reference_golden(golden, mode):
    """The numpy restatement of SparseDiffDMC.forward against the reference's
    own outputs: training mode with a deformation, training mode with alpha
    and beta, and the QEF inference mode (which the reference solves in FP32
    by QR: its vertices sit up to ~4.4e-6 from the FP64 solution)."""
    from oracle import dmc_oracle as D

    g = golden("dmc_small.npz")
    kw = {"train": dict(deform=g["deform"]), "ab": dict(alpha=g["alpha"], beta=g["beta"]),
          "eval": dict(deform=g["deform"], mode="qef")}[mode]
    r = D.forward(g["vox"], g["sdf"], g["cidx"], int(g["res"]), **kw)
    assert np.array_equal(r["faces"], g[mode + "_faces"])
    tol = 1e-5 if mode == "eval" else 2e-6
    keys = ("vertices", "L_dev") if mode == "ab" else ("vertices", "L_dev", "p_alpha", "n_alpha")
    for k in keys:
        assert r[k].shape == g[f"{mode}_{k}"].shape, k
        assert np.abs(r[k] - g[f"{mode}_{k}"]).max() <= tol, (k, np.abs(r[k] - g[f"{mode}_{k}"]).max())


@pytest.mark.parametrize("case", ["shell", "dense", "nodry"])
def test_dual_oracle_matches_reference_golden(golden, case):
    """The numpy restatement of construct_surface_dual_graph and the dam wet
    masks against the reference's own outputs (three cell sets, including
    neighbours whose linear key wraps at the grid's faces)."""
    from oracle import dual_oracle as D

    g = golden("dual_small.npz")
    lv = int(g[f"{case}_level"])
    dry = g[f"{case}_dry"] if f"{case}_dry" in g else None
    w, v, ci, adj, cells = D.dual_graph(g[f"{case}_dam"], g[f"{case}_coll"], dry, lv, g["bounds"])
    for k, a in (("world", w), ("vijk", v), ("cube_idx", ci), ("adj_idx", adj), ("cells", cells)):
        assert np.array_equal(a, g[f"{case}_{k}"]), k
    R = 2 ** lv
    for fn, k in ((D.dam_wet_faces, "faces"), (D.dam_wet_edges, "edges"), (D.dam_wet_corners, "corners")):
        assert np.array_equal(fn(g[f"{case}_dam"], g[f"{case}_coll"], R), g[f"{case}_wet_{k}"]), k


def test_clip_oracle_demo_polygon_count(orc):
    """The oracle's SAT + clip restatement on the reference demo's workload
    (demo.ipynb cell 5: icosphere(subdivisions=1), res 512, bounds = mesh
    bounds, octree_traverse with min_level 2, intersect_aabb(mode=3)).  The
    demo printed 1,172,044 polygons with 3-7 vertices; the reference is
    built with fast math, which decides a few dozen grazing contacts
    differently from IEEE single arithmetic."""
    v, f = synthetic.icosphere(1)
    V, F = v.numpy(), f.numpy()
    lo, hi = V.min(0), V.max(0)
    cand = orc.octree_traverse(V, F, lo, hi, 2, 9)
    cell = ((hi - lo) / np.float32(512)).astype(np.float32)
    mn = (cand.astype(np.float32) * cell + lo).astype(np.float32)
    mx = (mn + cell).astype(np.float32)
    r = orc.aabb_pairs(V, F, mn, mx, mode=3)
    n = len(r["aabb_ids"])
    assert abs(n - 1_172_044) <= 64, n
    assert r["poly_counts"].min() == 3 and r["poly_counts"].max() == 7


def test_clip_oracle_single_triangle(orc):
    """Hand-checked clip: a triangle in the plane y = 0.5 crossing the unit
    box; the polygon keeps the reference's duplicate vertices where an
    edge leaves through a box edge."""
    hit, cnt, verts, cen, area = orc.clip_pair([0, 0, 0], [1, 1, 1], [-1, 0.5, -1, 2, 0.5, -1, 0.5, 0.5, 2])
    assert hit and cnt == 6
    assert np.allclose(verts[:cnt, 1], 0.5) and np.all(verts[cnt:] == 0)
    assert np.isclose(area, 1.0)  # the unit square's cross-section
    # a box the triangle misses
    hit, cnt, *_ = orc.clip_pair([5, 5, 5], [6, 6, 6], [-1, 0.5, -1, 2, 0.5, -1, 0.5, 0.5, 2])
    assert not hit and cnt == 0
