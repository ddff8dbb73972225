"""Parity of Morton keys, SAT box queries and the octree descent on the GPU.

Integer outputs are compared bit-exactly: against the reference's own
Morton functions (golden fixture) and against the oracle's restatement of
triangle_aabb_sat / octree_traverse (same per-operation IEEE rounding, no
FMA contraction on either side).
"""

import numpy as np
import pytest
import torch

from atom3d_b200 import MeshBVH, OctreeIndexer, synthetic

pytestmark = pytest.mark.gpu


def test_morton_matches_reference(golden):
    g = golden("morton.npz")
    oc = OctreeIndexer(max_level=10, device="cuda")
    ijk = torch.from_numpy(g["ijk"]).cuda()
    m = oc._ijk_to_morton(ijk)
    assert np.array_equal(m.cpu().numpy(), g["morton"])
    assert np.array_equal(oc._morton_to_ijk(m, 10).cpu().numpy(), g["ijk_l10"])
    assert np.array_equal(oc._morton_to_ijk(m, 5).cpu().numpy(), g["ijk_l5"])


def test_aabb_hit_matches_oracle(orc):
    v, f = synthetic.displaced_sphere(4, 8, 0.05, 2)
    mesh = MeshBVH(v.cuda(), f.cuda())
    g = torch.Generator().manual_seed(0)
    c = torch.rand(30000, 3, generator=g) * 3 - 1.5
    h = torch.rand(30000, 3, generator=g) * 0.05 + 1e-4
    mn, mx = c - h, c + h
    hit = mesh.intersect_aabb(mn.cuda(), mx.cuda(), mode=0).hit.cpu().numpy()
    ref = orc.boxes_hit(v.numpy(), f.numpy(), mn.numpy(), mx.numpy())
    assert hit.sum() > 100
    assert np.array_equal(hit, ref)


def test_aabb_hit_grid_aligned_boxes_match_oracle(orc):
    v, f = synthetic.displaced_sphere(4, 8, 0.05, 2)
    mesh = MeshBVH(v.cuda(), f.cuda())
    oc = OctreeIndexer(max_level=6, bounds=torch.tensor([[-1.5] * 3, [1.5] * 3]), device="cuda")
    cubes = oc.all_cubes_at_level(6)
    mn, mx = oc.cube_aabb_level(cubes, 6)
    hit = mesh.aabb_hit(mn, mx).cpu().numpy()
    ref = orc.boxes_hit(v.numpy(), f.numpy(), mn.cpu().numpy(), mx.cpu().numpy())
    assert np.array_equal(hit, ref)


@pytest.mark.parametrize("level,min_level,max_level", [(3, 2, 5), (4, 0, 6), (5, 4, 7)])
def test_octree_traverse_matches_oracle(orc, level, min_level, max_level):
    v, f = synthetic.displaced_sphere(level, 8, 0.05, 2)
    mesh = MeshBVH(v.cuda(), f.cuda())
    lo, hi = [-1.5] * 3, [1.5] * 3
    oc = OctreeIndexer(max_level=max_level, bounds=torch.tensor([lo, hi]), device="cuda")
    got = oc.octree_traverse(mesh, min_level=min_level).cpu().numpy()
    ref = orc.octree_traverse(v.numpy(), f.numpy(), lo, hi, min_level, max_level)
    assert got.dtype == np.int64
    assert np.array_equal(got, ref)


def test_octree_subset_of_reference_cpu_broadphase(golden):
    g = golden("octree_cpu.npz")
    mesh = MeshBVH(torch.from_numpy(g["v"]).cuda(), torch.from_numpy(g["f"]).cuda())
    oc = OctreeIndexer(max_level=5, bounds=torch.tensor([[-1.5] * 3, [1.5] * 3]), device="cuda")
    got = oc.octree_traverse(mesh, min_level=2).cpu().numpy()
    sup = g["cand"]
    key = lambda a: set(map(tuple, a.tolist()))
    assert key(got) <= key(sup)
    assert len(got) > 0.5 * len(sup)


def test_octree_default_bounds_and_empty_region():
    v, f = synthetic.icosphere(3)
    mesh = MeshBVH((v * 0.2 + 5.0).cuda(), f.cuda())  # far outside [-1, 1]^3
    oc = OctreeIndexer(max_level=5, device="cuda")
    out = oc.octree_traverse(mesh, min_level=1)
    assert out.shape == (0, 3)
