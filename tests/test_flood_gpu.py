"""Parity of the sparse flood fill (bit-volume relaxation on the GPU) with
the oracle's sequential BFS restatement of the reference's flood_fill_kernel
and its host-side post-processing.  Integer outputs: bit-exact, same order."""

import itertools

import numpy as np
import pytest
import torch

from atom3d_b200 import MeshBVH, OctreeIndexer, flood_fill_3d_sparse, sparse_flood_fill, synthetic

pytestmark = pytest.mark.gpu


def shell(n=24, r=8.0, hole=False):
    ijk = np.array(list(itertools.product(range(n), repeat=3)))
    c = (n - 1) / 2
    d = np.linalg.norm(ijk - c, axis=1)
    keep = np.abs(d - r) < 0.9
    if hole:
        keep &= ~((ijk[:, 0] > c + r - 2) & (np.abs(ijk[:, 1] - c) < 2) & (np.abs(ijk[:, 2] - c) < 2))
    return ijk[keep]


def eq(a, b):
    a = a.cpu().numpy() if isinstance(a, torch.Tensor) else a
    return a.shape == b.shape and np.array_equal(a, b)


@pytest.mark.parametrize("conn", [6, 18, 26])
@pytest.mark.parametrize("hole", [False, True])
def test_flood_fill_3d_sparse_matches_oracle(orc, conn, hole):
    dam = shell(hole=hole) + 20
    for padding, src in [(2, (0, 0, 0)), (10, (21, 21, 21)), (3, (25, 24, 30))]:
        got = flood_fill_3d_sparse(torch.from_numpy(dam).cuda(), 64, source=src, padding=padding, connectivity=conn)
        ref = orc.flood_fill_3d_sparse(dam, 64, source=src, padding=padding, connectivity=conn)
        for g, r, name in zip(got, ref, ["water", "dry", "tide", "dam", "dam_mask", "ext"]):
            assert eq(g, r), (conn, hole, padding, src, name)


def test_crop_clamped_at_grid_boundary(orc):
    dam = shell(16, 6.0)  # touches coordinate 0 after padding clamp
    got = flood_fill_3d_sparse(torch.from_numpy(dam).cuda(), 16, padding=10)
    ref = orc.flood_fill_3d_sparse(dam, 16, padding=10)
    for g, r in zip(got, ref):
        assert eq(g, r)


def test_occupied_seed_and_empty_input():
    dam = np.array([[0, 0, 0], [1, 1, 1]])
    out = flood_fill_3d_sparse(torch.from_numpy(dam).cuda(), 16, padding=2)
    assert all(x.numel() == 0 for x in out)
    out = flood_fill_3d_sparse(torch.zeros(0, 3, dtype=torch.int64, device="cuda"), 16)
    assert all(x.numel() == 0 for x in out)


@pytest.mark.parametrize("k_ring", [1, 2, 12])
def test_sparse_flood_fill_on_mesh_matches_oracle(orc, k_ring):
    v, f = synthetic.displaced_sphere(4, 8, 0.05, 2)
    bounds = torch.tensor([[-1.5] * 3, [1.5] * 3])
    mesh = MeshBVH(v.cuda(), f.cuda())
    got = sparse_flood_fill(mesh, 64, connectivity=26, min_level=2, k_ring=k_ring, bounds=bounds.cuda())
    dam = orc.octree_traverse(v.numpy(), f.numpy(), [-1.5] * 3, [1.5] * 3, 2, 6)
    ref = orc.sparse_flood_fill_from_dam(dam, 64, connectivity=26, k_ring=k_ring)
    for k in ref:
        assert eq(got[k], ref[k]), k
    assert len(got["dry_ijk"]) > 0 and len(got["water_ijk"]) > 0


def test_flood_partition_properties_large():
    """Full-size size-independent properties (level-7 mesh, 512^3)."""
    v, f = synthetic.octree_mesh()
    bounds = torch.tensor([[-1.5] * 3, [1.5] * 3], device="cuda")
    mesh = MeshBVH(v.cuda(), f.cuda())
    out = sparse_flood_fill(mesh, 512, connectivity=26, min_level=4, bounds=bounds)
    oc = OctreeIndexer(max_level=9, bounds=bounds, device="cuda")
    dam_all = oc.octree_traverse(mesh, min_level=4)
    lo = dam_all.min(0).values - 10
    hi = dam_all.max(0).values + 10
    crop = int(torch.prod((hi.clamp(max=511) - lo.clamp(min=0) + 1)).item())
    total = sum(out[k].shape[0] for k in ("water_ijk", "dry_ijk", "tide_ijk", "dam_ijk"))
    assert total == crop
    # every label is sorted and unique
    for k, t in out.items():
        lin = (t[:, 0].long() * 512 + t[:, 1].long()) * 512 + t[:, 2].long()
        assert torch.all(lin[1:] > lin[:-1]), k
    # the sphere's centre is dry, the crop corner is water
    c = torch.tensor([256, 256, 256], device="cuda", dtype=torch.int32)
    assert (out["dry_ijk"] == c).all(1).any()
