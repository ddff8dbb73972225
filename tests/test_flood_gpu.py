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


def serpentine_dam(lo=20, hi=179, fine=True):
    """A closed box shell [lo, hi]^3 whose inside is a serpentine: walls at
    every other y, spanning x and z, each open at alternating x ends, so the
    water entering through one opening in the -x face walks every corridor
    across all bricks (many relaxation rounds).  With ``fine`` the walls of
    the corridors inside the first 32 x 32 rows also open at alternating ends
    of that brick, a path of about 16 x 32 steps inside one brick: longer than
    a brick's per-round iteration cap, so the brick has to queue itself again."""
    n = hi - lo + 1
    ax = np.arange(lo, hi + 1)
    X, Y, Z = np.meshgrid(ax, ax, ax, indexing="ij")
    shell = (X == lo) | (X == hi) | (Y == lo) | (Y == hi) | (Z == lo) | (Z == hi)
    shell &= ~((X == lo) & (Y == lo + 1) & (Z > lo) & (Z < hi))  # the inlet
    inner = (X > lo) & (X < hi) & (Y > lo) & (Y < hi) & (Z > lo) & (Z < hi)
    wall = inner & ((Y - lo) % 2 == 0)
    k = (Y - lo) // 2
    gap_x = np.where(k % 2 == 1, lo + 1, hi - 1)
    wall &= X != gap_x
    if fine:
        b0 = (lo // 32 + 1) * 32  # a brick fully inside the box
        inb = (X >= b0) & (X < b0 + 32) & (Y >= b0) & (Y < b0 + 32)
        # inside that brick the corridor walls open at alternating brick ends
        fine_gap = np.where(k % 2 == 1, b0, b0 + 31)
        wall &= ~(inb & (X == fine_gap))
    assert n > 64
    maze = np.argwhere(shell | wall).astype(np.int64) + lo
    # a sealed hollow box beside the maze: its inside stays dry
    b = np.arange(hi + 6, hi + 17)
    B = np.stack(np.meshgrid(b, b, b, indexing="ij"), -1).reshape(-1, 3)
    edge = ((B == b[0]) | (B == b[-1])).any(1)
    return np.concatenate([maze, B[edge]])


@pytest.mark.parametrize("conn", [6, 26])
def test_flood_serpentine_many_rounds_matches_oracle(orc, conn):
    from atom3d_b200.apps.sparse_flood_fill import _Flood

    dam = serpentine_dam()
    got = flood_fill_3d_sparse(torch.from_numpy(dam).cuda(), 256, padding=2, connectivity=conn)
    ref = orc.flood_fill_3d_sparse(dam, 256, padding=2, connectivity=conn)
    for g, r, name in zip(got, ref, ["water", "dry", "tide", "dam", "dam_mask", "ext"]):
        assert eq(g, r), (conn, name)
    assert ref[0].shape[0] + ref[2].shape[0] > 2_000_000  # the water did walk the maze
    assert ref[1].shape[0] >= 9 ** 3  # the sealed box
    fl = _Flood(torch.from_numpy(dam).cuda(), 256, (0, 0, 0), 2, conn, 0)
    assert fl.rounds > 100, fl.rounds


def test_flood_closure_512():
    """At 512^3: no free crop voxel outside the water touches the water
    (conn 26), i.e. the relaxation reached its fixed point."""
    v, f = synthetic.octree_mesh()
    bounds = torch.tensor([[-1.5] * 3, [1.5] * 3], device="cuda")
    mesh = MeshBVH(v.cuda(), f.cuda())
    out = sparse_flood_fill(mesh, 512, connectivity=26, min_level=4, bounds=bounds, verbose=False)
    oc = OctreeIndexer(max_level=9, bounds=bounds, device="cuda")
    dam = oc.octree_traverse(mesh, min_level=4)
    lo = (dam.min(0).values - 10).clamp(min=0)
    hi = (dam.max(0).values + 10).clamp(max=511)
    size = (hi - lo + 1).tolist()

    def vol(t):
        m = torch.zeros(size, dtype=torch.bool, device="cuda")
        if t.shape[0]:
            c = t.long() - lo
            m[c[:, 0], c[:, 1], c[:, 2]] = True
        return m

    wet = vol(out["water_ijk"]) | vol(out["tide_ijk"])
    occ = vol(dam)
    grown = torch.nn.functional.max_pool3d(wet.float()[None, None], 3, 1, 1)[0, 0] > 0.5
    leak = grown & ~wet & ~occ
    assert int(leak.sum()) == 0


@pytest.mark.parametrize("k_ring", [0, 1, 2, 3])
def test_get_dam_neighborhood_signs_matches_oracle(orc, k_ring):
    from atom3d_b200.apps import get_dam_neighborhood_signs

    g = np.random.default_rng(k_ring)
    dam = shell(24, 8.0) + 3
    # the grid's faces are reached too: a dam blob against coordinate 0 and R-1
    dam = np.concatenate([dam, [[0, 5, 5], [0, 6, 5], [31, 31, 31], [30, 31, 0]]])
    dam = dam[g.permutation(dam.shape[0])]
    box = np.argwhere(np.ones((32, 32, 32), bool))
    water = box[g.random(box.shape[0]) < 0.4]
    dry = box[g.random(box.shape[0]) < 0.3]
    got_ijk, got_s = get_dam_neighborhood_signs(torch.from_numpy(dam).cuda(), torch.from_numpy(water).cuda(),
                                                torch.from_numpy(dry).cuda().int(), 32, k_ring=k_ring)
    ref_ijk, ref_s = orc.dam_neighborhood_signs(dam, water, dry, 32, k_ring)
    assert got_ijk.dtype == torch.int32 and got_s.dtype == torch.int8
    assert eq(got_ijk, ref_ijk.astype(np.int32)) and eq(got_s, ref_s)
    assert (got_s == 0).sum().item() == np.unique(dam, axis=0).shape[0] if k_ring else True


def test_get_dam_neighborhood_signs_edge_cases():
    from atom3d_b200.apps import get_dam_neighborhood_signs

    e = torch.zeros(0, 3, dtype=torch.int64, device="cuda")
    a, b = get_dam_neighborhood_signs(e, e, e, 16)
    assert a.shape == (0, 3) and b.shape == (0,)
    with pytest.raises(ValueError):
        get_dam_neighborhood_signs(torch.tensor([[16, 0, 0]], device="cuda"), e, e, 16)
    a, b = get_dam_neighborhood_signs(torch.tensor([[0, 0, 0]], device="cuda"), e, e, 16, k_ring=1)
    assert a.shape == (8, 3) and int((b == 0).sum()) == 1 and int((b == 1).sum()) == 7
