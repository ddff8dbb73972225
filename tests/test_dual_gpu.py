"""Surface dual graph and dam wet masks on the GPU: against the reference's
own outputs (golden dual_small.npz), against the numpy oracle on a larger
shell, and end to end on the cell sets sparse_flood_fill produces."""

import numpy as np
import pytest
import torch

from atom3d_b200 import MeshBVH, synthetic
from atom3d_b200.apps import (construct_surface_dual_graph, get_dam_wet_corners, get_dam_wet_edges,
                              get_dam_wet_faces, sparse_flood_fill)
from atom3d_b200.grid.octree_indexer import OctreeIndexer

pytestmark = pytest.mark.gpu

CASES = ("shell", "dense", "nodry")


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("case", CASES)
def test_dual_graph_matches_reference_golden(golden, case):
    g = golden("dual_small.npz")
    lv = int(g[f"{case}_level"])
    dry = _t(g[f"{case}_dry"]) if f"{case}_dry" in g else None
    octree = OctreeIndexer(max_level=lv, bounds=_t(g["bounds"]), device="cuda")
    w, v, ci, adj, cells = construct_surface_dual_graph(_t(g[f"{case}_dam"]), _t(g[f"{case}_coll"]), dry, octree)
    assert cells.dtype == torch.int32 and v.dtype == torch.int64
    assert np.array_equal(cells.cpu().numpy(), g[f"{case}_cells"])
    assert np.array_equal(v.cpu().numpy(), g[f"{case}_vijk"])
    assert np.array_equal(ci.cpu().numpy(), g[f"{case}_cube_idx"])
    assert np.array_equal(adj.cpu().numpy(), g[f"{case}_adj_idx"])
    assert np.array_equal(w.cpu().numpy(), g[f"{case}_world"])  # a product then a sum, bit for bit


@pytest.mark.parametrize("case", CASES)
def test_dam_wet_matches_reference_golden(golden, case):
    g = golden("dual_small.npz")
    R = 2 ** int(g[f"{case}_level"])
    dam, coll = _t(g[f"{case}_dam"]), _t(g[f"{case}_coll"])
    for fn, k in ((get_dam_wet_faces, "faces"), (get_dam_wet_edges, "edges"), (get_dam_wet_corners, "corners")):
        out = fn(dam, coll, R)
        assert out.dtype == torch.bool
        assert np.array_equal(out.cpu().numpy(), g[f"{case}_wet_{k}"]), k


def test_dual_graph_matches_oracle_medium():
    from oracle import dual_oracle as D

    dam, coll, dry = synthetic.shell_cells(160, seed=12)
    bounds = torch.tensor([[-1.5, -1.4, -1.3], [1.2, 1.5, 1.6]])
    octree = OctreeIndexer(max_level=8, bounds=bounds.cuda(), device="cuda")  # cells use [0, 160) of 256
    got = construct_surface_dual_graph(dam.cuda(), coll.cuda(), dry.cuda(), octree)
    exp = D.dual_graph(dam.numpy(), coll.numpy(), dry.numpy(), 8, bounds.numpy())
    for a, b in zip(got, exp):
        assert np.array_equal(a.cpu().numpy(), b)
    for fn, ofn in ((get_dam_wet_faces, D.dam_wet_faces), (get_dam_wet_edges, D.dam_wet_edges),
                    (get_dam_wet_corners, D.dam_wet_corners)):
        assert np.array_equal(fn(dam.cuda(), coll.cuda(), 256).cpu().numpy(), ofn(dam.numpy(), coll.numpy(), 256))


def test_dual_graph_on_flood_fill_output():
    """The pipeline the reference's app serves: flood-fill labels, then the
    dual graph of dam + tide + dry-adjacent cells; checked against the
    oracle and for its structural properties."""
    from oracle import dual_oracle as D

    v, f = synthetic.displaced_sphere(5, 8, 0.05, 2)
    bvh = MeshBVH(v.cuda(), f.cuda())
    bounds = torch.tensor([[-1.5] * 3, [1.5] * 3], device="cuda")
    r = sparse_flood_fill(bvh, 128, bounds=bounds, min_level=3, verbose=False)
    octree = OctreeIndexer(max_level=7, bounds=bounds, device="cuda")
    w, vijk, ci, adj, cells = construct_surface_dual_graph(r["dam_ijk"], r["tide_ijk"], r["dry_adjacent_ijk"], octree)
    exp = D.dual_graph(r["dam_ijk"].cpu().numpy(), r["tide_ijk"].cpu().numpy(), r["dry_adjacent_ijk"].cpu().numpy(),
                       7, bounds.cpu().numpy())
    for a, b in zip((w, vijk, ci, adj, cells), exp):
        assert np.array_equal(a.cpu().numpy(), b)
    # structure: every corner found and consistent, adjacency symmetric
    assert bool((ci >= 0).all())
    assert torch.equal(vijk[ci[:, 0]], cells.long())
    assert torch.equal(vijk[ci[:, 7]], cells.long() + 1)
    n = cells.shape[0]
    for k, back in ((0, 1), (2, 3), (4, 5)):
        has = adj[:, k] >= 0
        i = torch.arange(n, device="cuda")[has]
        assert torch.equal(adj[adj[has, k], back], i)
    wet = get_dam_wet_faces(r["dam_ijk"], r["tide_ijk"], 128)
    assert np.array_equal(wet.cpu().numpy(), D.dam_wet_faces(r["dam_ijk"].cpu().numpy(),
                                                             r["tide_ijk"].cpu().numpy(), 128))
    assert bool(wet.any())


def test_dual_graph_edge_cases():
    octree = OctreeIndexer(max_level=4, device="cuda")
    e = torch.empty(0, 3, dtype=torch.int32, device="cuda")
    with pytest.raises(RuntimeError):
        construct_surface_dual_graph(e, e, None, octree)
    # one cell at the grid's far corner: its +x neighbour key falls off the
    # grid, the +y / +z keys wrap (the reference's linear key)
    one = torch.tensor([[15, 15, 15]], dtype=torch.int32, device="cuda")
    w, v, ci, adj, cells = construct_surface_dual_graph(one, e, None, octree)
    # vertices in lexicographic (x, y, z) order: corner c = (c&1, (c>>1)&1,
    # (c>>2)&1) has rank 4*(c&1) + 2*((c>>1)&1) + ((c>>2)&1)
    assert v.shape == (8, 3) and ci.tolist() == [[0, 4, 2, 6, 1, 5, 3, 7]] and adj.tolist() == [[-1] * 6]
    # two cells whose keys alias through the z face: (0, 1, 15) +z -> (0, 2, 0)
    two = torch.tensor([[0, 1, 15], [0, 2, 0]], dtype=torch.int32, device="cuda")
    _, _, _, adj, _ = construct_surface_dual_graph(two, e, None, octree)
    assert adj[0, 4].item() == 1 and adj[1, 5].item() == 0
    # int64 inputs promote the cell dtype like torch.cat
    *_, cells = construct_surface_dual_graph(one.long(), e, None, octree)
    assert cells.dtype == torch.int64
    with pytest.raises(ValueError):
        construct_surface_dual_graph(one + 1, e, None, octree)
    assert get_dam_wet_faces(e, one, 16).shape == (0, 6)
    assert not bool(get_dam_wet_edges(one, e, 16).any())
    assert get_dam_wet_corners(one, e, 16).shape == (1, 8)
