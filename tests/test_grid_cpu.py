"""CubeGrid / OctreeIndexer index maths against the reference's own outputs
(golden grid_small.npz, made by tests/golden/make_grid_golden.py).  These
helpers are plain PyTorch on any device, so they run here on the CPU; every
output must match bit for bit, dtype and shape included."""

import os
import sys

import numpy as np
import pytest
import torch

from atom3d_b200.grid.cube_grid import CubeGrid
from atom3d_b200.grid.octree_indexer import OctreeIndexer

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import make_grid_golden as G  # noqa: E402


@pytest.fixture(scope="module")
def grid_case(golden):
    g = golden("grid_small.npz")
    inp = {k[3:]: torch.from_numpy(np.asarray(g[k])) for k in g if k.startswith("in_")}
    return g, G.outputs(CubeGrid, OctreeIndexer, inp)


def test_grid_helpers_match_reference(grid_case):
    g, out = grid_case
    expected = sorted(k[4:] for k in g if k.startswith("out_"))
    assert expected and sorted(out) == expected
    for k in expected:
        a, b = out[k].detach().numpy(), np.asarray(g["out_" + k])
        assert a.dtype == b.dtype and a.shape == b.shape, (k, a.dtype, b.dtype, a.shape, b.shape)
        assert np.array_equal(a, b), k


def test_cube_aabb_level_rejects_other_shapes():
    oc = OctreeIndexer(3, device="cpu")
    with pytest.raises(ValueError):
        oc.cube_aabb_level(torch.zeros(4, 2, dtype=torch.int64), 2)


def test_filter_active_cubes_chunks_agree():
    """The chunked overlap test gives the all-pairs answer at any chunk size."""
    oc = OctreeIndexer(5, device="cpu")
    gen = torch.Generator().manual_seed(3)
    cubes = torch.randint(0, 32, (3000, 3), generator=gen)
    c = torch.rand(700, 3, generator=gen) * 2 - 1
    amin, amax = c - 0.03, c + 0.03
    got = oc.filter_active_cubes(cubes, 5, amin, amax)
    mn, mx = oc.cube_aabb_level(cubes, 5)
    ref = ((mn[:, None] <= amax[None]) & (mx[:, None] >= amin[None])).all(2).any(1)
    assert torch.equal(got, cubes[ref])
    assert 0 < got.shape[0] < cubes.shape[0]
