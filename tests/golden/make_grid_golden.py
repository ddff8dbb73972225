"""Generate tests/golden/grid_small.npz: outputs of the reference's
CubeGrid and OctreeIndexer host-side index maths (pure PyTorch, CPU) on
seeded inputs, for the CPU tests of atom3d_b200.grid.

Only the reference's grid modules and the two small modules they import
(constants, core/device_utils) are loaded, from a scratch copy arranged as
a minimal package, so no CUDA extension of the reference is built.

Usage:  python tests/golden/make_grid_golden.py --reference <Atom3d checkout>
"""

from __future__ import annotations

import argparse
import os
import shutil
import sys
import tempfile

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))

RES = 12
MAX_LEVEL = 6
BOUNDS = [[-1.2, -0.9, -1.1], [1.3, 1.0, 0.8]]


def import_reference_grid(path: str):
    tmp = tempfile.mkdtemp(prefix="atom3d_grid_ref_")
    pkg = os.path.join(tmp, "atom3d")
    for sub in ("", "core", "grid"):
        os.makedirs(os.path.join(pkg, sub), exist_ok=True)
        open(os.path.join(pkg, sub, "__init__.py"), "w").close()
    for rel in ("constants.py", "core/device_utils.py", "grid/cube_grid.py", "grid/octree_indexer.py"):
        shutil.copy(os.path.join(path, "atom3d", rel), os.path.join(pkg, rel))
    sys.path.insert(0, tmp)
    from atom3d.grid.cube_grid import CubeGrid
    from atom3d.grid.octree_indexer import OctreeIndexer

    return CubeGrid, OctreeIndexer


def inputs():
    g = torch.Generator().manual_seed(2024)
    lo, hi = torch.tensor(BOUNDS[0]), torch.tensor(BOUNDS[1])
    inp = {
        "ijk": torch.randint(0, RES, (50, 3), generator=g),
        "idx": torch.randint(0, RES ** 3, (50,), generator=g),
        "vidx": torch.randint(0, (RES + 1) ** 3, (40,), generator=g),
        "vijk": torch.randint(0, RES + 1, (40, 3), generator=g),
        "world": lo + (hi - lo) * torch.rand(40, 3, generator=g),
        "voxels": torch.unique(torch.randint(0, RES, (60, 3), generator=g), dim=0),
        "ijk3": torch.randint(0, 8, (10, 3), generator=g),
        "ijk4": torch.randint(0, 16, (30, 3), generator=g),
        "idx4": torch.randint(0, 16 ** 3, (30,), generator=g),
        "ijk5": torch.randint(0, 32, (30, 3), generator=g),
    }
    ne = 3 * RES * (RES + 1) ** 2
    inp["eidx"] = torch.cat([torch.randint(0, ne, (60,), generator=g), torch.tensor([0, ne - 1, ne // 3, 2 * ne // 3])])
    inp["edir"] = torch.where(torch.rand(64, generator=g) < 0.5, -1, 1)
    c = lo + (hi - lo) * torch.rand(25, 3, generator=g)
    half = 0.02 + 0.1 * torch.rand(25, 3, generator=g)
    inp["amin"], inp["amax"] = c - half, c + half
    return inp


def outputs(CubeGrid, OctreeIndexer, inp):
    b = torch.tensor(BOUNDS)
    cg = CubeGrid(RES, bounds=b, device="cpu")
    d = (RES, RES, RES)
    out = {
        "cell_size": cg.cell_size,
        "world_to_grid": cg.world_to_grid(inp["world"]),
        "grid_to_world": cg.grid_to_world(inp["ijk"]),
        "vertex_to_world": cg.vertex_to_world(inp["vijk"]),
        "ravel_ijk": cg.ravel_ijk(inp["ijk"], d),
        "unravel_idx": cg.unravel_idx(inp["idx"], d),
        "cube_to_ijk": cg.cube_to_ijk(inp["idx"]),
        "ijk_to_cube": cg.ijk_to_cube(inp["ijk"]),
        "cube_center": cg.cube_center(inp["idx"]),
        "cube_corner_vertex_indices": cg.cube_corner_vertex_indices(inp["idx"]),
        "cube_corner_coords": cg.cube_corner_coords(inp["idx"]),
        "vertex_ijk_from_indices": cg.vertex_ijk_from_indices(inp["vidx"]),
        "vertex_coords_from_indices": cg.vertex_coords_from_indices(inp["vidx"]),
        "all_cube_indices": cg.all_cube_indices(),
        "generate_all_cells": cg.generate_all_cells(),
    }
    out["cube_aabb_min"], out["cube_aabb_max"] = cg.cube_aabb(inp["idx"])
    # edge / face topology: every edge of the listed cubes, plus edges on the
    # grid's faces (incident cubes partly outside the grid)
    out["cube_edge_indices"] = cg.cube_edge_indices(inp["idx"])
    out["voxel_unique_edges_0"], out["voxel_unique_edges_1"] = cg.voxel_unique_edges(inp["voxels"])
    out["voxel_unique_edges_idx_0"], out["voxel_unique_edges_idx_1"] = cg.voxel_unique_edges(inp["idx"])
    out["edge_endpoints"] = cg.edge_endpoints(inp["eidx"])
    out["cube_face_indices"] = cg.cube_face_indices(inp["idx"])
    out["edge_incident_cubes"] = cg.edge_incident_cubes(inp["eidx"])
    out["edge_incident_cubes_dir"] = cg.edge_incident_cubes(inp["eidx"], inp["edir"])
    for k, t in enumerate(cg.voxel_unique_vertices(inp["voxels"])):
        out[f"voxel_unique_vertices_{k}"] = t
    oc = OctreeIndexer(MAX_LEVEL, bounds=b, device="cpu")
    for lv in range(MAX_LEVEL + 1):
        out[f"cell_size_level_{lv}"] = oc.get_cell_size(lv)
    out.update({
        "world_to_grid_level4": oc.world_to_grid_level(inp["world"], 4),
        "grid_to_world_level4": oc.grid_to_world_level(inp["ijk4"], 4),
        "subdivide3": oc.subdivide(inp["ijk3"], 3),
        "merge5": oc.merge(inp["ijk5"], 5),
        "all_cubes_at_level2": oc.all_cubes_at_level(2),
        "root_coords": oc.get_root_coords(),
        "cube_corner_coords_level4": oc.cube_corner_coords_level(inp["ijk4"], 4),
        "cube_to_ijk_level4": oc.cube_to_ijk_level(inp["idx4"], 4),
        "ijk_to_cube_level4": oc.ijk_to_cube_level(inp["ijk4"], 4),
        "cube_to_ijk_level_max": oc.cube_to_ijk_level(inp["idx4"]),
        "cube_edge_endpoints_level4": oc.cube_edge_endpoints_level(inp["ijk4"], 4),
        "filter_active_cubes4": oc.filter_active_cubes(inp["ijk4"], 4, inp["amin"], inp["amax"]),
    })
    out["cube_aabb_level4_ijk_min"], out["cube_aabb_level4_ijk_max"] = oc.cube_aabb_level(inp["ijk4"], 4)
    out["cube_aabb_level4_idx_min"], out["cube_aabb_level4_idx_max"] = oc.cube_aabb_level(inp["idx4"], 4)
    out["cube_aabb_level_max_min"], out["cube_aabb_level_max_max"] = oc.cube_aabb_level(inp["ijk5"])
    out["get_cell_aabb_level4_min"], out["get_cell_aabb_level4_max"] = oc.get_cell_aabb_level(inp["ijk4"], 4)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="path of the Atom3d checkout (read only)")
    args = ap.parse_args()
    CubeGrid, OctreeIndexer = import_reference_grid(args.reference)
    inp = inputs()
    out = outputs(CubeGrid, OctreeIndexer, inp)
    arrays = {f"in_{k}": v.numpy() for k, v in inp.items()}
    arrays.update({f"out_{k}": v.detach().numpy() for k, v in out.items()})
    np.savez_compressed(os.path.join(HERE, "grid_small.npz"), **arrays)
    print(f"wrote grid_small.npz with {len(arrays)} arrays")


if __name__ == "__main__":
    main()
