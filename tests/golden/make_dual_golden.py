"""Generate tests/golden/dual_small.npz by running the reference package's
construct_surface_dual_graph and get_dam_wet_faces / _edges / _corners
(atom3d/apps/sparse_flood_fill.py:169-291, pure PyTorch) on CPU tensors in
the build container.

Cases:
  shell   shell_cells(32): three sphere shells plus cells on the grid faces
          and duplicates across the lists; bounds [[-1.2,-1.1,-1.3],
          [1.3,1.2,1.1]] (max_level 5)
  dense   60 random cells in [0, 8)^3 (max_level 3): many neighbours off the
          grid's y and z faces, where the reference's linear key wraps
  nodry   the shell case with dry_adjacent_ijk = None

Usage:  python tests/golden/make_dual_golden.py --reference <Atom3d checkout>
"""

from __future__ import annotations

import argparse
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

from atom3d_b200 import synthetic  # noqa: E402
from make_golden import import_reference  # noqa: E402

BOUNDS = [[-1.2, -1.1, -1.3], [1.3, 1.2, 1.1]]


def cases():
    dam, coll, dry = synthetic.shell_cells(32, seed=6)
    g = torch.Generator().manual_seed(11)
    d = torch.randint(0, 8, (60, 3), generator=g).int()
    yield "shell", dam, coll, dry, 5
    yield "dense", d[:20].contiguous(), d[20:45].contiguous(), d[45:].contiguous(), 3
    yield "nodry", dam, coll, None, 5


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="path of the Atom3d checkout (read only)")
    args = ap.parse_args()
    import_reference(args.reference)
    from atom3d.apps.sparse_flood_fill import (construct_surface_dual_graph, get_dam_wet_corners,
                                               get_dam_wet_edges, get_dam_wet_faces)
    from atom3d.grid.octree_indexer import OctreeIndexer

    out = {}
    for name, dam, coll, dry, lv in cases():
        octree = OctreeIndexer(max_level=lv, bounds=torch.tensor(BOUNDS), device="cpu")
        R = 2 ** lv
        out[f"{name}_dam"] = dam.numpy()
        out[f"{name}_coll"] = coll.numpy()
        if dry is not None:
            out[f"{name}_dry"] = dry.numpy()
        out[f"{name}_level"] = np.int64(lv)
        w, v, ci, adj, cells = construct_surface_dual_graph(dam, coll, dry, octree)
        for k, t in (("world", w), ("vijk", v), ("cube_idx", ci), ("adj_idx", adj), ("cells", cells)):
            out[f"{name}_{k}"] = t.numpy()
        out[f"{name}_wet_faces"] = get_dam_wet_faces(dam, coll, R).numpy()
        out[f"{name}_wet_edges"] = get_dam_wet_edges(dam, coll, R).numpy()
        out[f"{name}_wet_corners"] = get_dam_wet_corners(dam, coll, R).numpy()
        print(name, "cells", cells.shape[0], cells.dtype, "verts", v.shape[0], v.dtype,
              "adj found", int((adj >= 0).sum()))
    out["bounds"] = np.array(BOUNDS, np.float32)
    np.savez_compressed(os.path.join(HERE, "dual_small.npz"), **out)


if __name__ == "__main__":
    main()
