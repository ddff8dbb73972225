"""atom3d_b200: B200-native geometry hot path of Atom3D.

Drop-in entry points (same names and signatures as the reference package
``atom3d``): MeshBVH(vertices, faces).udf/sdf, OctreeIndexer.octree_traverse,
sparse_flood_fill and SparseDiffDMC.  All compute runs in the sm_100a
library ``libatom3d_b200.so`` through its C ABI.
"""

__version__ = "0.1.0"

from .core.data_structures import AABBIntersectResult, ClosestPointResult
from .core.mesh_bvh import MeshBVH
from .grid.cube_grid import CubeGrid
from .grid.octree_indexer import OctreeIndexer
from .apps.sparse_flood_fill import flood_fill_3d_sparse, sparse_flood_fill
from .mesh_extractor.sparse_diffdmc import SparseDiffDMC, SparseDMC

__all__ = [
    "MeshBVH",
    "AABBIntersectResult",
    "ClosestPointResult",
    "OctreeIndexer",
    "CubeGrid",
    "sparse_flood_fill",
    "flood_fill_3d_sparse",
    "SparseDiffDMC",
    "SparseDMC",
]
