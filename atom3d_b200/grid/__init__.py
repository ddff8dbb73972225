from .cube_grid import CubeGrid
from .octree_indexer import OctreeIndexer

__all__ = ["OctreeIndexer", "CubeGrid"]
