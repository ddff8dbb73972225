from .data_structures import AABBIntersectResult, ClosestPointResult
from .device_utils import resolve_device
from .mesh_bvh import MeshBVH

__all__ = ["MeshBVH", "AABBIntersectResult", "ClosestPointResult", "resolve_device"]
