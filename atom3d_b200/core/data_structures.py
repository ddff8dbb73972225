"""Result containers returned by the public API.

Field names and meaning follow the reference's dataclasses
(atom3d/core/data_structures.py:10-108) so results are drop-in.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import torch


@dataclass
class AABBIntersectResult:
    """Box/mesh intersection: per-box hit flag plus optional (box, face) pairs."""

    hit: torch.Tensor
    aabb_ids: Optional[torch.Tensor] = None
    face_ids: Optional[torch.Tensor] = None
    centroids: Optional[torch.Tensor] = None
    areas: Optional[torch.Tensor] = None
    poly_verts: Optional[torch.Tensor] = None
    poly_counts: Optional[torch.Tensor] = None


@dataclass
class ClosestPointResult:
    """Closest-point query: distances [N], face ids [N] int32, points [N,3], uvw [N,3]."""

    distances: torch.Tensor
    face_ids: Optional[torch.Tensor]
    closest_points: Optional[torch.Tensor]
    uvw: Optional[torch.Tensor] = None
    pseudo_normals: Optional[torch.Tensor] = None


@dataclass
class RayIntersectResult:
    """Nearest hit per ray: hit [N] bool, t [N] (max_t on a miss), face ids [N]
    int32 (-1 on a miss), hit points [N,3], face normals [N,3], optional
    barycentrics [N,3]."""

    hit: torch.Tensor
    t: torch.Tensor
    face_ids: torch.Tensor
    hit_points: torch.Tensor
    normals: torch.Tensor
    bary_coords: Optional[torch.Tensor] = None


@dataclass
class RayAllHitResult:
    """Every hit of every ray, grouped by ray: ray index [H] int32, t [H],
    face ids [H] int32, sign(normal . direction) [H] int32, points [H,3],
    barycentrics [H,3]."""

    ray_idx: torch.Tensor
    t: torch.Tensor
    face_ids: torch.Tensor
    sign: torch.Tensor
    hit_points: torch.Tensor
    bary_coords: torch.Tensor
