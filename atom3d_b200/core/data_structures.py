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
    hit: torch.Tensor
    t: torch.Tensor
    face_ids: torch.Tensor
    hit_points: torch.Tensor
    normals: torch.Tensor
    bary_coords: Optional[torch.Tensor] = None
