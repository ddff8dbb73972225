"""CubeGrid: dense cube-grid index maths (drop-in subset of the reference's
atom3d/grid/cube_grid.py:33-557).

Integer index conventions are the reference's: linear index of (i, j, k) in
dims (nx, ny, nz) is (i * ny + j) * nz + k, cube corners follow CUBE_CORNERS
(x fastest), grid bounds default to [-1, 1]^3 and the cell size is
(hi - lo) / res in float32.  This module is host-side bookkeeping (PyTorch on
any device); the octree descent itself runs in the native library.
"""

from __future__ import annotations

from typing import Optional, Tuple, Union

import torch

from ..constants import CUBE_CORNERS, CUBE_EDGES, CUBE_FACES, EDGE_TO_FACES
from ..core.device_utils import resolve_device


class CubeGrid:
    def __init__(self, resolution: int, bounds: Optional[torch.Tensor] = None,
                 device: Optional[Union[str, torch.device]] = None):
        if not isinstance(resolution, int) or resolution < 1:
            raise ValueError(f"resolution must be positive int, got {resolution}")
        self.res = int(resolution)
        self.device = resolve_device(bounds, device=device, default="cuda")
        self.dtype = torch.float32
        self.index_dtype = torch.int64
        self.num_vertices_per_axis = self.res + 1
        self.num_cubes = self.res ** 3
        self.num_vertices = self.num_vertices_per_axis ** 3
        if bounds is not None:
            if tuple(bounds.shape) != (2, 3):
                raise ValueError(f"bounds must be [2,3], got {tuple(bounds.shape)}")
            self.bounds = bounds.to(device=self.device, dtype=self.dtype)
        else:
            self.bounds = torch.tensor([[-1.0] * 3, [1.0] * 3], device=self.device, dtype=self.dtype)
        self.cell_size = (self.bounds[1] - self.bounds[0]) / float(self.res)
        self.CUBE_CORNERS = CUBE_CORNERS.to(self.device)
        self.CUBE_EDGES = CUBE_EDGES.to(self.device)
        self.CUBE_FACES = CUBE_FACES.to(self.device)
        self.EDGE_TO_FACES = EDGE_TO_FACES.to(self.device)

    # coordinate conversions
    def world_to_grid(self, world_coords: torch.Tensor) -> torch.Tensor:
        return (world_coords.to(self.device, dtype=self.dtype) - self.bounds[0]) / self.cell_size

    def grid_to_world(self, grid_coords: torch.Tensor) -> torch.Tensor:
        return (grid_coords.to(self.device).float() + 0.5) * self.cell_size + self.bounds[0]

    def vertex_to_world(self, vertex_ijk: torch.Tensor) -> torch.Tensor:
        return vertex_ijk.to(self.device).float() * self.cell_size + self.bounds[0]

    # index utilities
    def ravel_ijk(self, ijk: torch.Tensor, dims: Tuple[int, int, int]) -> torch.Tensor:
        _, ny, nz = dims
        ijk = ijk.to(device=self.device, dtype=self.index_dtype)
        return (ijk[..., 0] * ny + ijk[..., 1]) * nz + ijk[..., 2]

    def unravel_idx(self, idx: torch.Tensor, dims: Tuple[int, int, int]) -> torch.Tensor:
        _, ny, nz = dims
        idx = idx.to(device=self.device, dtype=self.index_dtype)
        i = torch.div(idx, ny * nz, rounding_mode="floor")
        rem = idx - i * (ny * nz)
        j = torch.div(rem, nz, rounding_mode="floor")
        return torch.stack([i, j, rem - j * nz], dim=-1)

    # cubes
    def all_cube_indices(self) -> torch.Tensor:
        return torch.arange(self.num_cubes, device=self.device, dtype=self.index_dtype)

    def cube_to_ijk(self, cube_idx: torch.Tensor) -> torch.Tensor:
        return self.unravel_idx(cube_idx, (self.res,) * 3)

    def ijk_to_cube(self, ijk: torch.Tensor) -> torch.Tensor:
        return self.ravel_ijk(ijk, (self.res,) * 3)

    def cube_aabb(self, cube_idx: torch.Tensor):
        mins = self.vertex_to_world(self.cube_to_ijk(cube_idx))
        return mins, mins + self.cell_size

    def cube_center(self, cube_idx: torch.Tensor) -> torch.Tensor:
        return self.grid_to_world(self.cube_to_ijk(cube_idx))

    def cube_corner_vertex_indices(self, cube_idx: torch.Tensor) -> torch.Tensor:
        ijk = self.cube_to_ijk(cube_idx)
        corners = ijk[:, None, :] + self.CUBE_CORNERS[None]
        p = self.num_vertices_per_axis
        return self.ravel_ijk(corners.reshape(-1, 3), (p, p, p)).view(-1, 8)

    def cube_corner_coords(self, cube_idx: torch.Tensor) -> torch.Tensor:
        ijk = self.cube_to_ijk(cube_idx)
        return self.vertex_to_world(ijk[:, None, :] + self.CUBE_CORNERS[None])

    def vertex_ijk_from_indices(self, vertex_idx: torch.Tensor) -> torch.Tensor:
        p = self.num_vertices_per_axis
        return self.unravel_idx(vertex_idx.flatten(), (p, p, p)).view(*vertex_idx.shape, 3)

    def vertex_coords_from_indices(self, vertex_idx: torch.Tensor) -> torch.Tensor:
        return self.vertex_to_world(self.vertex_ijk_from_indices(vertex_idx))

    def voxel_unique_vertices(self, voxels: torch.Tensor):
        """(unique vertex indices [M], their world coords [M,3], cube->vertex map [N,8])."""
        if voxels.dim() == 2 and voxels.shape[1] == 3:
            cube_idx = self.ijk_to_cube(voxels)
        elif voxels.dim() == 1:
            cube_idx = voxels
        else:
            raise ValueError(f"voxels must be [N,3] or [N], got {tuple(voxels.shape)}")
        corner = self.cube_corner_vertex_indices(cube_idx)
        uniq, inv = torch.unique(corner.flatten(), return_inverse=True)
        return uniq, self.vertex_coords_from_indices(uniq), inv.view(-1, 8)

    def generate_all_cells(self) -> torch.Tensor:
        x = torch.arange(self.res, device=self.device, dtype=self.index_dtype)
        xx, yy, zz = torch.meshgrid(x, x, x, indexing="ij")
        return torch.stack([xx.flatten(), yy.flatten(), zz.flatten()], dim=1)
