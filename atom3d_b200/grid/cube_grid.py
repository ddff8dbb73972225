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
        # Global edge and face numbering (the reference's, cube_grid.py:126-155):
        # edges along x are numbered over dims (r, p, p), then those along y
        # over (p, r, p), then z over (p, p, r); faces normal to x over
        # (p, r, r), then y over (r, p, r), then z over (r, r, p); r = res,
        # p = res + 1.  Axis a's dims are p except r along a itself.
        r, p = self.res, self.num_vertices_per_axis
        self._axis_dims = [tuple(r if b == a else p for b in range(3)) for a in range(3)]
        self._face_dims = [tuple(p if b == a else r for b in range(3)) for a in range(3)]
        self._num_edges_x, self._num_edges_y, self._num_edges_z = (r * p * p,) * 3
        self._edge_offset_x, self._edge_offset_y, self._edge_offset_z = 0, r * p * p, 2 * r * p * p
        self.num_edges = 3 * r * p * p
        self._num_faces_x, self._num_faces_y, self._num_faces_z = (p * r * r,) * 3
        self._face_offset_x, self._face_offset_y, self._face_offset_z = 0, p * r * r, 2 * p * r * r
        self.num_faces = 3 * p * r * r
        ends = self.CUBE_CORNERS[self.CUBE_EDGES]  # [12, 2, 3]
        self._edge_axis = (ends[:, 1] - ends[:, 0]).abs().argmax(dim=1)
        self._edge_anchor_local = torch.minimum(ends[:, 0], ends[:, 1])

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

    # ---------------------------------------------------------------- edges
    def _axis_strides(self, dims_of_axis, axis: torch.Tensor) -> torch.Tensor:
        """Per-element (stride_i, stride_j) of the linear index over the
        axis-dependent dims (i * d1 + j) * d2 + k."""
        tab = torch.tensor([[d[1] * d[2], d[2]] for d in dims_of_axis], dtype=self.index_dtype, device=self.device)
        return tab[axis]

    def cube_edge_indices(self, cube_idx: Optional[torch.Tensor]) -> torch.Tensor:
        """[B,12] global edge index of each local edge of each cube
        (reference: atom3d/grid/cube_grid.py:281-318)."""
        if cube_idx is None:
            cube_idx = self.all_cube_indices()
        ijk = self.cube_to_ijk(cube_idx)
        anchor = ijk[:, None, :] + self._edge_anchor_local.to(self.index_dtype)[None]  # [B,12,3]
        st = self._axis_strides(self._axis_dims, self._edge_axis)  # [12,2]
        offs = torch.tensor([self._edge_offset_x, self._edge_offset_y, self._edge_offset_z], dtype=self.index_dtype,
                            device=self.device)[self._edge_axis]
        return anchor[..., 0] * st[:, 0] + anchor[..., 1] * st[:, 1] + anchor[..., 2] + offs

    def voxel_unique_edges(self, voxels: torch.Tensor) -> Tuple[torch.Tensor, torch.Tensor]:
        """(unique edge indices [E], cube -> edge map [N,12]) of the given
        cubes ([N,3] ijk or [N] linear; reference: cube_grid.py:266-279)."""
        if voxels.dim() == 2 and voxels.shape[1] == 3:
            cube_idx = self.ijk_to_cube(voxels)
        elif voxels.dim() == 1:
            cube_idx = voxels
        else:
            raise ValueError(f"voxels must be [N,3] or [N], got {tuple(voxels.shape)}")
        e = self.cube_edge_indices(cube_idx)
        uniq, inv = torch.unique(e.flatten(), return_inverse=True)
        return uniq, inv.view(e.shape[0], 12)

    def _edge_axis_of(self, edge_idx: torch.Tensor) -> torch.Tensor:
        # the reference's masks: x below the y offset, y below the z offset,
        # everything else counts as z
        return (edge_idx >= self._edge_offset_y).to(self.index_dtype) + (edge_idx >= self._edge_offset_z).to(
            self.index_dtype)

    def _edge_anchor_ijk(self, edge_idx: torch.Tensor, axis: torch.Tensor) -> torch.Tensor:
        offs = torch.tensor([self._edge_offset_x, self._edge_offset_y, self._edge_offset_z], dtype=self.index_dtype,
                            device=self.device)[axis]
        local = edge_idx - offs
        st = self._axis_strides(self._axis_dims, axis)
        i = torch.div(local, st[:, 0], rounding_mode="floor")
        rem = local - i * st[:, 0]
        j = torch.div(rem, st[:, 1], rounding_mode="floor")
        return torch.stack([i, j, rem - j * st[:, 1]], dim=-1)

    def edge_endpoints(self, edge_idx: torch.Tensor) -> torch.Tensor:
        """[E,2,3] world coordinates of both ends of each global edge, the
        lower end first (reference: cube_grid.py:320-360)."""
        edge_idx = edge_idx.to(self.device, dtype=self.index_dtype).flatten()
        axis = self._edge_axis_of(edge_idx)
        v0 = self._edge_anchor_ijk(edge_idx, axis)
        v1 = v0 + torch.nn.functional.one_hot(axis, 3).to(self.index_dtype)
        return torch.stack([self.vertex_to_world(v0), self.vertex_to_world(v1)], dim=1)

    def cube_face_indices(self, cube_idx: torch.Tensor) -> torch.Tensor:
        """[B,6] global face indices, ordered -z, +z, -x, +x, -y, +y
        (reference: cube_grid.py:366-381)."""
        ijk = self.cube_to_ijk(cube_idx)
        out = []
        for axis, off in ((2, self._face_offset_z), (0, self._face_offset_x), (1, self._face_offset_y)):
            for step in (0, 1):
                c = ijk.clone()
                c[:, axis] += step
                out.append(self.ravel_ijk(c, self._face_dims[axis]) + off)
        return torch.stack(out, dim=1)

    # right-handed counter-clockwise loop of the 4 cubes around an edge seen
    # along its +axis direction, as offsets from the edge's anchor vertex
    # (reference: cube_grid.py:387-520)
    _INCIDENT = (
        ((0, 0, 0), (0, 0, -1), (0, -1, -1), (0, -1, 0)),     # x edges, loop in (y, z)
        ((-1, 0, 0), (-1, 0, -1), (0, 0, -1), (0, 0, 0)),     # y edges, loop in (x, z)
        ((-1, 0, 0), (0, 0, 0), (0, -1, 0), (-1, -1, 0)),     # z edges, loop in (x, y)
    )

    def edge_incident_cubes(self, edge_idx: torch.Tensor,
                            edge_directions: Optional[torch.Tensor] = None) -> torch.Tensor:
        """[E,4] linear indices of the up to 4 cubes around each edge, a CCW
        loop about the edge's +axis direction (-1 outside the grid);
        ``edge_directions`` < 0 reverses an edge's loop."""
        edge_idx = edge_idx.to(device=self.device, dtype=self.index_dtype).flatten()
        E = edge_idx.numel()
        axis = self._edge_axis_of(edge_idx)
        anchor = self._edge_anchor_ijk(edge_idx, axis)
        loop = torch.tensor(self._INCIDENT, dtype=self.index_dtype, device=self.device)[axis]  # [E,4,3]
        cubes = anchor[:, None, :] + loop
        r = self.res
        valid = ((cubes >= 0) & (cubes < r)).all(dim=-1)
        lin = self.ijk_to_cube(cubes.view(-1, 3)).view(-1, 4)
        out = torch.where(valid, lin, torch.full_like(lin, -1))
        if edge_directions is not None:
            edge_directions = edge_directions.to(self.device).flatten()
            if edge_directions.numel() != E:
                raise ValueError(
                    f"edge_directions must have same length as edge_idx ({E}), got {edge_directions.numel()}")
            rev = edge_directions < 0
            out = torch.where(rev[:, None], out.flip(dims=[1]), out)
        return out
