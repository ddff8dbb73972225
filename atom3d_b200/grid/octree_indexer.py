"""OctreeIndexer: multi-level cube grid with the coarse-to-fine SAT descent
(drop-in for atom3d/grid/octree_indexer.py:17-509 except three Python-loop
helpers that are not ported: expand_nodes (:371-420), mark_active_nodes and
get_node_neighbors, none of them on the descent's path).

``octree_traverse`` runs the whole descent in one native call
(a3d_octree_traverse): per level, one SAT any-hit query per candidate cube
over the wide BVH, then a stable prefix-sum compaction, so the output order
is the reference's (meshgrid 'ij' at ``min_level``, parents in order, 8
children each in CUBE_CORNERS order).  Morton keys are computed by the
native a3d_morton_encode / a3d_morton_decode kernels.
"""

from __future__ import annotations

import ctypes
from typing import Optional, Tuple, Union

import torch

from .. import _lib
from .cube_grid import CubeGrid


class OctreeIndexer(CubeGrid):
    def __init__(self, max_level: int, bounds: Optional[torch.Tensor] = None,
                 device: Optional[Union[str, torch.device]] = None):
        self.max_level = max_level
        self._max_resolution = 2 ** max_level
        super().__init__(resolution=self._max_resolution, bounds=bounds, device=device)
        self._level_resolutions = [2 ** lv for lv in range(max_level + 1)]
        # float32 (hi - lo) / res, the reference's per-level cell size
        self._level_cell_sizes = [(self.bounds[1] - self.bounds[0]) / r for r in self._level_resolutions]
        self._descent_args = None

    def get_resolution(self, level: int) -> int:
        return self._level_resolutions[level]

    def get_cell_size(self, level: int) -> torch.Tensor:
        return self._level_cell_sizes[level]

    def get_num_cubes(self, level: int) -> int:
        return self.get_resolution(level) ** 3

    def world_to_grid_level(self, world_coords: torch.Tensor, level: int) -> torch.Tensor:
        return ((world_coords - self.bounds[0]) / self.get_cell_size(level)).floor().to(self.index_dtype)

    def grid_to_world_level(self, grid_coords: torch.Tensor, level: int) -> torch.Tensor:
        return (grid_coords.float() + 0.5) * self.get_cell_size(level) + self.bounds[0]

    def cube_aabb_level(self, cubes: torch.Tensor, level: Optional[int] = None) -> Tuple[torch.Tensor, torch.Tensor]:
        """AABBs of cubes given as [B, 3] ijk or [B] linear indices at `level`
        (default max_level)."""
        level = self.max_level if level is None else level
        if cubes.dim() == 1:
            cubes = self.cube_to_ijk_level(cubes, level)
        elif cubes.dim() != 2 or cubes.shape[1] != 3:
            raise ValueError(f"cubes must be [B, 3] ijk or [B] linear idx, got shape {cubes.shape}")
        cell = self.get_cell_size(level)
        mn = cubes.float() * cell + self.bounds[0]
        return mn, mn + cell

    def get_cell_aabb_level(self, grid_coords: torch.Tensor, level: int) -> Tuple[torch.Tensor, torch.Tensor]:
        """Cell AABB with the upper corner computed as (ijk + 1) * cell + lo,
        which can differ in the last bit from cube_aabb_level's min + cell."""
        cell = self.get_cell_size(level)
        return grid_coords.float() * cell + self.bounds[0], (grid_coords.float() + 1) * cell + self.bounds[0]

    def get_root_coords(self) -> torch.Tensor:
        return torch.zeros(1, 3, dtype=self.index_dtype, device=self.device)

    def cube_to_ijk_level(self, cube_idx: torch.Tensor, level: Optional[int] = None) -> torch.Tensor:
        r = self.get_resolution(self.max_level if level is None else level)
        return self.unravel_idx(cube_idx, (r, r, r))

    def ijk_to_cube_level(self, ijk: torch.Tensor, level: Optional[int] = None) -> torch.Tensor:
        r = self.get_resolution(self.max_level if level is None else level)
        return self.ravel_ijk(ijk, (r, r, r))

    def cube_corner_coords_level(self, cube_ijk: torch.Tensor, level: int) -> torch.Tensor:
        """World positions [B, 8, 3] of the cubes' corners in CUBE_CORNERS order."""
        corners = cube_ijk[:, None, :] + self.CUBE_CORNERS[None]
        return corners.float() * self.get_cell_size(level) + self.bounds[0]

    def cube_edge_endpoints_level(self, cube_ijk: torch.Tensor, level: int) -> torch.Tensor:
        """Endpoints [B, 12, 2, 3] of the cubes' edges in CUBE_EDGES order."""
        w = self.cube_corner_coords_level(cube_ijk, level)
        return torch.stack([w[:, self.CUBE_EDGES[:, 0]], w[:, self.CUBE_EDGES[:, 1]]], dim=2)

    def filter_active_cubes(self, cube_ijk: torch.Tensor, level: int, mesh_aabb_min: torch.Tensor,
                            mesh_aabb_max: torch.Tensor) -> torch.Tensor:
        """Cubes whose AABB overlaps some mesh AABB (closed intervals on every
        axis), in input order (reference: atom3d/grid/octree_indexer.py:
        441-468).  The cube x box test runs over chunks of cubes, so its
        temporary stays near 64M entries whatever the sizes."""
        cmin, cmax = self.cube_aabb_level(cube_ijk, level)
        amin = mesh_aabb_min.to(device=cmin.device, dtype=cmin.dtype)
        amax = mesh_aabb_max.to(device=cmin.device, dtype=cmin.dtype)
        n = int(cube_ijk.shape[0])
        keep = torch.zeros(n, dtype=torch.bool, device=cmin.device)
        step = max(1, (1 << 26) // max(3 * int(amin.shape[0]), 1))
        for s in range(0, n, step):
            e = min(n, s + step)
            ov = (cmin[s:e, None, :] <= amax[None]) & (cmax[s:e, None, :] >= amin[None])
            keep[s:e] = ov.all(dim=2).any(dim=1)
        return cube_ijk[keep]

    # ---------------------------------------------------------------- Morton
    def _ijk_to_morton(self, ijk: torch.Tensor) -> torch.Tensor:
        _lib.require_cuda(ijk, "ijk")
        x = ijk.to(torch.int64).contiguous()
        out = torch.empty(x.shape[0], dtype=torch.int64, device=x.device)
        _lib.call("a3d_morton_encode", x.data_ptr(), x.shape[0], out.data_ptr(), _lib.stream_ptr(x.device))
        return out

    def _morton_to_ijk(self, morton: torch.Tensor, level: int) -> torch.Tensor:
        _lib.require_cuda(morton, "morton")
        m = morton.to(torch.int64).contiguous()
        out = torch.empty(m.shape[0], 3, dtype=torch.int64, device=m.device)
        _lib.call("a3d_morton_decode", m.data_ptr(), m.shape[0], int(level), out.data_ptr(), _lib.stream_ptr(m.device))
        return out

    def linear_to_morton(self, linear_idx: torch.Tensor, level: int) -> torch.Tensor:
        r = self.get_resolution(level)
        return self._ijk_to_morton(self.unravel_idx(linear_idx, (r, r, r)))

    def morton_to_linear(self, morton: torch.Tensor, level: int) -> torch.Tensor:
        r = self.get_resolution(level)
        return self.ravel_ijk(self._morton_to_ijk(morton, level), (r, r, r))

    # ------------------------------------------------------- level transitions
    def subdivide(self, parent_coords: torch.Tensor, parent_level: int) -> torch.Tensor:
        ch = parent_coords[:, None, :] * 2 + self.CUBE_CORNERS.to(parent_coords.device)[None]
        return ch.reshape(-1, 3).to(self.index_dtype)

    def merge(self, child_coords: torch.Tensor, child_level: int) -> torch.Tensor:
        return torch.div(child_coords, 2, rounding_mode="floor")

    def all_cubes_at_level(self, level: int) -> torch.Tensor:
        r = self.get_resolution(level)
        x = torch.arange(r, device=self.device, dtype=self.index_dtype)
        xx, yy, zz = torch.meshgrid(x, x, x, indexing="ij")
        return torch.stack([xx.flatten(), yy.flatten(), zz.flatten()], dim=1)

    # -------------------------------------------------------------- traversal
    def _host_descent_args(self):
        """Grid origin and per-level cell sizes as C float arrays, read back
        with one device-to-host copy per indexer (both are fixed when the
        indexer is built)."""
        if self._descent_args is None:
            parts = [self.bounds[0].detach().float().reshape(3)]
            parts += [c.detach().float().reshape(3) for c in self._level_cell_sizes]
            v = torch.cat(parts).cpu().tolist()
            self._descent_args = ((ctypes.c_float * 3)(*v[:3]), (ctypes.c_float * (len(v) - 3))(*v[3:]))
        return self._descent_args

    def octree_traverse(self, bvh, min_level: int = 2) -> torch.Tensor:
        """Active cubes [K, 3] int64 at max_level, coarse-to-fine from min_level."""
        dev = bvh.device
        lo_c, cell_c = self._host_descent_args()
        cap = max(1 << (3 * min_level), 6 * (4 ** self.max_level), 1024)
        for _ in range(6):
            out = torch.empty(cap, 3, dtype=torch.int64, device=dev)
            ws = _lib.workspace(_lib.lib().a3d_octree_workspace_bytes(min_level, self.max_level, cap), dev)
            count = ctypes.c_int64(0)
            st = _lib.lib().a3d_octree_traverse(
                ctypes.byref(bvh._bvh.view), lo_c, cell_c, int(min_level), int(self.max_level), out.data_ptr(), cap,
                ctypes.byref(count), ws.data_ptr(), ws.numel(), _lib.stream_ptr(dev),
            )
            if st == _lib.A3D_ERR_WORKSPACE:
                need = int(count.value)
                cap = need if need > cap else cap * 4
                continue
            _lib.check("a3d_octree_traverse", st)
            return out[: int(count.value)]
        raise RuntimeError("octree_traverse: could not size the candidate buffers")
