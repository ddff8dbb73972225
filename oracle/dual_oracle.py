"""numpy restatement of construct_surface_dual_graph and get_dam_wet_faces /
_edges / _corners.  TEST INFRASTRUCTURE ONLY.

Follows atom3d/apps/sparse_flood_fill.py:
  get_dam_wet_faces             :169-185
  get_dam_wet_edges             :188-204
  get_dam_wet_corners           :207-223
  construct_surface_dual_graph  :226-291
and the neighbour tables of atom3d/constants.py:50-110.

The graph is restated with numpy's sorted unique rows and binary search on
the same linear keys as the reference: cells key (x*R + y)*R + z with
R = 2^max_level (so a neighbour off the y or z face of the grid finds the
cell its key wraps to, like the reference), vertices key with R + 1.
World positions are float32 origin + ijk * cell, a product then a sum.
"""

from __future__ import annotations

import numpy as np

CUBE_CORNERS = np.array([[i & 1, (i >> 1) & 1, (i >> 2) & 1] for i in range(8)], np.int64)
NEIGHBOR_OFFSETS_6 = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], np.int64)


def edge_neighbor_offsets():
    """[12, 3, 3]: edge e (x-, y-, then z-aligned, 4 each); perpendicular
    axes p < q get signs from bits 0 and 1 of e % 4 (constants.py:74-93)."""
    out = np.zeros((12, 3, 3), np.int64)
    for e in range(12):
        axis, k = divmod(e, 4)
        p, q = [a for a in range(3) if a != axis]
        out[e, 0, p] = -1 if k & 1 else 1
        out[e, 1, q] = -1 if k & 2 else 1
        out[e, 2] = out[e, 0] + out[e, 1]
    return out


def corner_neighbor_offsets():
    """[8, 7, 3] (constants.py:96-105)."""
    out = np.zeros((8, 7, 3), np.int64)
    for c in range(8):
        sx, sy, sz = (2 * CUBE_CORNERS[c] - 1).tolist()
        out[c] = [[sx, 0, 0], [0, sy, 0], [0, 0, sz], [sx, sy, 0], [sx, 0, sz], [0, sy, sz], [sx, sy, sz]]
    return out


def _keys(ijk, r):
    ijk = np.asarray(ijk, np.int64)
    return (ijk[..., 0] * r + ijk[..., 1]) * r + ijk[..., 2]


def _wet(dam, collision, resolution, offsets):
    dam = np.asarray(dam, np.int64).reshape(-1, 3)
    shape = (dam.shape[0],) + offsets.shape[:-1]
    if dam.shape[0] == 0:
        return np.zeros(shape, bool)
    coll = np.unique(_keys(np.asarray(collision, np.int64).reshape(-1, 3), resolution))
    nb = dam[:, None, :] + offsets.reshape(1, -1, 3)
    inb = ((nb >= 0) & (nb < resolution)).all(-1)
    return (inb & np.isin(_keys(nb, resolution), coll)).reshape(shape)


def dam_wet_faces(dam, collision, resolution):
    """bool [N,6] (sparse_flood_fill.py:169-185)."""
    return _wet(dam, collision, resolution, NEIGHBOR_OFFSETS_6)


def dam_wet_edges(dam, collision, resolution):
    """bool [N,12]: any of the 3 edge neighbours (sparse_flood_fill.py:188-204)."""
    return _wet(dam, collision, resolution, edge_neighbor_offsets()).any(-1)


def dam_wet_corners(dam, collision, resolution):
    """bool [N,8]: any of the 7 corner neighbours (sparse_flood_fill.py:207-223)."""
    return _wet(dam, collision, resolution, corner_neighbor_offsets()).any(-1)


def dual_graph(dam, collision, dry_adjacent, max_level, bounds):
    """(voxelgrid_vertices f32 [V,3], vertices_ijk int64 [V,3], cube_idx int64
    [N,8], adj_idx int64 [N,6], active_cells_ijk [N,3]) as
    construct_surface_dual_graph (sparse_flood_fill.py:226-291)."""
    lists = [np.asarray(c).reshape(-1, 3) for c in (dam, collision, dry_adjacent) if c is not None and len(c)]
    R = 2 ** int(max_level)
    cells = np.unique(np.concatenate(lists, 0), axis=0)
    n = cells.shape[0]
    ck = _keys(cells, R)  # ascending: cells are sorted rows in [0, R)
    cand = cells.astype(np.int64)[:, None, :] + CUBE_CORNERS[None]
    verts = np.unique(cand.reshape(-1, 3), axis=0)
    vk = _keys(verts, R + 1)
    cube_idx = np.full((n, 8), -1, np.int64)
    if n:
        q = _keys(cand, R + 1).reshape(-1)
        pos = np.clip(np.searchsorted(vk, q), 0, len(vk) - 1)
        found = vk[pos] == q
        cube_idx.reshape(-1)[found] = pos[found]
    adj = np.full((n, 6), -1, np.int64)
    if n:
        q = _keys(cells.astype(np.int64)[:, None, :] + NEIGHBOR_OFFSETS_6[None], R).reshape(-1)
        pos = np.clip(np.searchsorted(ck, q), 0, n - 1)
        found = ck[pos] == q
        adj.reshape(-1)[found] = pos[found]
    b = np.asarray(bounds, np.float32).reshape(2, 3)
    cell = (b[1] - b[0]) / np.float32(R)
    world = b[0] + verts.astype(np.float32) * cell
    return world.astype(np.float32), verts, cube_idx, adj, cells
