"""Sparse flood fill and the surface dual graph (drop-in for
atom3d/apps/sparse_flood_fill.py:34-291 and atom3d/kernels/flood_fill.py:
118-258).

sparse_flood_fill: octree SAT descent for the dam voxels, then the native
bit-volume flood fill and k-ring classification (a3d_flood_*).  Output
dictionary, dtypes (int32 [K,3]) and ordering (lexicographic (x, y, z), like
torch.nonzero / torch.unique(dim=0)) are the reference's.

construct_surface_dual_graph and get_dam_wet_faces / _edges / _corners run
on bit volumes over the cells' bounding box (a3d_dual_graph_*, a3d_dam_wet):
no sort, no dense resolution^3 mask.
"""

from __future__ import annotations

import ctypes
import logging
import math
from typing import Dict, Optional, Tuple

import torch

from .. import _lib
from ..constants import SIGN_DRY, SIGN_WATER
from ..grid.octree_indexer import OctreeIndexer

logger = logging.getLogger(__name__)

WATER, DRY, TIDE, DAM, EXT_DAM, EXT_TIDE, DRY_ADJ = range(7)


class FloodGeom(ctypes.Structure):
    _fields_ = [
        ("vol_lo", ctypes.c_int64 * 3),
        ("vol_dims", ctypes.c_int32 * 3),
        ("crop_lo", ctypes.c_int64 * 3),
        ("crop_hi", ctypes.c_int64 * 3),
        ("seed", ctypes.c_int64 * 3),
        ("connectivity", ctypes.c_int32),
        ("k_ring", ctypes.c_int32),
    ]


class DualGeom(ctypes.Structure):
    _fields_ = [("lo", ctypes.c_int64 * 3), ("hi", ctypes.c_int64 * 3), ("resolution", ctypes.c_int64)]


_SIGS = {
    "a3d_flood_bbox": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p,
                                      ctypes.c_size_t, ctypes.c_void_p]),
    "a3d_flood_workspace_bytes": (ctypes.c_size_t, [ctypes.POINTER(FloodGeom)]),
    "a3d_flood_fill": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(FloodGeom), ctypes.c_void_p,
                                      ctypes.c_size_t, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int),
                                      ctypes.c_void_p]),
    "a3d_flood_extract": (ctypes.c_int, [ctypes.POINTER(FloodGeom), ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]),
    "a3d_flood_test": (ctypes.c_int, [ctypes.POINTER(FloodGeom), ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int,
                                      ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]),
    "a3d_ring_signs": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                                      ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(FloodGeom), ctypes.c_void_p,
                                      ctypes.c_size_t, ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p]),
    "a3d_ring_signs_emit": (ctypes.c_int, [ctypes.POINTER(FloodGeom), ctypes.c_void_p, ctypes.c_size_t,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]),
    "a3d_cells_bbox": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_int64), ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p, ctypes.c_size_t,
                                      ctypes.c_void_p]),
    "a3d_dual_workspace_bytes": (ctypes.c_size_t, [ctypes.POINTER(DualGeom)]),
    "a3d_dual_graph_count": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_int64),
                                            ctypes.c_int, ctypes.POINTER(DualGeom), ctypes.c_void_p,
                                            ctypes.c_size_t, ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p]),
    "a3d_dual_graph_emit": (ctypes.c_int, [ctypes.POINTER(DualGeom), ctypes.c_void_p, ctypes.c_size_t,
                                           ctypes.c_int64, ctypes.c_int64, ctypes.POINTER(ctypes.c_float),
                                           ctypes.POINTER(ctypes.c_float), ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "a3d_dam_wet_workspace_bytes": (ctypes.c_size_t, [ctypes.POINTER(ctypes.c_int64)]),
    "a3d_dam_wet": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                                   ctypes.POINTER(ctypes.c_int64), ctypes.c_int64, ctypes.c_void_p, ctypes.c_size_t,
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
}


def _bind():
    lib = _lib.lib()
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


class _Flood:
    """Native flood fill over the dam voxels' padded bounding box."""

    def __init__(self, dam: torch.Tensor, resolution: int, source, padding: int, connectivity: int, k_ring: int):
        lib = _bind()
        _lib.require_cuda(dam, "dam voxels")
        self.dev = dam.device
        self.stream = _lib.stream_ptr(self.dev)
        d = dam.to(torch.int64).contiguous()
        self.n = int(d.shape[0])
        self.counts = [0] * 9
        self.empty = self.n == 0
        if self.empty:
            return
        ws0 = _lib.workspace(64, self.dev)
        bb = (ctypes.c_int64 * 6)()
        _lib.check("a3d_flood_bbox", lib.a3d_flood_bbox(d.data_ptr(), self.n, bb, ws0.data_ptr(), ws0.numel(),
                                                        self.stream))
        R = int(resolution)
        clo = [max(bb[a] - padding, 0) for a in range(3)]
        chi = [min(bb[3 + a] + padding, R - 1) for a in range(3)]
        extra = max(0, int(k_ring) - int(padding))
        vlo = [max(clo[a] - extra, 0) for a in range(3)]
        vhi = [min(chi[a] + extra, R - 1) for a in range(3)]
        src = [int(x) for x in source]
        inside = all(clo[a] <= src[a] <= chi[a] for a in range(3))
        seed = src if inside else clo  # local (0, 0, 0) when the source is outside the crop
        g = FloodGeom()
        for a in range(3):
            g.vol_lo[a] = vlo[a]
            g.vol_dims[a] = vhi[a] - vlo[a] + 1
            g.crop_lo[a] = clo[a]
            g.crop_hi[a] = chi[a]
            g.seed[a] = seed[a]
        g.connectivity = int(connectivity)
        g.k_ring = int(k_ring)
        self.geom = g
        self.crop_lo = clo
        self.ws = _lib.workspace(lib.a3d_flood_workspace_bytes(ctypes.byref(g)), self.dev)
        counts = (ctypes.c_int64 * 9)()
        rounds = ctypes.c_int(0)
        _lib.check("a3d_flood_fill", lib.a3d_flood_fill(d.data_ptr(), self.n, ctypes.byref(g), self.ws.data_ptr(),
                                                        self.ws.numel(), counts, ctypes.byref(rounds), self.stream))
        self.counts = list(counts)
        self.rounds = rounds.value
        self.seed_occupied = bool(counts[8])
        if self.seed_occupied:
            where = "Start point" if inside else "Default start (0,0,0)"
            print(f"[Flood Fill Warning] {where} {tuple(src) if inside else ''} is OCCUPIED. Returning empty result.")
            self.empty = True
        self._dam = d

    def extract(self, label: int) -> torch.Tensor:
        if self.empty:
            return torch.empty(0, 3, dtype=torch.int32, device=self.dev)
        k = int(self.counts[label])
        out = torch.empty(k, 3, dtype=torch.int32, device=self.dev)
        if k:
            _lib.check("a3d_flood_extract", _bind().a3d_flood_extract(
                ctypes.byref(self.geom), self.ws.data_ptr(), self.ws.numel(), label, out.data_ptr(), k, self.stream))
        return out

    def test(self, label: int, ijk: torch.Tensor) -> torch.Tensor:
        x = ijk.to(torch.int64).contiguous()
        out = torch.zeros(x.shape[0], dtype=torch.bool, device=self.dev)
        if self.empty or x.shape[0] == 0:
            return out
        _lib.check("a3d_flood_test", _bind().a3d_flood_test(
            ctypes.byref(self.geom), self.ws.data_ptr(), self.ws.numel(), label, x.data_ptr(), x.shape[0],
            out.data_ptr(), self.stream))
        return out


def _empty3(device):
    return torch.empty(0, 3, dtype=torch.int32, device=device)


def flood_fill_3d_sparse(
    dam_coords: torch.Tensor,
    resolution: int,
    source: Tuple[int, int, int] = (0, 0, 0),
    padding: int = 2,
    connectivity: int = 26,
    return_water_dry: bool = True,
):
    """(water, dry, collision, true_dam, dam_mask, extended_dam), int32 [K,3]
    each plus a bool [N] mask (reference: atom3d/kernels/flood_fill.py:118)."""
    dev = dam_coords.device
    fl = _Flood(dam_coords, resolution, source, padding, connectivity, 0)
    if fl.empty:
        return _empty3(dev), _empty3(dev), _empty3(dev), _empty3(dev), torch.empty(0, dtype=torch.bool, device=dev), \
            _empty3(dev)
    water = fl.extract(WATER) if return_water_dry else _empty3(dev)
    dry = fl.extract(DRY) if return_water_dry else _empty3(dev)
    return water, dry, fl.extract(TIDE), fl.extract(DAM), fl.test(DAM, dam_coords), fl.extract(EXT_DAM)


def get_dam_neighborhood_signs(
    dam_ijk: torch.Tensor,
    water_ijk: torch.Tensor,
    dry_ijk: torch.Tensor,
    resolution: int,
    k_ring: int = 1,
) -> Tuple[torch.Tensor, torch.Tensor]:
    """k-ring neighbourhood of the dam cells and its signs (reference:
    atom3d/apps/sparse_flood_fill.py:34-100).

    Returns (neighbor_ijk int32 [K,3], signs int8 [K]): the dam grown by
    ``k_ring`` 26-neighbourhood rings inside [0, resolution)^3, unique and in
    lexicographic order, with sign 0 for dam cells, else +1 (SIGN_WATER) for
    water cells, else -1 (SIGN_DRY) for dry cells, else +1.  With k_ring = 0
    the dam list comes back as given (every sign 0), like the reference's
    empty expansion loop.  Runs on bit volumes over the dam's bounding box
    (a3d_ring_signs); dam cells must lie in [0, resolution).
    """
    dev = dam_ijk.device
    if len(dam_ijk) == 0:
        return torch.empty(0, 3, dtype=torch.int32, device=dev), torch.empty(0, dtype=torch.int8, device=dev)
    k_ring = int(k_ring)
    if k_ring < 0:
        raise ValueError(f"k_ring must be >= 0, got {k_ring}")
    if k_ring == 0:
        return dam_ijk.int(), torch.zeros(dam_ijk.shape[0], dtype=torch.int8, device=dev)
    lib = _bind()
    _lib.require_cuda(dam_ijk, "dam_ijk")
    R = int(resolution)

    def lst(t, what):
        if t is None or len(t) == 0:
            return torch.empty(0, 3, dtype=torch.int64, device=dev)
        if t.dim() != 2 or t.shape[1] != 3:
            raise ValueError(f"{what} must be [K,3], got {tuple(t.shape)}")
        return t.to(device=dev, dtype=torch.int64).contiguous()

    dam, water, dry = lst(dam_ijk, "dam_ijk"), lst(water_ijk, "water_ijk"), lst(dry_ijk, "dry_ijk")
    stream = _lib.stream_ptr(dev)
    ws0 = _lib.workspace(64, dev)
    bb = (ctypes.c_int64 * 6)()
    _lib.check("a3d_flood_bbox", lib.a3d_flood_bbox(dam.data_ptr(), dam.shape[0], bb, ws0.data_ptr(), ws0.numel(),
                                                    stream))
    if min(bb[:3]) < 0 or max(bb[3:]) >= R:
        raise ValueError(f"dam_ijk: coordinates must lie in [0, {R}), got range {list(bb[:3])}..{list(bb[3:])}")
    g = FloodGeom()
    for a in range(3):
        lo, hi = max(bb[a] - k_ring, 0), min(bb[3 + a] + k_ring, R - 1)
        g.vol_lo[a] = g.crop_lo[a] = g.seed[a] = lo
        g.crop_hi[a] = hi
        g.vol_dims[a] = hi - lo + 1
    g.connectivity = 26
    g.k_ring = k_ring
    ws = _lib.workspace(lib.a3d_flood_workspace_bytes(ctypes.byref(g)), dev)
    count = ctypes.c_int64(0)
    _lib.check("a3d_ring_signs", lib.a3d_ring_signs(
        dam.data_ptr(), dam.shape[0], water.data_ptr(), water.shape[0], dry.data_ptr(), dry.shape[0], ctypes.byref(g),
        ws.data_ptr(), ws.numel(), ctypes.byref(count), stream))
    k = int(count.value)
    ijk = torch.empty(k, 3, dtype=torch.int32, device=dev)
    signs = torch.empty(k, dtype=torch.int8, device=dev)
    _lib.check("a3d_ring_signs_emit", lib.a3d_ring_signs_emit(ctypes.byref(g), ws.data_ptr(), ws.numel(),
                                                              ijk.data_ptr(), signs.data_ptr(), k, stream))
    return ijk, signs


def sparse_flood_fill(
    bvh,
    resolution: int,
    source: Tuple[int, int, int] = (0, 0, 0),
    connectivity: int = 26,
    min_level: int = 0,
    k_ring: int = 1,
    bounds: Optional[torch.Tensor] = None,
    verbose: bool = True,
) -> Dict[str, torch.Tensor]:
    """Inside/outside classification of a mesh at ``resolution``^3 voxels.

    Same arguments and returned keys as the reference
    (atom3d/apps/sparse_flood_fill.py:103-166): dam_ijk, water_ijk, dry_ijk,
    tide_ijk, extended_tide_ijk, dry_adjacent_ijk (int32 [K,3]).
    """
    dev = bvh.device
    max_level = int(math.log2(resolution))
    octree = OctreeIndexer(max_level=max_level, bounds=bounds, device=dev)
    dam = octree.octree_traverse(bvh, min_level=min_level)
    fl = _Flood(dam, resolution, source, 10, connectivity, k_ring)
    if fl.empty:
        e = _empty3(dev)
        return {"dam_ijk": e, "water_ijk": e.clone(), "dry_ijk": e.clone(), "tide_ijk": e.clone(),
                "extended_tide_ijk": e.clone(), "dry_adjacent_ijk": e.clone()}
    out = {
        "dam_ijk": fl.extract(DAM),
        "water_ijk": fl.extract(WATER),
        "dry_ijk": fl.extract(DRY),
        "tide_ijk": fl.extract(TIDE),
        "extended_tide_ijk": fl.extract(EXT_TIDE),
        "dry_adjacent_ijk": fl.extract(DRY_ADJ),
    }
    if verbose:
        logger.info("Sparse flood fill: %d dam voxels, %d relaxation rounds", out["dam_ijk"].shape[0], fl.rounds)
    return out


# ---------------------------------------------------------------------------
# surface dual graph and dam wet masks
# ---------------------------------------------------------------------------
def _cells32(t: torch.Tensor, what: str) -> torch.Tensor:
    _lib.require_cuda(t, what)
    if t.dim() != 2 or t.shape[1] != 3:
        raise ValueError(f"{what} must be [K,3], got {tuple(t.shape)}")
    return t.to(torch.int32).contiguous()


def _bbox(lib, cells, dev):
    """(lo, hi) over the lists, None when all are empty (synchronises)."""
    ptrs = (ctypes.c_void_p * len(cells))(*[c.data_ptr() for c in cells])
    cnts = (ctypes.c_int64 * len(cells))(*[c.shape[0] for c in cells])
    bb = (ctypes.c_int64 * 6)()
    ws = _lib.workspace(64, dev)
    _lib.check("a3d_cells_bbox", lib.a3d_cells_bbox(ptrs, cnts, len(cells), bb, ws.data_ptr(), ws.numel(),
                                                    _lib.stream_ptr(dev)))
    if bb[0] > bb[3]:
        return None
    return list(bb[:3]), list(bb[3:])


def _check_range(box, resolution, what):
    lo, hi = box
    if min(lo) < 0 or max(hi) >= resolution:
        raise ValueError(f"{what}: coordinates must lie in [0, {resolution}), got range {lo}..{hi}")


def _dam_wet(dam_ijk, collision_ijk, resolution, which):
    dev = dam_ijk.device
    width = {"faces": 6, "edges": 12, "corners": 8}[which]
    if len(dam_ijk) == 0:
        return torch.zeros((0, width), dtype=torch.bool, device=dev)
    lib = _bind()
    dam = _cells32(dam_ijk, "dam_ijk")
    out = torch.empty((dam.shape[0], width), dtype=torch.bool, device=dev)
    coll = _cells32(collision_ijk, "collision_ijk") if len(collision_ijk) else torch.empty(0, 3, dtype=torch.int32,
                                                                                           device=dev)
    box = _bbox(lib, [coll], dev) if coll.shape[0] else None
    bb = (ctypes.c_int64 * 6)()
    if box is not None:
        _check_range(box, resolution, "collision_ijk")
        for a in range(3):
            bb[a], bb[3 + a] = box[0][a], box[1][a]
    ws = _lib.workspace(lib.a3d_dam_wet_workspace_bytes(bb) if box is not None else 256, dev)
    ptr = {k: (out.data_ptr() if k == which else None) for k in ("faces", "edges", "corners")}
    _lib.check("a3d_dam_wet", lib.a3d_dam_wet(dam.data_ptr(), dam.shape[0], coll.data_ptr(), coll.shape[0], bb,
                                              int(resolution), ws.data_ptr(), ws.numel(), ptr["faces"],
                                              ptr["edges"], ptr["corners"], _lib.stream_ptr(dev)))
    return out


def get_dam_wet_faces(dam_ijk: torch.Tensor, collision_ijk: torch.Tensor, resolution: int) -> torch.Tensor:
    """bool [N,6]: the face neighbour (+x,-x,+y,-y,+z,-z) of each dam cell is a
    collision cell (atom3d/apps/sparse_flood_fill.py:169-185)."""
    return _dam_wet(dam_ijk, collision_ijk, resolution, "faces")


def get_dam_wet_edges(dam_ijk: torch.Tensor, collision_ijk: torch.Tensor, resolution: int) -> torch.Tensor:
    """bool [N,12]: one of the 3 cells sharing each edge is a collision cell
    (atom3d/apps/sparse_flood_fill.py:188-204; EDGE_NEIGHBOR_OFFSETS)."""
    return _dam_wet(dam_ijk, collision_ijk, resolution, "edges")


def get_dam_wet_corners(dam_ijk: torch.Tensor, collision_ijk: torch.Tensor, resolution: int) -> torch.Tensor:
    """bool [N,8]: one of the 7 cells sharing each corner is a collision cell
    (atom3d/apps/sparse_flood_fill.py:207-223; CORNER_NEIGHBOR_OFFSETS)."""
    return _dam_wet(dam_ijk, collision_ijk, resolution, "corners")


def construct_surface_dual_graph(
    dam_ijk: torch.Tensor,
    collision_ijk: torch.Tensor,
    dry_adjacent_ijk: Optional[torch.Tensor],
    octree: OctreeIndexer,
) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor]:
    """Topology of the active cells (dam, collision and dry-adjacent union).

    Returns, like atom3d/apps/sparse_flood_fill.py:226-291:
      voxelgrid_vertices float32 [V,3]  octree.bounds[0] + vertices_ijk * cell
      vertices_ijk       int64 [V,3]    unique cube corners, lexicographic
      cube_idx           int64 [N,8]    corners of each cell (CUBE_CORNERS order)
      adj_idx            int64 [N,6]    face neighbours (+x,-x,+y,-y,+z,-z) or -1
      active_cells_ijk   [N,3]          unique cells, lexicographic; the
                                        promoted dtype of the inputs
    Cells must lie in [0, 2^max_level).
    """
    lists = [c for c in (dam_ijk, collision_ijk, dry_adjacent_ijk) if c is not None and len(c) > 0]
    if not lists:
        raise RuntimeError("construct_surface_dual_graph: no active cells (all inputs are empty)")
    dev = lists[0].device
    out_dtype = lists[0].dtype
    for c in lists[1:]:
        out_dtype = torch.promote_types(out_dtype, c.dtype)
    lib = _bind()
    cells = [_cells32(c, "cell list") for c in lists]
    R = 2 ** int(octree.max_level)
    box = _bbox(lib, cells, dev)
    _check_range(box, R, "construct_surface_dual_graph")
    g = DualGeom()
    for a in range(3):
        g.lo[a], g.hi[a] = box[0][a], box[1][a]
    g.resolution = R
    ws = _lib.workspace(lib.a3d_dual_workspace_bytes(ctypes.byref(g)), dev)
    stream = _lib.stream_ptr(dev)
    ptrs = (ctypes.c_void_p * len(cells))(*[c.data_ptr() for c in cells])
    cnts = (ctypes.c_int64 * len(cells))(*[c.shape[0] for c in cells])
    nv = (ctypes.c_int64 * 2)()
    _lib.check("a3d_dual_graph_count", lib.a3d_dual_graph_count(ptrs, cnts, len(cells), ctypes.byref(g),
                                                                ws.data_ptr(), ws.numel(), nv, stream))
    n, v = int(nv[0]), int(nv[1])
    # the reference's float32 (hi - lo) / R and lo, as host floats
    b = octree.bounds.to(torch.float32)
    cmin = b[0].tolist()
    cell = ((b[1] - b[0]) / float(R)).tolist()
    cells_ijk = torch.empty((n, 3), dtype=torch.int32, device=dev)
    vijk = torch.empty((v, 3), dtype=torch.int64, device=dev)
    world = torch.empty((v, 3), dtype=torch.float32, device=dev)
    cube_idx = torch.empty((n, 8), dtype=torch.int64, device=dev)
    adj_idx = torch.empty((n, 6), dtype=torch.int64, device=dev)
    _lib.check("a3d_dual_graph_emit", lib.a3d_dual_graph_emit(
        ctypes.byref(g), ws.data_ptr(), ws.numel(), n, v, (ctypes.c_float * 3)(*cmin), (ctypes.c_float * 3)(*cell),
        cells_ijk.data_ptr(), vijk.data_ptr(), world.data_ptr(), cube_idx.data_ptr(), adj_idx.data_ptr(), stream))
    if out_dtype != torch.int32:
        cells_ijk = cells_ijk.to(out_dtype)
    return world, vijk, cube_idx, adj_idx, cells_ijk


__all__ = ["sparse_flood_fill", "flood_fill_3d_sparse", "get_dam_wet_faces", "get_dam_wet_edges",
           "get_dam_wet_corners", "construct_surface_dual_graph", "SIGN_WATER", "SIGN_DRY"]
