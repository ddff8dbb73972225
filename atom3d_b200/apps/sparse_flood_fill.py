"""Sparse flood fill (drop-in for atom3d/apps/sparse_flood_fill.py:34-166 and
atom3d/kernels/flood_fill.py:118-258).

sparse_flood_fill: octree SAT descent for the dam voxels, then the native
bit-volume flood fill and k-ring classification (a3d_flood_*).  Output
dictionary, dtypes (int32 [K,3]) and ordering (lexicographic (x, y, z), like
torch.nonzero / torch.unique(dim=0)) are the reference's.
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


__all__ = ["sparse_flood_fill", "flood_fill_3d_sparse", "SIGN_WATER", "SIGN_DRY"]
