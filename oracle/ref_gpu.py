"""The reference's own CUDA kernels, driven on the GPU (TEST INFRASTRUCTURE ONLY).

Only tests/ and bench.py's reference arm use this module, as the checker and
as the reference's GPU timing; the product package never does.

Loads the pybind modules that ``oracle/build_ref.py`` compiles from the
reference sources into ``oracle/_ref/`` (``bvh_cuda``: build_bvh, bvh_udf,
bvh_aabb_intersect; ``floodfill_cuda``: flood_fill) and restates the thin
PyTorch glue the reference wraps around them, line for line in behaviour:

  * RefBVH                 atom3d/kernels/bvh.py:67-90 (BVHAccelerator, leaf 4),
                           udf at :92-113, aabb_intersect through
                           atom3d/core/mesh_bvh.py:339-360 (mode 0)
  * octree_traverse        atom3d/grid/octree_indexer.py:470-509 with
                           all_cubes_at_level :426-439, subdivide :191-216,
                           cube_aabb_level :302-337 and the per-level cell
                           sizes of :51-55
  * flood_fill_3d_sparse   atom3d/kernels/flood_fill.py:118-258 and
                           flood_fill_3d :75-116
  * dam_neighborhood_signs atom3d/apps/sparse_flood_fill.py:34-100
  * sparse_flood_fill      atom3d/apps/sparse_flood_fill.py:103-166

The kernels themselves are the reference's, compiled with its flags
(``-O3 --use_fast_math``), so SAT decisions, closest faces and flood labels
are the reference implementation's own on this GPU.
"""

from __future__ import annotations

import importlib.util
import math
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_mods: dict = {}

# CUBE_CORNERS order of the reference (atom3d/constants.py): bit 0 -> x,
# bit 1 -> y, bit 2 -> z.
_CORNERS = [[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0], [0, 0, 1], [1, 0, 1], [0, 1, 1], [1, 1, 1]]


def so_path(name: str) -> str:
    return os.path.join(REF_DIR, name, name + ".so")


def available() -> bool:
    return all(os.path.exists(so_path(n)) for n in ("bvh_cuda", "floodfill_cuda"))


def module(name: str):
    """The compiled reference extension ``name`` (bvh_cuda / floodfill_cuda)."""
    if name not in _mods:
        path = so_path(name)
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is missing: run oracle/build_ref.py --reference <checkout>")
        import torch  # noqa: F401  (the extension links against torch's libraries)

        spec = importlib.util.spec_from_file_location(name, path)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        _mods[name] = mod
    return _mods[name]


class RefBVH:
    """The reference's BVHAccelerator: host SAH build, GPU queries."""

    def __init__(self, vertices: torch.Tensor, faces: torch.Tensor, leaf: int = 4):
        m = module("bvh_cuda")
        self.device = vertices.device
        self.vertices = vertices.contiguous().float()
        self.faces = faces.contiguous().int()
        self.nodes, self.triangles = m.build_bvh(self.vertices, self.faces, int(leaf))

    def udf(self, points: torch.Tensor):
        """(distances f32, face_ids int32, closest [K,3], uvw [K,3])."""
        return module("bvh_cuda").bvh_udf(self.nodes, self.triangles, points.contiguous().float())

    def aabb_hit(self, box_min: torch.Tensor, box_max: torch.Tensor) -> torch.Tensor:
        hit, _, _ = module("bvh_cuda").bvh_aabb_intersect(self.nodes, self.triangles, box_min.contiguous(),
                                                          box_max.contiguous())
        return hit


def level_cell_sizes(bounds: torch.Tensor, max_level: int):
    return [(bounds[1] - bounds[0]) / (2 ** lv) for lv in range(max_level + 1)]


def octree_traverse(bvh: RefBVH, bounds: torch.Tensor, min_level: int, max_level: int) -> torch.Tensor:
    """Candidate cubes at max_level, int64 [K,3], in the reference's order."""
    dev = bvh.device
    bounds = bounds.to(device=dev, dtype=torch.float32)
    cells = level_cell_sizes(bounds, max_level)
    corners = torch.tensor(_CORNERS, dtype=torch.int64, device=dev)

    def boxes(ijk, level):
        mn = ijk.float() * cells[level] + bounds[0]
        return mn, mn + cells[level]

    res = 2 ** min_level
    x = torch.arange(res, device=dev, dtype=torch.int64)
    xx, yy, zz = torch.meshgrid(x, x, x, indexing="ij")
    cur = torch.stack([xx.flatten(), yy.flatten(), zz.flatten()], dim=1)
    cur = cur[bvh.aabb_hit(*boxes(cur, min_level))]
    for level in range(min_level + 1, max_level + 1):
        if cur.numel() == 0:
            break
        cur = ((cur * 2)[:, None, :] + corners[None, :, :]).reshape(-1, 3)
        cur = cur[bvh.aabb_hit(*boxes(cur, level))]
    return cur


def flood_fill_3d(occupancy: torch.Tensor, start_point, connectivity: int = 26) -> torch.Tensor:
    z, y, x = start_point
    return module("floodfill_cuda").flood_fill(occupancy.contiguous(), x, y, z, connectivity)


def _empty(dev):
    e = torch.empty(0, 3, dtype=torch.int32, device=dev)
    return e, e.clone(), e.clone(), e.clone(), torch.empty(0, dtype=torch.bool, device=dev), e.clone()


def flood_fill_3d_sparse(dam: torch.Tensor, resolution: int, source=(0, 0, 0), padding: int = 2,
                         connectivity: int = 26):
    """(water, dry, collision, true_dam, dam_mask, extended_dam) as the reference returns them."""
    dev = dam.device
    if len(dam) == 0:
        return _empty(dev)
    bmin = torch.clamp(dam.min(dim=0)[0] - padding, min=0)
    bmax = torch.clamp(dam.max(dim=0)[0] + padding, max=resolution - 1)
    size = (bmax - bmin + 1).tolist()
    occ = torch.zeros(size, dtype=torch.bool, device=dev)
    loc = dam - bmin
    occ[loc[:, 0], loc[:, 1], loc[:, 2]] = True
    ls = torch.tensor(source, dtype=torch.int32, device=dev) - bmin
    if bool((ls >= 0).all()) and bool((ls < torch.tensor(size, device=dev)).all()):
        ls = ls.long()
        if bool(occ[ls[0], ls[1], ls[2]]):
            return _empty(dev)
        start = (int(ls[0]), int(ls[1]), int(ls[2]))
    else:
        start = (0, 0, 0)
        if bool(occ[0, 0, 0]):
            return _empty(dev)
    mask = flood_fill_3d(occ, start, connectivity)
    flooded = (mask > 0).float()[None, None]
    if connectivity == 6:
        k = torch.zeros(1, 1, 3, 3, 3, device=dev)
        for c in ((1, 1, 1), (0, 1, 1), (2, 1, 1), (1, 0, 1), (1, 2, 1), (1, 1, 0), (1, 1, 2)):
            k[0, 0, c[0], c[1], c[2]] = 1
        dil = torch.nn.functional.conv3d(flooded, k, padding=1)[0, 0] > 0.5
    else:
        dil = torch.nn.functional.max_pool3d(flooded, kernel_size=3, stride=1, padding=1)[0, 0] > 0.5
    del flooded
    ext = (mask == -2) & occ & dil
    del dil
    mask[ext] = -1
    b = bmin.int()

    def coords(m):
        c = torch.nonzero(m, as_tuple=False)
        return c.int() + b if len(c) > 0 else torch.empty(0, 3, dtype=torch.int32, device=dev)

    extd = coords(ext)
    del ext
    coll = coords(mask == 1)
    water = coords(mask == 2)
    dry = coords(mask == -2)
    tdam = coords(mask == -1)
    dam_mask = mask[loc[:, 0], loc[:, 1], loc[:, 2]] == -1
    return water, dry, coll, tdam, dam_mask, extd


def dam_neighborhood_signs(dam: torch.Tensor, water: torch.Tensor, dry: torch.Tensor, resolution: int,
                           k_ring: int = 1):
    """(neighbour ijk int32 [K,3], signs int8 [K]): 1 water, -1 dry, 0 dam."""
    dev = dam.device
    if len(dam) == 0:
        return torch.empty(0, 3, dtype=torch.int32, device=dev), torch.empty(0, dtype=torch.int8, device=dev)
    R = resolution
    offs = torch.tensor([[dx, dy, dz] for dx in (-1, 0, 1) for dy in (-1, 0, 1) for dz in (-1, 0, 1)
                         if (dx, dy, dz) != (0, 0, 0)], dtype=torch.int64, device=dev)
    front = dam.long()
    allv = dam.long()
    for ring in range(k_ring):
        nb = (front[:, None, :] + offs[None]).reshape(-1, 3)
        nb = nb[((nb >= 0) & (nb < R)).all(dim=1)]
        allv = torch.unique(torch.cat([allv, nb], 0), dim=0)
        if ring < k_ring - 1:
            front = allv
    lin = allv[:, 0] * R * R + allv[:, 1] * R + allv[:, 2]
    signs = torch.full((len(allv),), 1, dtype=torch.int8, device=dev)

    def member(s):
        if len(s) == 0:
            return torch.zeros(len(allv), dtype=torch.bool, device=dev)
        sl, _ = torch.sort(s[:, 0].long() * R * R + s[:, 1].long() * R + s[:, 2].long())
        i = torch.clamp(torch.searchsorted(sl, lin), 0, len(sl) - 1)
        return sl[i] == lin

    is_dam, is_water, is_dry = member(dam), member(water), member(dry)
    signs[is_dry] = -1
    signs[is_water] = 1
    signs[is_dam] = 0
    return allv.int(), signs


def sparse_flood_fill(bvh: RefBVH, resolution: int, bounds: torch.Tensor, source=(0, 0, 0),
                      connectivity: int = 26, min_level: int = 0, k_ring: int = 1):
    """The reference's sparse_flood_fill dict, with its own SAT and BFS kernels."""
    max_level = int(math.log2(resolution))
    dam = octree_traverse(bvh, bounds, min_level, max_level)
    water, dry, coll, tdam, _, _ = flood_fill_3d_sparse(dam, resolution, source, padding=10,
                                                        connectivity=connectivity)
    nb, signs = dam_neighborhood_signs(tdam, water, dry, resolution, k_ring)
    return {
        "dam_ijk": tdam,
        "water_ijk": water,
        "dry_ijk": dry,
        "tide_ijk": coll,
        "extended_tide_ijk": nb[signs == 1],
        "dry_adjacent_ijk": nb[signs == -1],
    }
