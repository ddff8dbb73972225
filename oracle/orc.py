"""Python side of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, as the checker.  The product package never does.

Wraps liboracle.so (oracle.c) with numpy arrays and restates, in numpy, the
host-side post-processing of the reference's flood fill:
  * flood_fill_3d_sparse          atom3d/kernels/flood_fill.py:118-258
  * get_dam_neighborhood_signs    atom3d/apps/sparse_flood_fill.py:34-100
  * sparse_flood_fill (dict)      atom3d/apps/sparse_flood_fill.py:103-166
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")

_lib = None


def build() -> str:
    src = os.path.join(HERE, "oracle.c")
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        os.makedirs(os.path.dirname(LIB), exist_ok=True)
        cmd = ["gcc", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-pthread", "-std=gnu11", "-shared",
               "-o", LIB, src, "-lm", "-lpthread"]
        subprocess.run(cmd, check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = ctypes.CDLL(LIB)
        _lib.orc_octree_traverse.restype = ctypes.c_int64
        _lib.orc_sat.restype = ctypes.c_int
        _lib.orc_get_threads.restype = ctypes.c_int
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def set_threads(n: int) -> None:
    lib().orc_set_threads(ctypes.c_int(n))


def threads() -> int:
    return int(lib().orc_get_threads())


I64 = ctypes.c_int64


def udf_exact(V, F, P):
    """FP64 brute force: (dist f64 [N], face id [N], closest f64 [N,3])."""
    V, F, P = _f32(V), _i32(F), _f32(P)
    n = P.shape[0]
    d = np.empty(n, np.float64)
    fid = np.empty(n, np.int32)
    cp = np.empty((n, 3), np.float64)
    lib().orc_udf_exact_f64(_p(V), _p(F), I64(F.shape[0]), _p(P), I64(n), _p(d), _p(fid), _p(cp))
    return d, fid, cp


def tri_dist(V, F, P, fid):
    """FP64 distance from P[i] to face fid[i]."""
    V, F, P, fid = _f32(V), _i32(F), _f32(P), _i32(fid)
    out = np.empty(P.shape[0], np.float64)
    lib().orc_tri_dist_f64(_p(V), _p(F), _p(P), _p(fid), I64(P.shape[0]), _p(out))
    return out


def ref_udf_bruteforce(V, F, P):
    """Reference FP32 triangle maths over all faces: (dist, fid, cp, uvw)."""
    V, F, P = _f32(V), _i32(F), _f32(P)
    n = P.shape[0]
    d = np.empty(n, np.float32)
    fid = np.empty(n, np.int32)
    cp = np.empty((n, 3), np.float32)
    uvw = np.empty((n, 3), np.float32)
    lib().orc_ref_udf_bruteforce(_p(V), _p(F), I64(F.shape[0]), _p(P), I64(n), _p(d), _p(fid), _p(cp), _p(uvw))
    return d, fid, cp, uvw


def ref_bvh_udf(nodes, tris, P):
    """bvh_udf_kernel restated over a reference build_bvh tree."""
    nodes, tris, P = _f32(nodes), _f32(tris), _f32(P)
    n = P.shape[0]
    d = np.empty(n, np.float32)
    fid = np.empty(n, np.int32)
    cp = np.empty((n, 3), np.float32)
    uvw = np.zeros((n, 3), np.float32)
    lib().orc_ref_bvh_udf(_p(nodes), _p(tris), _p(P), I64(n), _p(d), _p(fid), _p(cp), _p(uvw))
    return d, fid, cp, uvw


def sat(tri9, mn, mx) -> bool:
    t, a, b = _f32(tri9), _f32(mn), _f32(mx)
    return bool(lib().orc_sat(_p(t), _p(a), _p(b)))


def boxes_hit(V, F, bmin, bmax):
    V, F, bmin, bmax = _f32(V), _i32(F), _f32(bmin), _f32(bmax)
    h = np.empty(bmin.shape[0], np.uint8)
    lib().orc_boxes_hit(_p(V), _p(F), I64(F.shape[0]), _p(bmin), _p(bmax), I64(bmin.shape[0]), _p(h))
    return h.astype(bool)


def boxes_hit_exact_box(V, F, bmin, bmax):
    """Per box: some triangle whose own box overlaps it exactly passes SAT."""
    V, F, bmin, bmax = _f32(V), _i32(F), _f32(bmin), _f32(bmax)
    h = np.empty(bmin.shape[0], np.uint8)
    lib().orc_boxes_hit_exact_box(_p(V), _p(F), I64(F.shape[0]), _p(bmin), _p(bmax), I64(bmin.shape[0]), _p(h))
    return h.astype(bool)


def ref_octree_traverse(nodes, tris, lo, hi, min_level, max_level):
    """octree_traverse with bvh_aabb_intersect_kernel restated over a reference
    build_bvh tree as the per-level test (tree-dependent, like the reference)."""
    cells = level_cells(lo, hi, max_level)
    lo32 = _f32(lo)
    corners = np.array([[i & 1, (i >> 1) & 1, (i >> 2) & 1] for i in range(8)], np.int64)

    def boxes(ijk, lv):
        mn = (ijk.astype(np.float32) * cells[lv] + lo32).astype(np.float32)
        return mn, (mn + cells[lv]).astype(np.float32)

    r = 1 << min_level
    x = np.arange(r, dtype=np.int64)
    cur = np.stack(np.meshgrid(x, x, x, indexing="ij"), -1).reshape(-1, 3)
    cur = cur[ref_bvh_aabb_hit(nodes, tris, *boxes(cur, min_level))]
    for lv in range(min_level + 1, max_level + 1):
        if cur.shape[0] == 0:
            break
        cur = ((cur * 2)[:, None, :] + corners[None]).reshape(-1, 3)
        cur = cur[ref_bvh_aabb_hit(nodes, tris, *boxes(cur, lv))]
    return cur


def ref_bvh_aabb_hit(nodes, tris, bmin, bmax):
    nodes, tris, bmin, bmax = _f32(nodes), _f32(tris), _f32(bmin), _f32(bmax)
    h = np.empty(bmin.shape[0], np.uint8)
    lib().orc_ref_bvh_aabb_hit(_p(nodes), _p(tris), _p(bmin), _p(bmax), I64(bmin.shape[0]), _p(h))
    return h.astype(bool)


def level_cells(lo, hi, max_level):
    """float32 (hi - lo) / 2^level per level, like the reference's tensors."""
    lo = np.asarray(lo, np.float32)
    hi = np.asarray(hi, np.float32)
    ext = (hi - lo).astype(np.float32)
    return np.stack([(ext / np.float32(2 ** lv)).astype(np.float32) for lv in range(max_level + 1)])


def octree_traverse(V, F, lo, hi, min_level, max_level, cap=None):
    V, F = _f32(V), _i32(F)
    lo = _f32(lo)
    cells = _f32(level_cells(lo, hi, max_level))
    cap = cap or (1 << 22)
    while True:
        out = np.empty((cap, 3), np.int64)
        k = lib().orc_octree_traverse(_p(V), _p(F), I64(F.shape[0]), _p(lo), _p(cells), ctypes.c_int(min_level),
                                      ctypes.c_int(max_level), _p(out), I64(cap))
        if k < 0:
            cap = -k
            continue
        return out[:k]


def morton_encode(ijk):
    a = np.ascontiguousarray(np.asarray(ijk, dtype=np.int64))
    out = np.empty(a.shape[0], np.int64)
    lib().orc_morton_encode(_p(a), I64(a.shape[0]), _p(out))
    return out


def flood_fill_dense(occ: np.ndarray, seed, connectivity: int = 26) -> np.ndarray:
    """Labels of the BFS over a dense [D,H,W] crop (seed in array index order)."""
    occ = np.ascontiguousarray(occ.astype(np.uint8))
    D, H, W = occ.shape
    mask = np.empty(occ.shape, np.int32)
    s0, s1, s2 = (int(x) for x in seed)
    lib().orc_flood_fill(_p(occ), D, H, W, s2, s1, s0, connectivity, _p(mask))
    return mask


def _dilate(m: np.ndarray, conn: int) -> np.ndarray:
    """Binary dilation with the 6-cross (conn 6) or full 3x3x3 box (else)."""
    out = m.copy()
    D, H, W = m.shape
    pad = np.zeros((D + 2, H + 2, W + 2), bool)
    pad[1:-1, 1:-1, 1:-1] = m
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                if conn == 6 and abs(dx) + abs(dy) + abs(dz) != 1:
                    continue
                out |= pad[1 + dz:1 + dz + D, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W]
    return out


def flood_fill_3d_sparse(dam, resolution, source=(0, 0, 0), padding=2, connectivity=26):
    """numpy restatement of flood_fill_3d_sparse; returns the same 6-tuple."""
    dam = np.asarray(dam, np.int64).reshape(-1, 3)
    empty3 = np.zeros((0, 3), np.int32)
    if dam.shape[0] == 0:
        return empty3, empty3, empty3, empty3, np.zeros(0, bool), empty3
    bmin = np.maximum(dam.min(0) - padding, 0)
    bmax = np.minimum(dam.max(0) + padding, resolution - 1)
    size = bmax - bmin + 1
    occ = np.zeros(tuple(size), bool)
    loc = dam - bmin
    occ[loc[:, 0], loc[:, 1], loc[:, 2]] = True
    ls = np.asarray(source, np.int64) - bmin
    if (ls >= 0).all() and (ls < size).all():
        if occ[tuple(ls)]:
            return empty3, empty3, empty3, empty3, np.zeros(0, bool), empty3
        seed = ls
    else:
        seed = np.zeros(3, np.int64)
        if occ[0, 0, 0]:
            return empty3, empty3, empty3, empty3, np.zeros(0, bool), empty3
    mask = flood_fill_dense(occ, seed, connectivity)
    flooded = mask > 0
    dil = _dilate(flooded, 6 if connectivity == 6 else 26)
    ext = (mask == -2) & occ & dil
    mask[ext] = -1

    def coords(m):
        c = np.argwhere(m).astype(np.int32)
        return (c + bmin.astype(np.int32)) if c.shape[0] else empty3

    water = coords(mask == 2)
    dry = coords(mask == -2)
    coll = coords(mask == 1)
    tdam = coords(mask == -1)
    extd = coords(ext)
    dam_mask = mask[loc[:, 0], loc[:, 1], loc[:, 2]] == -1
    return water, dry, coll, tdam, dam_mask, extd


def dam_neighborhood_signs(dam, water, dry, resolution, k_ring=1):
    """numpy restatement of get_dam_neighborhood_signs."""
    dam = np.asarray(dam, np.int64).reshape(-1, 3)
    if dam.shape[0] == 0:
        return np.zeros((0, 3), np.int32), np.zeros(0, np.int8)
    offs = np.array([[dx, dy, dz] for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)
                     if (dx, dy, dz) != (0, 0, 0)], np.int64)
    front = dam
    allv = dam
    for ring in range(k_ring):
        nb = (front[:, None, :] + offs[None]).reshape(-1, 3)
        nb = nb[((nb >= 0) & (nb < resolution)).all(1)]
        allv = np.unique(np.concatenate([allv, nb], 0), axis=0)
        if ring < k_ring - 1:
            front = allv
    R = resolution
    lin = (allv[:, 0] * R + allv[:, 1]) * R + allv[:, 2]

    def member(s):
        s = np.asarray(s, np.int64).reshape(-1, 3)
        if s.shape[0] == 0:
            return np.zeros(lin.shape[0], bool)
        sl = np.sort((s[:, 0] * R + s[:, 1]) * R + s[:, 2])
        i = np.clip(np.searchsorted(sl, lin), 0, sl.shape[0] - 1)
        return sl[i] == lin

    signs = np.ones(lin.shape[0], np.int8)
    signs[member(dry)] = -1
    signs[member(water)] = 1
    signs[member(dam)] = 0
    return allv.astype(np.int32), signs


def sparse_flood_fill_from_dam(dam, resolution, source=(0, 0, 0), connectivity=26, k_ring=1):
    """The dict of sparse_flood_fill given its octree output ``dam``."""
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


def ref_bvh_udf_counts(nodes, tris, P):
    """(node box evaluations, triangle evaluations) of bvh_udf_kernel over a
    reference tree, summed over the queries."""
    nodes, tris, P = _f32(nodes), _f32(tris), _f32(P)
    c = np.zeros(2, np.int64)
    lib().orc_ref_bvh_udf_counts(_p(nodes), _p(tris), _p(P), I64(P.shape[0]), _p(c))
    return int(c[0]), int(c[1])


# --------------------------------------------------------------------- rays
def ray_nearest(V, F, O, D, max_t=1e10):
    """Brute-force nearest hit (reference ray maths): hit, t, face, point, uvw."""
    V, F, O, D = _f32(V), _i32(F), _f32(O), _f32(D)
    n = O.shape[0]
    hit = np.empty(n, np.uint8)
    t = np.empty(n, np.float32)
    fid = np.empty(n, np.int32)
    hp = np.empty((n, 3), np.float32)
    uvw = np.empty((n, 3), np.float32)
    lib().orc_ray_nearest(_p(V), _p(F), I64(F.shape[0]), _p(O), _p(D), I64(n), ctypes.c_float(max_t), _p(hit),
                          _p(t), _p(fid), _p(hp), _p(uvw))
    return hit.astype(bool), t, fid, hp, uvw


def ray_all(V, F, O, D, max_t=1e10, cap=256):
    """Every non-grazing hit per ray (face order): list of (t, face, sign) arrays."""
    V, F, O, D = _f32(V), _i32(F), _f32(O), _f32(D)
    n = O.shape[0]
    counts = np.empty(n, np.int32)
    t = np.empty((n, cap), np.float32)
    fid = np.empty((n, cap), np.int32)
    sign = np.empty((n, cap), np.int32)
    lib().orc_ray_all(_p(V), _p(F), I64(F.shape[0]), _p(O), _p(D), I64(n), ctypes.c_float(max_t), I64(cap),
                      _p(counts), _p(t), _p(fid), _p(sign))
    out = []
    for i in range(n):
        k = min(int(counts[i]), cap)
        out.append((t[i, :k].copy(), fid[i, :k].copy(), sign[i, :k].copy()))
    return counts, out


def parity_votes(V, F, P, dirs, max_t=1e6, coalesce=1e-4):
    """Per point, number of directions whose coalesced signed crossing count is odd."""
    V, F, P, dirs = _f32(V), _i32(F), _f32(P), _f32(dirs)
    votes = np.empty(P.shape[0], np.int32)
    lib().orc_parity_votes(_p(V), _p(F), I64(F.shape[0]), _p(P), I64(P.shape[0]), _p(dirs), ctypes.c_int(dirs.shape[0]),
                           ctypes.c_float(max_t), ctypes.c_float(coalesce), _p(votes))
    return votes


# ------------------------------------------------------------ box/mesh pairs
def clip_pair(bmin, bmax, tri9, eps=1e-8):
    """One triangle clipped against one box: (hit, count, verts [8,3], centroid, area)."""
    mn, mx, t = _f32(bmin).reshape(3), _f32(bmax).reshape(3), _f32(tri9).reshape(9)
    verts = np.zeros(24, np.float32)
    cen = np.zeros(3, np.float32)
    cnt = ctypes.c_int(0)
    area = ctypes.c_float(0)
    hit = lib().orc_clip_pair(_p(mn), _p(mx), _p(t), ctypes.c_float(eps), _p(verts), ctypes.byref(cnt), _p(cen),
                              ctypes.byref(area))
    return bool(hit), cnt.value, verts.reshape(8, 3), cen, np.float32(area.value)


def aabb_pairs(V, F, bmin, bmax, mode=1, eps=1e-8):
    """MeshBVH.intersect_aabb by brute force: dict with hit [N] and, per
    (box, face) pair in box then face order, aabb_ids / face_ids (int64) and
    for modes 2-3 poly_counts, centroids, areas (+ poly_verts for mode 3)."""
    V, F, bmin, bmax = _f32(V), _i32(F), _f32(bmin), _f32(bmax)
    n, nf = bmin.shape[0], F.shape[0]
    clip = 1 if mode >= 2 else 0
    counts = np.zeros(n, np.int64)
    lib().orc_aabb_pair_counts(_p(V), _p(F), I64(nf), _p(bmin), _p(bmax), I64(n), ctypes.c_int(clip),
                               ctypes.c_float(eps), _p(counts))
    offs = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=offs[1:])
    P = int(offs[-1])
    out = dict(hit=counts > 0, aabb_ids=np.zeros(P, np.int64), face_ids=np.zeros(P, np.int64))
    pc = np.zeros(P, np.int32)
    cen = np.zeros((P, 3), np.float32)
    ar = np.zeros(P, np.float32)
    pv = np.zeros((P, 8, 3), np.float32) if mode == 3 else None
    lib().orc_aabb_pairs_fill(_p(V), _p(F), I64(nf), _p(bmin), _p(bmax), I64(n), ctypes.c_int(clip),
                              ctypes.c_float(eps), _p(offs), _p(out["aabb_ids"]), _p(out["face_ids"]), _p(pc), _p(cen),
                              _p(ar), _p(pv) if pv is not None else None)
    if mode >= 2:
        out.update(poly_counts=pc, centroids=cen, areas=ar)
    if mode == 3:
        out["poly_verts"] = pv
    return out


def clip_counts(bmin, bmax, tri9, eps=1e-8):
    """Clipped polygon vertex count for each row (box k, triangle k)."""
    mn, mx, t = _f32(bmin).reshape(-1, 3), _f32(bmax).reshape(-1, 3), _f32(tri9).reshape(-1, 9)
    out = np.empty(mn.shape[0], np.int32)
    lib().orc_clip_batch(_p(mn), _p(mx), _p(t), I64(mn.shape[0]), ctypes.c_float(eps), _p(out))
    return out
