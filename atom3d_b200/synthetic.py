"""Seeded synthetic workloads (meshes, queries, SDF grids).

No public dataset is involved; every input of the tests and benchmarks is
generated here from a fixed seed:

* ``icosphere(level)`` — icosahedron refined ``level`` times by edge
  midpoints pushed to the unit sphere: 10*4^level+2 vertices,
  20*4^level faces, outward (counter-clockwise) winding.
* ``udf_small`` — level 5, radius scaled per vertex by 1+N(0, 0.01);
  100,000 queries uniform in [-1.5, 1.5]^3.
* ``octree_mesh`` — level 7, r = 1 + 0.05 * sum_k<8 sin(f_k (d_k . x) + phi_k)
  with f_k ~ U[2, 8], d_k uniform on the sphere, phi_k ~ U[0, 2 pi).
* ``udf_large`` — level 8, same displacement with 16 terms; queries: half
  area-weighted surface samples + N(0, 0.02) per axis, half uniform in the
  mesh box scaled by 1.2 about its centre.
* ``batch_meshes`` — meshes of level U{3..8} (log-uniform triangle count)
  under random affine maps (scale U[0.5, 2], random rotation, translation
  U[-1, 1]^3); 8 queries per triangle.
* ``dmc_spheres`` — SDF = min_i(|x - c_i| - r_i) over 32 spheres
  (c ~ U[-0.7, 0.7]^3, r ~ U[0.05, 0.2]) + N(0, 1e-3), sampled at the
  unique corners of the cubes of a [-1, 1]^3 grid whose centre satisfies
  |sdf| <= 2h + sqrt(3)/2 h (h = 2 / res).
* ``shell_cells`` — flood-fill-like cell sets of a sphere of radius
  0.3 res about a jittered centre: dam = cells whose centre lies within 0.9
  of the sphere, collision = the next shell outside (0.9..1.9), dry
  adjacent = the next shell inside; plus cells on the grid's faces and
  duplicates across the lists.
"""

from __future__ import annotations

import math

import torch

# ---------------------------------------------------------------------------
# meshes
# ---------------------------------------------------------------------------


def _icosahedron() -> tuple[torch.Tensor, torch.Tensor]:
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = torch.tensor(
        [
            [-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
            [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
            [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1],
        ],
        dtype=torch.float64,
    )
    f = torch.tensor(
        [
            [0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
            [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
            [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
            [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1],
        ],
        dtype=torch.int64,
    )
    return v / v.norm(dim=1, keepdim=True), f


def icosphere(level: int) -> tuple[torch.Tensor, torch.Tensor]:
    """Unit icosphere as (float32 [V,3], int32 [F,3]) on the CPU."""
    v, f = _icosahedron()
    for _ in range(level):
        nv = v.shape[0]
        e = torch.cat([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], dim=0)  # [3F,2]
        lo = torch.minimum(e[:, 0], e[:, 1])
        hi = torch.maximum(e[:, 0], e[:, 1])
        key = lo * nv + hi
        uk, inv = torch.unique(key, return_inverse=True)
        mid = (v[uk // nv] + v[uk % nv]) * 0.5
        mid = mid / mid.norm(dim=1, keepdim=True)
        m = inv.view(3, -1) + nv  # midpoints of edges 01, 12, 20 per face
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        m01, m12, m20 = m[0], m[1], m[2]
        f = torch.cat(
            [
                torch.stack([a, m01, m20], 1),
                torch.stack([b, m12, m01], 1),
                torch.stack([c, m20, m12], 1),
                torch.stack([m01, m12, m20], 1),
            ],
            dim=0,
        )
        v = torch.cat([v, mid], dim=0)
    return v.float(), f.int()


def _sinusoid_radius(v: torch.Tensor, n_terms: int, amp: float, g: torch.Generator) -> torch.Tensor:
    freq = torch.rand(n_terms, generator=g, dtype=torch.float64) * 6.0 + 2.0
    d = torch.randn(n_terms, 3, generator=g, dtype=torch.float64)
    d = d / d.norm(dim=1, keepdim=True)
    phase = torch.rand(n_terms, generator=g, dtype=torch.float64) * (2 * math.pi)
    x = v.double() / v.double().norm(dim=1, keepdim=True)
    s = torch.sin(freq[None, :] * (x @ d.T) + phase[None, :]).sum(dim=1)
    return 1.0 + amp * s


def displaced_sphere(level: int, n_terms: int, amp: float, seed: int) -> tuple[torch.Tensor, torch.Tensor]:
    v, f = icosphere(level)
    g = torch.Generator().manual_seed(seed)
    r = _sinusoid_radius(v, n_terms, amp, g)
    return (v.double() * r[:, None]).float(), f


def udf_small(seed: int = 1, n_queries: int = 100_000):
    """Level-5 sphere with N(0, 0.01) radial noise and uniform queries."""
    v, f = icosphere(5)
    g = torch.Generator().manual_seed(seed)
    r = 1.0 + 0.01 * torch.randn(v.shape[0], generator=g, dtype=torch.float64)
    v = (v.double() * r[:, None]).float()
    q = (torch.rand(n_queries, 3, generator=g, dtype=torch.float64) * 3.0 - 1.5).float()
    return v, f, q


def octree_mesh(seed: int = 2, level: int = 7):
    return displaced_sphere(level, 8, 0.05, seed)


def surface_samples(v: torch.Tensor, f: torch.Tensor, n: int, g: torch.Generator) -> torch.Tensor:
    """Area-weighted uniform samples on the triangles (float64)."""
    vd = v.double()
    a, b, c = vd[f[:, 0].long()], vd[f[:, 1].long()], vd[f[:, 2].long()]
    area = torch.linalg.cross(b - a, c - a).norm(dim=1)
    idx = torch.multinomial(area, n, replacement=True, generator=g)
    r1 = torch.rand(n, generator=g, dtype=torch.float64, device=vd.device)
    r2 = torch.rand(n, generator=g, dtype=torch.float64, device=vd.device)
    s = r1.sqrt()
    w0, w1, w2 = 1 - s, s * (1 - r2), s * r2
    return w0[:, None] * a[idx] + w1[:, None] * b[idx] + w2[:, None] * c[idx]


def mixed_queries(v: torch.Tensor, f: torch.Tensor, n: int, g: torch.Generator, sigma: float = 0.02,
                  box_scale: float = 1.2) -> torch.Tensor:
    """Half near-surface (surface sample + N(0, sigma)), half uniform in the
    box scaled by ``box_scale`` about its centre."""
    n_s = n // 2
    n_u = n - n_s
    dev = v.device
    near = surface_samples(v, f, n_s, g) + sigma * torch.randn(n_s, 3, generator=g, dtype=torch.float64, device=dev)
    lo, hi = v.double().min(0).values, v.double().max(0).values
    c, h = (lo + hi) * 0.5, (hi - lo) * 0.5 * box_scale
    uni = c + (torch.rand(n_u, 3, generator=g, dtype=torch.float64, device=dev) * 2.0 - 1.0) * h
    return torch.cat([near, uni], 0).float()


def udf_large(seed: int = 3, level: int = 8, n_queries: int = 16 * 1024 * 1024):
    v, f = displaced_sphere(level, 16, 0.05, seed)
    g = torch.Generator().manual_seed(seed + 1000)
    q = mixed_queries(v, f, n_queries, g)
    return v, f, q


def _random_rotation(g: torch.Generator) -> torch.Tensor:
    q = torch.randn(4, generator=g, dtype=torch.float64)
    q = q / q.norm()
    w, x, y, z = q.tolist()
    return torch.tensor(
        [
            [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
            [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
            [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
        ],
        dtype=torch.float64,
    )


def batch_specs(n_meshes: int = 256, seed: int = 4, min_level: int = 3, max_level: int = 8):
    """Per-mesh parameters of the batched workload: subdivision level drawn
    uniformly from [min_level, max_level] (log-uniform triangle counts),
    displacement seed, scale U[0.5, 2], rotation from a normalised
    quaternion, translation U[-1, 1]^3, query seed."""
    g = torch.Generator().manual_seed(seed)
    specs = []
    for i in range(n_meshes):
        level = int(torch.randint(min_level, max_level + 1, (1,), generator=g))
        scale = float(torch.rand(1, generator=g, dtype=torch.float64)) * 1.5 + 0.5
        rot = _random_rotation(g)
        trans = torch.rand(3, generator=g, dtype=torch.float64) * 2.0 - 1.0
        specs.append({"level": level, "disp_seed": seed * 1000 + i, "scale": scale, "rot": rot, "trans": trans,
                      "query_seed": seed * 100000 + i})
    return specs


_ICO_CACHE: dict = {}


def _icosphere_cached(level: int):
    if level not in _ICO_CACHE:
        _ICO_CACHE[level] = icosphere(level)
    return _ICO_CACHE[level]


def batch_meshes(n_meshes: int = 256, seed: int = 4, min_level: int = 3, max_level: int = 8,
                 queries_per_tri: int = 8, device="cpu"):
    """List of (vertices, faces, queries) generated on ``device``: each mesh
    is a level-L icosphere radially displaced by 8 seeded sinusoids of
    amplitude 0.05, then scaled, rotated and translated; its queries
    (queries_per_tri per triangle) follow ``mixed_queries``."""
    out = []
    dev = torch.device(device)
    for sp in batch_specs(n_meshes, seed, min_level, max_level):
        v0, f = _icosphere_cached(sp["level"])
        g = torch.Generator().manual_seed(sp["disp_seed"])
        freq = torch.rand(8, generator=g, dtype=torch.float64) * 6.0 + 2.0
        d = torch.randn(8, 3, generator=g, dtype=torch.float64)
        d = d / d.norm(dim=1, keepdim=True)
        phase = torch.rand(8, generator=g, dtype=torch.float64) * (2 * math.pi)
        vd = v0.to(dev).double()
        x = vd / vd.norm(dim=1, keepdim=True)
        r = 1.0 + 0.05 * torch.sin(freq.to(dev)[None, :] * (x @ d.to(dev).T) + phase.to(dev)[None, :]).sum(dim=1)
        v = (vd * r[:, None]).float().double()
        vw = (v @ sp["rot"].to(dev).T) * sp["scale"] + sp["trans"].to(dev)
        fd = f.to(dev)
        gq = torch.Generator(device=dev).manual_seed(sp["query_seed"])
        q = mixed_queries(vw.float(), fd, queries_per_tri * f.shape[0], gq)
        out.append((vw.float(), fd, q))
    return out


# ---------------------------------------------------------------------------
# SDF grids for the DMC extractor
# ---------------------------------------------------------------------------


def spheres_sdf(x: torch.Tensor, centres: torch.Tensor, radii: torch.Tensor) -> torch.Tensor:
    d = torch.cdist(x.double(), centres.double()) - radii.double()[None, :]
    return d.min(dim=1).values


def dmc_spheres(res: int = 512, seed: int = 5, n_spheres: int = 32, noise: float = 1e-3, device: str = "cpu"):
    """Active cubes near the zero set of a union of spheres.

    Returns (voxel_coords int64 [N,3], sdf float32 [M], cube_idx int64 [N,8],
    unique_vertex_ijk int64 [M,3]).  cube_idx follows the reference's
    CubeGrid.voxel_unique_vertices numbering (ascending linear vertex index).
    """
    g = torch.Generator().manual_seed(seed)
    centres = torch.rand(n_spheres, 3, generator=g, dtype=torch.float64) * 1.4 - 0.7
    radii = torch.rand(n_spheres, generator=g, dtype=torch.float64) * 0.15 + 0.05
    h = 2.0 / res
    band = 2 * h + 0.5 * math.sqrt(3.0) * h
    # coarse pass: only blocks of 8^3 cubes whose centre is near the surface
    blk = 8
    nb = res // blk
    bi = torch.stack(torch.meshgrid(*[torch.arange(nb)] * 3, indexing="ij"), -1).reshape(-1, 3)
    bc = (bi.double() + 0.5) * blk * h - 1.0
    bd = spheres_sdf(bc, centres, radii).abs()
    keep = bd <= band + 0.5 * math.sqrt(3.0) * blk * h
    bi = bi[keep]
    off = torch.stack(torch.meshgrid(*[torch.arange(blk)] * 3, indexing="ij"), -1).reshape(-1, 3)
    cand = (bi[:, None, :] * blk + off[None, :, :]).reshape(-1, 3)
    cc = (cand.double() + 0.5) * h - 1.0
    cd = torch.empty(cand.shape[0], dtype=torch.float64)
    step = 1 << 20
    for s in range(0, cand.shape[0], step):
        cd[s:s + step] = spheres_sdf(cc[s:s + step], centres, radii)
    vox = cand[cd.abs() <= band]
    # lexicographic (x, y, z) order of the cubes
    lin = (vox[:, 0] * res + vox[:, 1]) * res + vox[:, 2]
    vox = vox[torch.argsort(lin)]
    corners = torch.tensor([[i & 1, (i >> 1) & 1, (i >> 2) & 1] for i in range(8)], dtype=torch.int64)
    p = res + 1
    cidx = vox[:, None, :] + corners[None]
    vlin = (cidx[..., 0] * p + cidx[..., 1]) * p + cidx[..., 2]
    uv, inv = torch.unique(vlin.reshape(-1), return_inverse=True)
    vijk = torch.stack([uv // (p * p), (uv // p) % p, uv % p], -1)
    vx = vijk.double() * h - 1.0
    sdf = torch.empty(vx.shape[0], dtype=torch.float64)
    for s in range(0, vx.shape[0], step):
        sdf[s:s + step] = spheres_sdf(vx[s:s + step], centres, radii)
    sdf = sdf + noise * torch.randn(sdf.shape[0], generator=g, dtype=torch.float64)
    return (vox.to(device), sdf.float().to(device), inv.view(-1, 8).to(device), vijk.to(device))


def shell_cells(res: int = 32, seed: int = 6, face_cells: int = 24):
    """(dam, collision, dry_adjacent) int32 [K,3] cell lists in [0, res)^3.

    Besides the three shells, collision also holds ``face_cells`` random
    cells on the six faces of the grid (where the reference's linear-key
    neighbour lookup wraps) and a few dam cells again (duplicates across
    lists); dry_adjacent repeats some of its own rows.
    """
    g = torch.Generator().manual_seed(seed)
    c = res / 2 + (torch.rand(3, generator=g, dtype=torch.float64) - 0.5) * 0.1 * res
    r = 0.3 * res
    ijk = torch.stack(torch.meshgrid(*[torch.arange(res)] * 3, indexing="ij"), -1).reshape(-1, 3)
    d = ((ijk.double() + 0.5) - c).norm(dim=1) - r
    dam = ijk[d.abs() < 0.9]
    coll = ijk[(d >= 0.9) & (d < 1.9)]
    dry = ijk[(d <= -0.9) & (d > -1.9)]
    fc = torch.randint(0, res, (face_cells, 3), generator=g)
    axis = torch.randint(0, 3, (face_cells,), generator=g)
    side = torch.randint(0, 2, (face_cells,), generator=g) * (res - 1)
    fc[torch.arange(face_cells), axis] = side
    pick = torch.randperm(dam.shape[0], generator=g)[: max(1, dam.shape[0] // 20)]
    coll = torch.cat([coll, fc, dam[pick]])
    coll = coll[torch.randperm(coll.shape[0], generator=g)]
    dry = torch.cat([dry, dry[: dry.shape[0] // 10]])
    return dam.int().contiguous(), coll.int().contiguous(), dry.int().contiguous()
