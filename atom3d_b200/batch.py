"""Batches of meshes of uneven size: one build and shared persistent queries.

No counterpart in the reference (its MeshBVH holds one mesh).  All meshes'
triangles are sorted together with the mesh id above each triangle's Morton
code, each mesh gets its own radix tree and wide-BVH root inside one shared
node array, and the queries of all meshes are Morton-sorted (mesh id first)
and served by persistent traversal launches whose warps take pools of
queries from a global counter, so small and large meshes balance across the
SMs (launches of at most 16,777,216 queries).  Build and query issue no host
synchronisation, so ``BatchedMeshBVH.capture`` records both in one CUDA
graph; ``autotune`` picks the leaf size and the traversal's launch shape
(pool size, resident blocks per SM) by timing them on a strided sample of
the queries.

Face ids returned are local to each query's mesh, as a per-mesh
``MeshBVH(v, f).udf`` returns them.
"""

from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import torch

from . import _lib
from .core.mesh_bvh import udf_status


class BvhBatch(ctypes.Structure):
    _fields_ = [
        ("nodes", ctypes.c_void_p), ("tris", ctypes.c_void_p), ("num_faces", ctypes.c_int64),
        ("num_meshes", ctypes.c_int32), ("roots", ctypes.c_void_p), ("bounds", ctypes.c_void_p),
    ]


class UdfTuning(ctypes.Structure):
    _fields_ = [("pool", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32), ("leaf_max", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]

    def as_dict(self):
        return {"pool": self.pool, "blocks_per_sm": self.blocks_per_sm, "leaf_max": self.leaf_max}


_vp, _i64, _i32, _sz = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_size_t
_SIGS = {
    "a3d_batch_build_workspace_bytes": (_sz, [_i64, _i32]),
    "a3d_batch_build": (ctypes.c_int, [_vp, _vp, _vp, _vp, _i32, _i64, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp,
                                       _vp, _sz, _vp]),
    "a3d_batch_udf_workspace_bytes": (_sz, [_i64, _i32]),
    "a3d_batch_udf": (ctypes.c_int, [ctypes.POINTER(BvhBatch), _vp, _vp, _i64, _vp, _vp, _vp, _vp,
                                     ctypes.POINTER(UdfTuning), _vp, _vp, _sz, _vp]),
    "a3d_batch_autotune_workspace_bytes": (_sz, [_i64, _i32]),
    "a3d_batch_autotune": (ctypes.c_int, [ctypes.POINTER(BvhBatch), _vp, _vp, _i64, _i64, _vp, _sz,
                                          ctypes.POINTER(UdfTuning), ctypes.POINTER(ctypes.c_float), _vp]),
}


def _bind():
    lib = _lib.lib()
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def offsets(counts: Sequence[int], device) -> torch.Tensor:
    """Exclusive prefix sums [0, c0, c0+c1, ...] as an int64 tensor on ``device``."""
    c = torch.as_tensor(list(counts), dtype=torch.int64)
    return torch.cat([torch.zeros(1, dtype=torch.int64), torch.cumsum(c, 0)]).to(device)


def _aligned(nbytes: int, align: int, device) -> torch.Tensor:
    raw = torch.empty(nbytes + align, dtype=torch.uint8, device=device)
    off = (-raw.data_ptr()) % align
    return raw[off:off + nbytes]


class BatchedMeshBVH:
    """Wide BVHs of many meshes in one node array.

    ``meshes`` is a list of (vertices [V_i,3], faces [F_i,3]) CUDA tensors
    (faces index the mesh's own vertices), or pass the concatenations with
    ``vertex_counts``/``face_counts``.  The build runs at construction unless
    ``build=False``.
    """

    def __init__(self, meshes=None, *, vertices: Optional[torch.Tensor] = None, faces: Optional[torch.Tensor] = None,
                 vertex_counts: Optional[Sequence[int]] = None, face_counts: Optional[Sequence[int]] = None,
                 leaf_max: int = 8, device=None, build: bool = True):
        if meshes is not None:
            vertex_counts = [int(v.shape[0]) for v, _ in meshes]
            face_counts = [int(f.shape[0]) for _, f in meshes]
            device = device or meshes[0][0].device
            vertices = torch.cat([v.to(device).float() for v, _ in meshes]).contiguous()
            faces = torch.cat([f.to(device).int() for _, f in meshes]).contiguous()
        if vertices is None or faces is None or vertex_counts is None or face_counts is None:
            raise ValueError("BatchedMeshBVH needs meshes, or vertices/faces with their per-mesh counts")
        _lib.require_cuda(vertices, "vertices")
        if any(int(c) <= 0 for c in face_counts):
            raise ValueError("every mesh of a batch needs at least one face")
        self.device = vertices.device
        self.num_meshes = len(face_counts)
        self.face_counts = [int(c) for c in face_counts]
        self.num_faces = int(sum(self.face_counts))
        if int(faces.shape[0]) != self.num_faces or int(vertices.shape[0]) != int(sum(vertex_counts)):
            raise ValueError("counts do not match the concatenated arrays")
        self.vertices = vertices.detach().float().contiguous()
        self.faces = faces.int().contiguous()
        self.vert_off = offsets(vertex_counts, self.device)
        self.face_off = offsets(face_counts, self.device)
        self.leaf_max = int(leaf_max)
        n, m = self.num_faces, self.num_meshes
        dev = self.device
        self.nodes = _aligned(n * 64, 64, dev)
        self.tris = _aligned(n * 64, 64, dev)
        self.roots = torch.zeros(m, dtype=torch.int32, device=dev)
        self.bounds = torch.zeros(m, 6, dtype=torch.float32, device=dev)
        self.num_nodes = torch.zeros(1, dtype=torch.int64, device=dev)
        self.build_status = torch.zeros(2, dtype=torch.int32, device=dev)
        self._build_ws = _lib.workspace(_bind().a3d_batch_build_workspace_bytes(n, m), dev)
        self.view = BvhBatch(self.nodes.data_ptr(), self.tris.data_ptr(), n, m, self.roots.data_ptr(),
                             self.bounds.data_ptr())
        self.tuning = UdfTuning(0, 0, self.leaf_max, 0)
        self._udf_ws = None
        if build:
            self.build()
            self.check()

    # ----------------------------------------------------------------- build
    def build(self) -> None:
        """Launch the batched build on the current stream (no host sync)."""
        _lib.check("a3d_batch_build", _bind().a3d_batch_build(
            self.vertices.data_ptr(), self.vert_off.data_ptr(), self.faces.data_ptr(), self.face_off.data_ptr(),
            self.num_meshes, self.num_faces, self.leaf_max, self.nodes.data_ptr(), self.tris.data_ptr(),
            self.roots.data_ptr(), self.bounds.data_ptr(), self.num_nodes.data_ptr(), self.build_status.data_ptr(),
            self._build_ws.data_ptr(), self._build_ws.numel(), _lib.stream_ptr(self.device)))

    def check(self) -> None:
        """Read the build's device status (synchronises)."""
        st = self.build_status.tolist()
        if st[0]:
            raise ValueError("batched build: a face index is out of range for its mesh")
        if st[1]:
            raise RuntimeError("batched build: tree deeper than the collapse's level limit")

    # ----------------------------------------------------------------- query
    def _workspace(self, nq: int) -> torch.Tensor:
        need = _bind().a3d_batch_udf_workspace_bytes(nq, self.num_meshes)
        if self._udf_ws is None or self._udf_ws.numel() < need:
            self._udf_ws = _lib.workspace(need, self.device)
        return self._udf_ws

    def udf_into(self, points: torch.Tensor, query_offsets: torch.Tensor, dist: torch.Tensor, fid: torch.Tensor,
                 cp: torch.Tensor, uvw: Optional[torch.Tensor] = None, stats: Optional[torch.Tensor] = None,
                 tuning: Optional[UdfTuning] = None) -> None:
        """Closest points of all queries into preallocated outputs (no host sync)."""
        nq = int(points.shape[0])
        if points.dtype != torch.float32 or not points.is_contiguous():
            raise ValueError("points must be contiguous float32 [Q,3]")
        ws = self._workspace(nq)
        t = tuning if tuning is not None else self.tuning
        _lib.check("a3d_batch_udf", _bind().a3d_batch_udf(
            ctypes.byref(self.view), points.data_ptr(), query_offsets.data_ptr(), nq, dist.data_ptr(),
            fid.data_ptr(), cp.data_ptr(), _lib.ptr(uvw), ctypes.byref(t), _lib.ptr(stats), ws.data_ptr(),
            ws.numel(), _lib.stream_ptr(self.device)))

    def query_status(self) -> dict:
        """Status words of the last query (synchronises): queries re-run,
        deep-stack overflow, guard faults (must be 0)."""
        return udf_status(self._udf_ws, self.device)

    def udf(self, points: torch.Tensor, query_counts: Sequence[int], return_uvw: bool = False):
        """(distances, mesh-local face ids, closest points[, uvw]) for
        queries concatenated mesh by mesh (``query_counts[m]`` for mesh m)."""
        _lib.require_cuda(points, "points")
        if len(query_counts) != self.num_meshes:
            raise ValueError("one query count per mesh")
        p = points.detach().float().contiguous()
        nq = int(p.shape[0])
        if nq != int(sum(query_counts)):
            raise ValueError("query counts do not match the points")
        qoff = offsets(query_counts, self.device)
        dist = torch.empty(nq, dtype=torch.float32, device=self.device)
        fid = torch.empty(nq, dtype=torch.int32, device=self.device)
        cp = torch.empty(nq, 3, dtype=torch.float32, device=self.device)
        uvw = torch.empty(nq, 3, dtype=torch.float32, device=self.device) if return_uvw else None
        self.udf_into(p, qoff, dist, fid, cp, uvw)
        return (dist, fid, cp, uvw) if return_uvw else (dist, fid, cp)

    # -------------------------------------------------------------- autotune
    def autotune(self, points: torch.Tensor, query_offsets: torch.Tensor, sample: int = 1 << 21,
                 leaf_sizes: Sequence[int] = (2, 4, 8)) -> dict:
        """Pick leaf size and launch shape by timing each on every
        ceil(Q/sample)-th query; rebuilds with the winner.  Returns the
        timings seen."""
        lib = _bind()
        nq = int(points.shape[0])
        ns = min(sample, nq)
        ws = _lib.workspace(lib.a3d_batch_autotune_workspace_bytes(ns, self.num_meshes), self.device)
        seen = {}
        best = None
        for lm in leaf_sizes:
            self.leaf_max = int(lm)
            self.build()
            self.check()
            t = UdfTuning()
            ms = ctypes.c_float(0.0)
            _lib.check("a3d_batch_autotune", lib.a3d_batch_autotune(
                ctypes.byref(self.view), points.data_ptr(), query_offsets.data_ptr(), nq, ns, ws.data_ptr(),
                ws.numel(), ctypes.byref(t), ctypes.byref(ms), _lib.stream_ptr(self.device)))
            t.leaf_max = int(lm)
            seen[int(lm)] = {"sample_ms": float(ms.value), **t.as_dict()}
            if best is None or ms.value < best[0]:
                best = (float(ms.value), t)
        self.tuning = best[1]
        self.leaf_max = int(best[1].leaf_max)
        self.build()
        self.check()
        return {"best": self.tuning.as_dict(), "sample_ms": best[0], "sample_queries": ns, "candidates": seen}

    # ----------------------------------------------------------- CUDA graphs
    def capture(self, points: torch.Tensor, query_offsets: torch.Tensor, dist: torch.Tensor, fid: torch.Tensor,
                cp: torch.Tensor, rebuild: bool = True) -> torch.cuda.CUDAGraph:
        """Record build (when ``rebuild``) + query into one CUDA graph over
        these static buffers; ``graph.replay()`` reruns both."""
        self._workspace(int(points.shape[0]))
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            # one eager pass first so every lazily created resource exists
            if rebuild:
                self.build()
            self.udf_into(points, query_offsets, dist, fid, cp)
            s.synchronize()
            with torch.cuda.graph(g, stream=s):
                if rebuild:
                    self.build()
                self.udf_into(points, query_offsets, dist, fid, cp)
        torch.cuda.current_stream(self.device).wait_stream(s)
        return g
