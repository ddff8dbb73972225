"""ctypes binding of libatom3d_b200.so (the C ABI declared in include/atom3d_b200.h).

The library is the only compute path of this package: every public op calls
into it and raises if it is missing or if no CUDA device is present.  There
is no CPU or PyTorch fallback.
"""

from __future__ import annotations

import ctypes
import os
import threading

import torch

from . import build as _build

c_i64 = ctypes.c_int64
c_u32 = ctypes.c_uint32
c_int = ctypes.c_int
c_size = ctypes.c_size_t
c_vp = ctypes.c_void_p
c_fp = ctypes.POINTER(ctypes.c_float)


class BvhView(ctypes.Structure):
    _fields_ = [
        ("nodes", c_vp),
        ("tris", c_vp),
        ("num_nodes", c_i64),
        ("num_tris", c_i64),
        ("lo", ctypes.c_float * 3),
        ("hi", ctypes.c_float * 3),
    ]


class SignData(ctypes.Structure):
    _fields_ = [
        ("face_normals", c_vp),
        ("vertex_pn", c_vp),
        ("edge_pn", c_vp),
        ("he_edge_idx", c_vp),
        ("faces", c_vp),
    ]


# name -> (restype, argtypes)
_SIGNATURES: dict[str, tuple] = {
    "a3d_last_error": (ctypes.c_char_p, []),
    "a3d_version": (ctypes.c_char_p, []),
    "a3d_udf_status": (c_int, [c_vp, ctypes.POINTER(c_u32), c_vp]),
    "a3d_ray_workspace_bytes": (c_size, [c_i64]),
    "a3d_ray_nearest": (c_int, [c_vp, c_vp, c_vp, c_i64, ctypes.c_float, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                                c_vp, c_size, c_vp]),
    "a3d_ray_all_count": (c_int, [c_vp, c_vp, c_vp, c_i64, ctypes.c_float, c_vp, c_vp, c_size, c_vp]),
    "a3d_ray_all_collect": (c_int, [c_vp, c_vp, c_vp, c_i64, ctypes.c_float, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                                    c_vp, c_vp]),
    "a3d_ray_parity_votes": (c_int, [c_vp, c_vp, c_i64, c_vp, ctypes.c_int32, ctypes.c_float, ctypes.c_float, c_vp,
                                     c_vp, c_size, c_vp]),
    "a3d_ray_status": (c_int, [c_vp, ctypes.POINTER(c_u32), c_vp]),
    "a3d_bvh_build_workspace_bytes": (c_size, [c_i64]),
    "a3d_bvh_build": (
        c_int,
        [c_vp, c_i64, c_vp, c_i64, c_int, c_vp, c_i64, c_vp, c_vp, c_size, ctypes.POINTER(c_i64), c_fp, c_vp],
    ),
    "a3d_mesh_normals_workspace_bytes": (c_size, [c_i64, c_i64]),
    "a3d_mesh_normals": (
        c_int,
        [c_vp, c_i64, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp, c_i64, c_vp, ctypes.POINTER(c_i64), c_vp, c_size, c_vp],
    ),
    "a3d_udf_workspace_bytes": (c_size, [c_i64, c_u32]),
    "a3d_udf": (
        c_int,
        [
            ctypes.POINTER(BvhView), c_vp, c_i64, c_vp, c_vp, c_vp, c_vp,
            ctypes.POINTER(SignData), c_vp, c_vp, c_u32, c_vp, c_size, c_vp,
        ],
    ),
    "a3d_udf_backward": (c_int, [c_vp, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "a3d_morton_encode": (c_int, [c_vp, c_i64, c_vp, c_vp]),
    "a3d_morton_decode": (c_int, [c_vp, c_i64, c_int, c_vp, c_vp]),
    "a3d_aabb_hit_workspace_bytes": (c_size, [c_i64]),
    "a3d_aabb_hit": (c_int, [ctypes.POINTER(BvhView), c_vp, c_vp, c_i64, c_vp, c_vp, c_size, c_vp]),
    "a3d_aabb_pairs_workspace_bytes": (c_size, [c_i64]),
    "a3d_aabb_clip_workspace_bytes": (c_size, [c_i64]),
    "a3d_exclusive_scan_workspace_bytes": (c_size, [c_i64]),
    "a3d_exclusive_scan_u32": (c_int, [c_vp, c_i64, c_vp, c_vp, c_size, c_vp]),
    "a3d_sort_pairs_workspace_bytes": (c_size, [c_i64]),
    "a3d_sort_pairs_u64": (c_int, [c_vp, c_vp, c_i64, c_int, c_int, c_vp, c_size, c_vp]),
    "a3d_aabb_pairs_count": (c_int, [ctypes.POINTER(BvhView), c_vp, c_vp, c_i64, c_int, c_vp, c_vp, c_size,
                                     ctypes.POINTER(c_i64), c_vp]),
    "a3d_aabb_pairs_clip": (c_int, [ctypes.POINTER(BvhView), c_vp, c_vp, c_i64, c_vp, c_size, c_vp, c_size, c_i64,
                                    c_vp, ctypes.POINTER(c_i64), c_vp]),
    "a3d_aabb_pairs_write": (c_int, [ctypes.POINTER(BvhView), c_vp, c_vp, c_i64, c_int, c_vp, c_size, c_vp, c_size,
                                     c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "a3d_octree_workspace_bytes": (c_size, [c_int, c_int, c_i64]),
    "a3d_octree_traverse": (
        c_int,
        [ctypes.POINTER(BvhView), c_fp, c_fp, c_int, c_int, c_vp, c_i64, ctypes.POINTER(c_i64), c_vp, c_size, c_vp],
    ),
}

A3D_OK = 0
A3D_ERR_ARGUMENT = 1
A3D_ERR_WORKSPACE = 2
A3D_ERR_CUDA = 3
A3D_ERR_OVERFLOW = 4
A3D_ERR_TIMEOUT = 5
A3D_UDF_SORT_QUERIES = 1
A3D_UDF_ASSUME_SORTED = 2
A3D_UDF_NO_REUSE = 4
A3D_UDF_BOUND_SEEDS = 8

_lib = None
_lock = threading.Lock()


class Atom3dError(RuntimeError):
    """Raised when a C-ABI call returns a non-zero status."""

    def __init__(self, fn: str, status: int, msg: str):
        super().__init__(f"{fn} failed with status {status}: {msg}")
        self.status = status


def library_path() -> str:
    return _build.lib_path()


def load(build_if_missing: bool = False) -> ctypes.CDLL:
    """Load (and bind) the shared library; raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = library_path()
        if not os.path.exists(path):
            if build_if_missing:
                _build.build()
            else:
                raise ImportError(
                    f"atom3d_b200 native library not found at {path}; run `python -m atom3d_b200.build`"
                )
        lib = ctypes.CDLL(path)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def lib() -> ctypes.CDLL:
    return load()


def check(fn: str, status: int) -> None:
    if status != A3D_OK:
        msg = lib().a3d_last_error().decode(errors="replace")
        raise Atom3dError(fn, status, msg)


def require_cuda(t: torch.Tensor, what: str = "tensor") -> None:
    if not t.is_cuda:
        raise RuntimeError(
            f"atom3d_b200 runs on CUDA only: {what} is on {t.device} (no CPU fallback by design)"
        )


def stream_ptr(device: torch.device | None = None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def ptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    return t.data_ptr()


def workspace(nbytes: int, device: torch.device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)


def call(name: str, *args) -> None:
    check(name, getattr(lib(), name)(*args))
