"""The C-ABI library loads on a CPU-only host and exports every entry point
declared in include/*.h (no compute call is made here)."""

import ctypes
import os
import re

from conftest import REPO


def declared_symbols():
    syms = set()
    inc = os.path.join(REPO, "include")
    for name in os.listdir(inc):
        if not name.endswith(".h"):
            continue
        text = open(os.path.join(inc, name)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(a3d_[A-Za-z0-9_]+)\s*\(", text):
            syms.add(m.group(1))
    return syms


def test_library_exports_every_declared_symbol(lib):
    syms = declared_symbols()
    assert len(syms) >= 10
    missing = [s for s in sorted(syms) if not hasattr(lib, s)]
    assert not missing, f"undefined entry points: {missing}"


def test_version_and_error_string(lib):
    assert b"sm_100a" in lib.a3d_version()
    assert isinstance(lib.a3d_last_error(), bytes)


def test_argument_errors_are_reported_without_a_gpu(lib):
    # a null mesh is rejected before any CUDA call
    st = lib.a3d_bvh_build(None, 0, None, 0, 0, None, 0, None, None, 0, None, None, None)
    assert st == 1  # A3D_ERR_ARGUMENT
    assert b"empty mesh" in lib.a3d_last_error()


def test_workspace_queries(lib):
    assert lib.a3d_bvh_build_workspace_bytes(1000) > 1000 * 48
    assert lib.a3d_udf_workspace_bytes(1000, 1) > lib.a3d_udf_workspace_bytes(1000, 0)


def test_library_has_no_cuda_runtime_dependency():
    # cudart is linked statically so the .so loads where torch's runtime lives elsewhere
    from atom3d_b200 import _lib

    path = _lib.library_path()
    ctypes.CDLL(path)
    data = open("/proc/self/maps").read()
    assert path in data


def _call(lib, name, *args):
    fn = getattr(lib, name)
    st = fn(*args)
    return st, lib.a3d_last_error()


def test_entry_points_reject_bad_arguments_before_any_device_work(lib):
    """Argument errors come back as A3D_ERR_ARGUMENT with a message, before
    any CUDA call (so they hold on a host without a GPU), the C-ABI
    counterpart of the reference's TORCH_CHECK errors."""
    i64, sz, ci = ctypes.c_int64, ctypes.c_size_t, ctypes.c_int
    cases = [
        ("a3d_udf", (None, None, i64(4), None, None, None, None, None, None, None, ctypes.c_uint32(0), None, sz(0),
                     None), b"invalid bvh"),
        ("a3d_udf_noalloc", (None, None, i64(-1), None, None, None, None, None), b"negative"),
        ("a3d_udf_noalloc", (None, None, i64((1 << 20) + 1), None, None, None, None, None), b"1048576"),
        ("a3d_mesh_normals", (None, i64(0), None, i64(0), None, None, None, None, i64(0), None, None, None, sz(0),
                              None), b"empty mesh"),
        ("a3d_octree_traverse", (None, None, None, ci(0), ci(0), None, i64(0), None, None, sz(0), None),
         b"invalid bvh"),
        ("a3d_flood_fill", (None, i64(0), None, None, sz(0), None, None, None), b"null argument"),
        ("a3d_dmc_prepare", (None, None, sz(0), None, None), b"null argument"),
        ("a3d_dual_graph_count", (None, None, ci(-1), None, None, sz(0), None, None), b"bad argument"),
        ("a3d_ray_nearest", (None, None, None, i64(1), ctypes.c_float(1.0), None, None, None, None, None, None, None,
                             None, sz(0), None), b"invalid bvh"),
    ]
    for name, args, msg in cases:
        st, err = _call(lib, name, *args)
        assert st == 1, (name, st, err)  # A3D_ERR_ARGUMENT
        assert msg in err, (name, err)
