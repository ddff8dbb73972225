"""The allocation-free closest-point entry point (a3d_udf_noalloc).

It exists for callers that may not call cudaMalloc (an application that owns
all device memory, or a loop where an allocation would synchronise the
device): its scratch is a file-scope device array instead of a workspace.
This file sorts last so that a failure here leaves every other test run.
Two calls in a row are checked against the regular entry point a3d_udf on
the same inputs, with the distance tolerance the UDF tests use.
"""

import ctypes

import numpy as np
import pytest
import torch

from atom3d_b200 import MeshBVH, _lib, synthetic

pytestmark = pytest.mark.gpu

MAX_QUERIES = 1 << 20


def noalloc_fn():
    fn = _lib.lib().a3d_udf_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.POINTER(_lib.BvhView), ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return fn


def call_noalloc(mesh, q):
    n = q.shape[0]
    d = torch.empty(n, device="cuda")
    f = torch.empty(n, dtype=torch.int32, device="cuda")
    cp = torch.empty(n, 3, device="cuda")
    uvw = torch.empty(n, 3, device="cuda")
    st = noalloc_fn()(ctypes.byref(mesh._bvh.view), q.data_ptr(), n, d.data_ptr(), f.data_ptr(), cp.data_ptr(),
                      uvw.data_ptr(), _lib.stream_ptr(q.device))
    _lib.check("a3d_udf_noalloc", st)
    return d, f, cp, uvw


def test_noalloc_matches_regular_entry_point_twice():
    v, f, _ = synthetic.udf_small(n_queries=1)
    mesh = MeshBVH(v.cuda(), f.cuda())
    diag = float((v.max(0).values - v.min(0).values).norm())
    g = torch.Generator().manual_seed(17)
    for n in (200_000, MAX_QUERIES):  # two calls in a row, different sizes
        q = (torch.rand(n, 3, generator=g) * 3.0 - 1.5).cuda()
        d, fid, cp, uvw = call_noalloc(mesh, q)
        rd, rf, rcp, ruvw = mesh._bvh.query(q)
        torch.cuda.synchronize()
        assert torch.abs(d - rd).max().item() <= 1e-6 * diag
        assert torch.abs(cp - rcp).max().item() <= 1e-6 * diag
        assert torch.equal(fid, rf)
        assert np.isfinite(d.cpu().numpy()).all()


def test_noalloc_status_words_readable():
    """A caller without the scratch address still reads the last call's
    status words (re-runs, overflow, faults) through the accessor."""
    v, f, _ = synthetic.udf_small(n_queries=1)
    mesh = MeshBVH(v.cuda(), f.cuda())
    q = (torch.rand(50_000, 3, generator=torch.Generator().manual_seed(3)) * 3.0 - 1.5).cuda()
    call_noalloc(mesh, q)
    fn = _lib.lib().a3d_udf_noalloc_status
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    st = (ctypes.c_uint32 * 4)(7, 7, 7, 7)
    _lib.check("a3d_udf_noalloc_status", fn(ctypes.addressof(st), _lib.stream_ptr(q.device)))
    assert st[1] == 0 and st[2] == 0 and st[3] == 0
    assert st[0] < q.shape[0]


def test_noalloc_rejects_oversized_batches():
    v, f, _ = synthetic.udf_small(n_queries=1)
    mesh = MeshBVH(v.cuda(), f.cuda())
    q = torch.zeros(MAX_QUERIES + 1, 3, device="cuda")
    n = q.shape[0]
    out = torch.empty(n, device="cuda")
    st = noalloc_fn()(ctypes.byref(mesh._bvh.view), q.data_ptr(), n, out.data_ptr(), out.data_ptr(),
                      out.data_ptr(), None, _lib.stream_ptr(q.device))
    assert st == _lib.A3D_ERR_ARGUMENT
    assert b"1048576" in _lib.lib().a3d_last_error()
