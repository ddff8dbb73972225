"""SparseDiffDMC: sparse differentiable Dual Marching Cubes
(drop-in for atom3d/mesh_extractor/sparse_diffdmc.py:10-232).

Training mode (a freshly constructed module, inference_mode "auto" or
"weighted_avg") runs the native pipeline: a3d_dmc_prepare (topology),
a3d_dmc_emit (geometry) and, in backward, a3d_dmc_backward, a hand-written
adjoint behind torch.autograd.Function that recomputes per-edge quantities.
Gradients flow to sdf, deform, alpha and beta like the reference's autograd
graph.  The QEF inference mode (a module in eval mode, or inference_mode
"qef") runs a3d_dmc_corner_gradients (unless corner_gradients are given)
and a3d_dmc_emit_qef; it is forward-only.  Per-corner features
(v_features [M, C]) are interpolated to the dual vertices by
a3d_dmc_features (training mode also appends each quad centre's mean) and
are differentiable in training mode (a3d_dmc_features_backward).

The kernels compute in float32.  float64 inputs raise TypeError unless the
caller asks for float32 arithmetic with dtype=torch.float32 (the reference
computes in the input dtype); other floating dtypes are cast to float32 and
the outputs back to the input dtype.
"""

from __future__ import annotations

import ctypes
from typing import NamedTuple, Optional

import torch
import torch.nn as nn

from .. import _lib
from ..constants import CUBE_CORNERS
from .dmc_tables import table


class SparseDiffDMCOutput(NamedTuple):
    vertices: torch.Tensor
    faces: torch.Tensor
    L_dev: torch.Tensor
    p_alpha: torch.Tensor
    n_alpha: torch.Tensor
    v_features: Optional[torch.Tensor] = None


class DmcInputs(ctypes.Structure):
    _fields_ = [
        ("voxel_coords", ctypes.c_void_p),
        ("sdf", ctypes.c_void_p),
        ("cube_idx", ctypes.c_void_p),
        ("deform", ctypes.c_void_p),
        ("alpha", ctypes.c_void_p),
        ("beta", ctypes.c_void_p),
        ("num_cubes", ctypes.c_int64),
        ("num_corners", ctypes.c_int64),
        ("resolution", ctypes.c_int32),
        ("isovalue", ctypes.c_float),
        ("weight_scale", ctypes.c_float),
    ]


_SIGS = {
    "a3d_dmc_workspace_bytes": (ctypes.c_size_t, [ctypes.c_int64, ctypes.c_int64]),
    "a3d_dmc_prepare": (ctypes.c_int, [ctypes.POINTER(DmcInputs), ctypes.c_void_p, ctypes.c_size_t,
                                       ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p]),
    "a3d_dmc_emit": (ctypes.c_int, [ctypes.POINTER(DmcInputs), ctypes.c_void_p, ctypes.c_size_t,
                                    ctypes.POINTER(ctypes.c_int64)] + [ctypes.c_void_p] * 6),
    "a3d_dmc_backward": (ctypes.c_int, [ctypes.POINTER(DmcInputs), ctypes.c_void_p, ctypes.c_size_t,
                                        ctypes.POINTER(ctypes.c_int64)] + [ctypes.c_void_p] * 9),
    "a3d_dmc_features": (ctypes.c_int, [ctypes.POINTER(DmcInputs), ctypes.c_void_p, ctypes.c_size_t,
                                        ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]),
    "a3d_dmc_features_backward": (ctypes.c_int, [ctypes.POINTER(DmcInputs), ctypes.c_void_p, ctypes.c_size_t,
                                                 ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p, ctypes.c_int32,
                                                 ctypes.c_int32] + [ctypes.c_void_p] * 7),
    "a3d_dmc_corner_gradients_workspace_bytes": (ctypes.c_size_t, [ctypes.c_int64, ctypes.c_int64]),
    "a3d_dmc_corner_gradients": (ctypes.c_int, [ctypes.POINTER(DmcInputs), ctypes.c_void_p, ctypes.c_size_t,
                                                ctypes.c_void_p, ctypes.c_void_p]),
    "a3d_dmc_emit_qef": (ctypes.c_int, [ctypes.POINTER(DmcInputs), ctypes.c_void_p, ctypes.c_size_t,
                                        ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p, ctypes.c_float]
                         + [ctypes.c_void_p] * 6),
    "a3d_dmc_backward_qef": (ctypes.c_int, [ctypes.POINTER(DmcInputs), ctypes.c_void_p, ctypes.c_size_t,
                                            ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p, ctypes.c_float]
                             + [ctypes.c_void_p] * 9),
}


def _bind():
    lib = _lib.lib()
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


class _DmcContext:
    """Device inputs + workspace holding the topology between the passes."""

    def __init__(self, vox, sdf, cidx, res, deform, alpha, beta, iso, wscale):
        self.keep = [vox, sdf, cidx, deform, alpha, beta]
        self.inp = DmcInputs(
            vox.data_ptr(), sdf.data_ptr(), cidx.data_ptr(), _lib.ptr(deform), _lib.ptr(alpha), _lib.ptr(beta),
            vox.shape[0], sdf.shape[0], int(res), float(iso), float(wscale),
        )
        self.dev = sdf.device
        self.stream = _lib.stream_ptr(self.dev)
        lib = _bind()
        self.ws = _lib.workspace(lib.a3d_dmc_workspace_bytes(vox.shape[0], sdf.shape[0]), self.dev)
        self.counts = (ctypes.c_int64 * 6)()
        _lib.check("a3d_dmc_prepare", lib.a3d_dmc_prepare(ctypes.byref(self.inp), self.ws.data_ptr(), self.ws.numel(),
                                                          self.counts, self.stream))

    @property
    def sizes(self):
        ns, ng, ne, nq, nv, _ = list(self.counts)
        return ns, ng, nq, nv


def _features(c, feat, with_centres, rows):
    """Dual-vertex features [rows, C] (a3d_dmc_features); an empty tensor
    when there are none."""
    if feat is None:
        return torch.empty(0, device=c.dev)
    C = feat.shape[1]
    out = torch.empty(rows, C, dtype=torch.float32, device=c.dev)
    if c.counts[0] > 0 and c.counts[4] > 0:
        _lib.check("a3d_dmc_features", _bind().a3d_dmc_features(
            ctypes.byref(c.inp), c.ws.data_ptr(), c.ws.numel(), c.counts, feat.data_ptr(), C, int(with_centres),
            out.data_ptr(), c.stream))
    return out


class _DmcFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sdf, deform, alpha, beta, vfeat, vox, cidx, res, iso, wscale):
        c = _DmcContext(vox, sdf, cidx, res, deform, alpha, beta, iso, wscale)
        ns, ng, nq, nv = c.sizes
        dev = sdf.device
        verts = torch.empty(nv + nq, 3, dtype=torch.float32, device=dev)
        faces = torch.empty(4 * nq, 3, dtype=torch.int64, device=dev)
        ldev = torch.empty(ng, dtype=torch.float32, device=dev)
        pa = torch.empty(ng, 3, dtype=torch.float32, device=dev)
        na = torch.empty(ng, 3, dtype=torch.float32, device=dev)
        if ns > 0:
            _lib.check("a3d_dmc_emit", _bind().a3d_dmc_emit(
                ctypes.byref(c.inp), c.ws.data_ptr(), c.ws.numel(), c.counts, verts.data_ptr(), faces.data_ptr(),
                ldev.data_ptr(), pa.data_ptr(), na.data_ptr(), c.stream))
        vf = _features(c, vfeat, True, nv + nq)
        ctx.dmc = c
        ctx.vfeat = vfeat
        ctx.has = (deform is not None, alpha is not None, beta is not None)
        ctx.mark_non_differentiable(faces)
        # outputs the loss does not use arrive as None (null pointers to the
        # backward kernels) instead of zero tensors filled per call
        ctx.set_materialize_grads(False)
        return verts, faces, ldev, pa, na, vf

    @staticmethod
    def backward(ctx, g_verts, g_faces, g_ldev, g_pa, g_na, g_vf):
        c = ctx.dmc
        need = ctx.needs_input_grad
        dev = c.dev
        n, m = c.inp.num_cubes, c.inp.num_corners

        def cont(t):
            return None if t is None else t.contiguous().float()

        g_sdf = torch.zeros(m, dtype=torch.float32, device=dev) if need[0] else None
        g_def = torch.zeros(m, 3, dtype=torch.float32, device=dev) if (need[1] and ctx.has[0]) else None
        g_alpha = torch.zeros(n, 8, dtype=torch.float32, device=dev) if (need[2] and ctx.has[1]) else None
        g_beta = torch.zeros(n, 12, dtype=torch.float32, device=dev) if (need[3] and ctx.has[2]) else None
        gv, gl, gp, gn = cont(g_verts), cont(g_ldev), cont(g_pa), cont(g_na)
        if c.counts[0] > 0 and any(x is not None for x in (g_sdf, g_def, g_alpha, g_beta)):
            _lib.check("a3d_dmc_backward", _bind().a3d_dmc_backward(
                ctypes.byref(c.inp), c.ws.data_ptr(), c.ws.numel(), c.counts, _lib.ptr(gv), _lib.ptr(gl),
                _lib.ptr(gp), _lib.ptr(gn), _lib.ptr(g_sdf), _lib.ptr(g_def), _lib.ptr(g_alpha), _lib.ptr(g_beta),
                c.stream))
        g_feat = None
        vfeat = ctx.vfeat
        if vfeat is not None and g_vf is not None and g_vf.numel() > 0 and c.counts[0] > 0 and c.counts[4] > 0:
            C = vfeat.shape[1]
            nv = int(c.counts[4])
            g_feat = torch.zeros_like(vfeat) if need[4] else None
            scratch = torch.zeros(nv, C, dtype=torch.float32, device=dev)
            _lib.check("a3d_dmc_features_backward", _bind().a3d_dmc_features_backward(
                ctypes.byref(c.inp), c.ws.data_ptr(), c.ws.numel(), c.counts, vfeat.data_ptr(), C, 1,
                cont(g_vf).data_ptr(), scratch.data_ptr(), _lib.ptr(g_feat), _lib.ptr(g_sdf), _lib.ptr(g_alpha),
                _lib.ptr(g_beta), c.stream))
        return g_sdf, g_def, g_alpha, g_beta, g_feat, None, None, None, None, None


class _DmcQefFn(torch.autograd.Function):
    """QEF inference mode.  Differentiable like the reference's eval mode:
    vertices, L_dev, p_alpha and n_alpha w.r.t. sdf, deform, alpha, the
    vertex features and caller-given corner gradients (gradients the library
    estimates carry none, as in the reference)."""

    @staticmethod
    def forward(ctx, sdf, deform, alpha, beta, vfeat, vox, cidx, res, iso, wscale, reg, corner_gradients):
        c = _DmcContext(vox, sdf, cidx, res, deform, alpha, beta, iso, wscale)
        ns, ng, nq, nv = c.sizes
        dev = sdf.device
        lib = _bind()
        if corner_gradients is None:
            m = sdf.shape[0]
            corner_gradients = torch.empty(m, 3, dtype=torch.float32, device=dev)
            gws = _lib.workspace(lib.a3d_dmc_corner_gradients_workspace_bytes(vox.shape[0], m), dev)
            _lib.check("a3d_dmc_corner_gradients", lib.a3d_dmc_corner_gradients(
                ctypes.byref(c.inp), gws.data_ptr(), gws.numel(), corner_gradients.data_ptr(), c.stream))
        verts = torch.empty(nv, 3, dtype=torch.float32, device=dev)
        faces = torch.empty(2 * nq, 3, dtype=torch.int64, device=dev)
        ldev = torch.empty(ng, dtype=torch.float32, device=dev)
        pa = torch.empty(ng, 3, dtype=torch.float32, device=dev)
        na = torch.empty(ng, 3, dtype=torch.float32, device=dev)
        if ns > 0:
            _lib.check("a3d_dmc_emit_qef", lib.a3d_dmc_emit_qef(
                ctypes.byref(c.inp), c.ws.data_ptr(), c.ws.numel(), c.counts, corner_gradients.data_ptr(),
                float(reg), verts.data_ptr(), faces.data_ptr(), ldev.data_ptr(), pa.data_ptr(), na.data_ptr(),
                c.stream))
        vf = _features(c, vfeat, False, nv)
        ctx.dmc = c
        ctx.vfeat = vfeat
        ctx.reg = float(reg)
        ctx.cg = corner_gradients.detach()
        ctx.has = (deform is not None, alpha is not None, beta is not None)
        ctx.mark_non_differentiable(faces)
        ctx.set_materialize_grads(False)
        return verts, faces, ldev, pa, na, vf

    @staticmethod
    def backward(ctx, g_verts, g_faces, g_ldev, g_pa, g_na, g_vf):
        c = ctx.dmc
        need = ctx.needs_input_grad
        dev = c.dev
        n, m = c.inp.num_cubes, c.inp.num_corners

        def cont(t):
            return None if t is None else t.contiguous().float()

        g_sdf = torch.zeros(m, dtype=torch.float32, device=dev) if need[0] else None
        g_def = torch.zeros(m, 3, dtype=torch.float32, device=dev) if (need[1] and ctx.has[0]) else None
        g_alpha = torch.zeros(n, 8, dtype=torch.float32, device=dev) if (need[2] and ctx.has[1]) else None
        g_beta = torch.zeros(n, 12, dtype=torch.float32, device=dev) if (need[3] and ctx.has[2]) else None
        g_cg = torch.zeros(m, 3, dtype=torch.float32, device=dev) if need[11] else None
        gv, gl, gp, gn = cont(g_verts), cont(g_ldev), cont(g_pa), cont(g_na)
        outs = (g_sdf, g_def, g_alpha, g_cg)
        if c.counts[0] > 0 and any(x is not None for x in outs) and any(x is not None for x in (gv, gl, gp, gn)):
            _lib.check("a3d_dmc_backward_qef", _bind().a3d_dmc_backward_qef(
                ctypes.byref(c.inp), c.ws.data_ptr(), c.ws.numel(), c.counts, ctx.cg.data_ptr(), ctx.reg,
                _lib.ptr(gv), _lib.ptr(gl), _lib.ptr(gp), _lib.ptr(gn), _lib.ptr(g_sdf), _lib.ptr(g_def),
                _lib.ptr(g_alpha), _lib.ptr(g_cg), c.stream))
        g_feat = None
        vfeat = ctx.vfeat
        if vfeat is not None and g_vf is not None and g_vf.numel() > 0 and c.counts[0] > 0 and c.counts[4] > 0:
            C = vfeat.shape[1]
            nv = int(c.counts[4])
            g_feat = torch.zeros_like(vfeat) if need[4] else None
            scratch = torch.zeros(nv, C, dtype=torch.float32, device=dev)
            _lib.check("a3d_dmc_features_backward", _bind().a3d_dmc_features_backward(
                ctypes.byref(c.inp), c.ws.data_ptr(), c.ws.numel(), c.counts, vfeat.data_ptr(), C, 0,
                cont(g_vf).data_ptr(), scratch.data_ptr(), _lib.ptr(g_feat), _lib.ptr(g_sdf), _lib.ptr(g_alpha),
                _lib.ptr(g_beta), c.stream))
        return g_sdf, g_def, g_alpha, g_beta, g_feat, None, None, None, None, None, None, g_cg


class SparseDMC(nn.Module):
    """Alias wrapper (reference: sparse_diffdmc.py:20-33)."""

    def __init__(self, *args, **kwargs):
        super().__init__()
        self.module = SparseDiffDMC(*args, **kwargs)

    def forward(self, *args, **kwargs):
        return self.module.forward(*args, **kwargs)


class SparseDiffDMC(nn.Module):
    def __init__(self, device: str = "cuda", dtype: torch.dtype = torch.float32):
        super().__init__()
        self.device = device
        self.dtype = dtype
        for name in ("dmc_table", "num_vd_table", "check_table", "tet_table"):
            self.register_buffer(name, torch.from_numpy(table(name)).to(device))
        self.register_buffer("quad_split_1", torch.tensor([0, 1, 2, 0, 2, 3], dtype=torch.long, device=device))
        self.register_buffer("quad_split_2", torch.tensor([0, 1, 3, 3, 1, 2], dtype=torch.long, device=device))
        self.register_buffer("quad_split_train", torch.tensor([0, 1, 1, 2, 2, 3, 3, 0], dtype=torch.long,
                                                              device=device))
        self.register_buffer("cube_corners", CUBE_CORNERS.to(device).float())
        self.register_buffer("cube_corners_idx", torch.pow(2, torch.arange(8, dtype=torch.long, device=device)))
        self.register_buffer("cube_edges", torch.tensor([0, 1, 1, 5, 4, 5, 0, 4, 2, 3, 3, 7, 6, 7, 2, 6, 2, 0, 3, 1,
                                                         7, 5, 6, 4], dtype=torch.long, device=device))

    def forward(
        self,
        voxel_coords: torch.Tensor,
        sdf: torch.Tensor,
        cube_idx: torch.Tensor,
        resolution: int,
        deform: Optional[torch.Tensor] = None,
        beta: Optional[torch.Tensor] = None,
        alpha: Optional[torch.Tensor] = None,
        gamma: Optional[torch.Tensor] = None,
        v_features: Optional[torch.Tensor] = None,
        isovalue: float = 0.0,
        qef_reg_scale: float = 1e-2,
        weight_scale: float = 0.99,
        inference_mode: str = "auto",
        dtype: Optional[torch.dtype] = None,
        corner_gradients: Optional[torch.Tensor] = None,
    ) -> SparseDiffDMCOutput:
        mode = ("weighted_avg" if self.training else "qef") if inference_mode == "auto" else inference_mode
        if mode not in ("weighted_avg", "qef"):
            raise ValueError(f"SparseDiffDMC: unknown inference_mode {inference_mode!r}")
        _lib.require_cuda(sdf, "sdf")
        dev = sdf.device
        out_dtype = dtype or (sdf.dtype if sdf.dtype.is_floating_point else torch.float32)
        if out_dtype == torch.float64:
            raise TypeError("SparseDiffDMC computes in float32 on the GPU; pass float32 inputs, or "
                            "dtype=torch.float32 to accept float32 arithmetic on float64 inputs")

        def f32(t, shape_last=None):
            if t is None:
                return None
            return t.to(device=dev, dtype=torch.float32).contiguous()

        vox = voxel_coords.to(device=dev, dtype=torch.int64).contiguous()
        cidx = cube_idx.to(device=dev, dtype=torch.int64).contiguous()
        s = f32(sdf)
        vf_in = None
        if v_features is not None:
            if v_features.dim() != 2 or v_features.shape[0] != sdf.shape[0]:
                raise ValueError(f"v_features must be [M, C] with M = {sdf.shape[0]}, got {tuple(v_features.shape)}")
            vf_in = f32(v_features)
        if mode == "qef":
            # alpha moves p_alpha (and the features' interpolation), not the
            # QEF vertices; beta weighs the features; gamma does not enter
            cg = f32(corner_gradients)
            verts, faces, ldev, pa, na, vf = _DmcQefFn.apply(
                s, f32(deform), f32(alpha), f32(beta), vf_in, vox, cidx, int(resolution), float(isovalue),
                float(weight_scale), float(qef_reg_scale), cg)
        else:
            verts, faces, ldev, pa, na, vf = _DmcFn.apply(s, f32(deform), f32(alpha), f32(beta), vf_in, vox, cidx,
                                                          int(resolution), float(isovalue), float(weight_scale))
        if vf_in is None:
            vf = None
        if out_dtype != torch.float32:
            verts, ldev, pa, na = (t.to(out_dtype) for t in (verts, ldev, pa, na))
            if vf is not None:
                vf = vf.to(out_dtype)
        return SparseDiffDMCOutput(vertices=verts, faces=faces, L_dev=ldev, p_alpha=pa, n_alpha=na, v_features=vf)
