"""Learned conservative distance bound for the closest-point traversal.

No counterpart in the reference.  A Fourier-feature MLP
(3 -> 64 -> 128 -> 128 -> 128 -> 1, ReLU) learns a mesh's unsigned distance
from samples produced by the plain traversal itself; a calibrated margin
turns its prediction into a per-query upper bound that seeds the traversal's
pruning radius (``MeshBVH.udf(points, bound=...)``).  Queries whose bound
turns out too small are re-run without it, so results are identical with or
without the network; the plain method decides which bounds missed.

Training and inference run in hand-written BF16 tensor-core kernels
(csrc/mlp.cu): inference in one tcgen05 kernel with its accumulators in
tensor memory (a3d_mlp_bound), training in mma.sync GEMMs (a3d_gemm_bf16,
a3d_mlp_*); PyTorch only holds the buffers.
"""

from __future__ import annotations

import ctypes
import math
from typing import Optional

import torch

from .. import _lib


class MlpWeights(ctypes.Structure):
    _fields_ = [
        ("w1t", ctypes.c_void_p), ("w2t", ctypes.c_void_p), ("w3t", ctypes.c_void_p),
        ("b1", ctypes.c_void_p), ("b2", ctypes.c_void_p), ("b3", ctypes.c_void_p),
        ("w4", ctypes.c_void_p), ("b4", ctypes.c_float), ("freq", ctypes.c_void_p),
        ("norm", ctypes.c_float * 4), ("scale", ctypes.c_float), ("margin", ctypes.c_float),
        ("log_space", ctypes.c_int32),
    ]


class GemmArgs(ctypes.Structure):
    _fields_ = [
        ("A", ctypes.c_void_p), ("B", ctypes.c_void_p),
        ("sam", ctypes.c_int64), ("sak", ctypes.c_int64), ("sbk", ctypes.c_int64), ("sbn", ctypes.c_int64),
        ("m", ctypes.c_int32), ("n", ctypes.c_int32), ("k", ctypes.c_int32),
        ("bias", ctypes.c_void_p), ("mask", ctypes.c_void_p), ("relu", ctypes.c_int32),
        ("Cf", ctypes.c_void_p), ("accumulate", ctypes.c_int32), ("Cb", ctypes.c_void_p),
    ]


_SIGS = {
    "a3d_mlp_bound": (ctypes.c_int, [ctypes.POINTER(MlpWeights), ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                     ctypes.c_void_p]),
    "a3d_mlp_bound_status": (ctypes.c_int, [ctypes.POINTER(ctypes.c_uint), ctypes.c_void_p]),
    "a3d_gemm_bf16": (ctypes.c_int, [ctypes.POINTER(GemmArgs), ctypes.c_void_p]),
    "a3d_mlp_fourier": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_float), ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p]),
    "a3d_mlp_head": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "a3d_mlp_colsum": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p,
                                      ctypes.c_void_p]),
    "a3d_adam": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                ctypes.c_void_p]),
    "a3d_to_bf16": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]),
}


def _bind():
    lib = _lib.lib()
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


N_FREQ, N_IN, N_HID = 32, 64, 128
# parameter block layout (fp32 masters): W1 [64,128], W2, W3 [128,128] as
# [in, out]; b1, b2, b3, w4 [128]; b4 [1]
_SHAPES = [("W1", (N_IN, N_HID)), ("W2", (N_HID, N_HID)), ("W3", (N_HID, N_HID)), ("b1", (N_HID,)),
           ("b2", (N_HID,)), ("b3", (N_HID,)), ("w4", (N_HID,)), ("b4", (1,))]


class LearnedBound:
    """Per-mesh learned upper bound on the unsigned distance."""

    def __init__(self, lo, hi, device="cuda", sigma: float = 1.5, seed: int = 0, log_space: bool = False):
        """``log_space``: the network learns log(distance + eps) instead of the
        distance, so its error is relative (near-surface queries get tight
        bounds) and the bound is exp(y) * scale + margin."""
        self.dev = torch.device(device)
        self.log_space = bool(log_space)
        self.eps = 1e-4
        self.coverage = None
        lo = torch.as_tensor(lo, dtype=torch.float32)
        hi = torch.as_tensor(hi, dtype=torch.float32)
        c = (lo + hi) * 0.5
        half = float((hi - lo).max()) * 0.5 * 1.25
        self.norm = [float(c[0]), float(c[1]), float(c[2]), 1.0 / half]
        g = torch.Generator().manual_seed(seed)
        self.freq = (torch.randn(N_FREQ, 3, generator=g) * sigma).float().to(self.dev).contiguous()
        sizes = [math.prod(s) for _, s in _SHAPES]
        self.params = torch.zeros(sum(sizes), dtype=torch.float32, device=self.dev)
        self.views = {}
        off = 0
        for (name, shape), sz in zip(_SHAPES, sizes):
            self.views[name] = self.params[off:off + sz].view(shape)
            off += sz
        for name, fan_in in (("W1", N_IN), ("W2", N_HID), ("W3", N_HID)):
            b = math.sqrt(6.0 / fan_in)
            self.views[name].copy_((torch.rand(self.views[name].shape, generator=g) * 2 - 1) * b)
        self.views["w4"].copy_((torch.rand(N_HID, generator=g) * 2 - 1) * math.sqrt(3.0 / N_HID))
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step = 0
        self.scale = 1.0
        self.margin = 0.0
        self._bf16 = {}
        self._refresh_bf16()

    # ---------------------------------------------------------------- helpers
    @property
    def stream(self):
        return _lib.stream_ptr(self.dev)

    def _refresh_bf16(self):
        lib = _bind()
        for name in ("W1", "W2", "W3"):
            w = self.views[name]
            b = self._bf16.get(name)
            if b is None:
                b = torch.empty(w.shape, dtype=torch.bfloat16, device=self.dev)
                self._bf16[name] = b
            _lib.check("a3d_to_bf16", lib.a3d_to_bf16(w.data_ptr(), w.numel(), b.data_ptr(), self.stream))
        # inference layout: transposed [out][in]
        self._t = {k: self._bf16[k].t().contiguous() for k in ("W1", "W2", "W3")}

    def _gemm(self, A, B, sam, sak, sbk, sbn, m, n, k, bias=None, mask=None, relu=False, Cf=None, acc=False, Cb=None):
        a = GemmArgs(A.data_ptr(), B.data_ptr(), sam, sak, sbk, sbn, m, n, k, _lib.ptr(bias), _lib.ptr(mask),
                     int(relu), _lib.ptr(Cf), int(acc), _lib.ptr(Cb))
        _lib.check("a3d_gemm_bf16", _bind().a3d_gemm_bf16(ctypes.byref(a), self.stream))

    # --------------------------------------------------------------- training
    def forward_backward(self, x: torch.Tensor, target: Optional[torch.Tensor], under_weight: float = 4.0):
        """One forward (and backward when ``target`` is given) pass over a
        batch; returns (prediction, loss).  Gradients land in ``self.grads``."""
        lib = _bind()
        n = int(x.shape[0])
        d = self.dev
        bf = torch.bfloat16
        feat = torch.empty(n, N_IN, dtype=bf, device=d)
        nrm = (ctypes.c_float * 4)(*self.norm)
        _lib.check("a3d_mlp_fourier", lib.a3d_mlp_fourier(x.data_ptr(), n, nrm, self.freq.data_ptr(),
                                                          feat.data_ptr(), self.stream))
        h1 = torch.empty(n, N_HID, dtype=bf, device=d)
        h2 = torch.empty_like(h1)
        h3 = torch.empty_like(h1)
        W = self._bf16
        V = self.views
        self._gemm(feat, W["W1"], N_IN, 1, N_HID, 1, n, N_HID, N_IN, bias=V["b1"], relu=True, Cb=h1)
        self._gemm(h1, W["W2"], N_HID, 1, N_HID, 1, n, N_HID, N_HID, bias=V["b2"], relu=True, Cb=h2)
        self._gemm(h2, W["W3"], N_HID, 1, N_HID, 1, n, N_HID, N_HID, bias=V["b3"], relu=True, Cb=h3)
        y = torch.empty(n, dtype=torch.float32, device=d)
        loss = torch.zeros(1, dtype=torch.float32, device=d)
        if target is None:
            _lib.check("a3d_mlp_head", lib.a3d_mlp_head(h3.data_ptr(), n, V["w4"].data_ptr(), V["b4"].data_ptr(),
                                                        None, 1.0, y.data_ptr(), None, None, None, None, self.stream))
            return y, None
        G = {}
        off = 0
        for (name, shape) in _SHAPES:
            sz = math.prod(shape)
            G[name] = self.grads[off:off + sz].view(shape)
            off += sz
        self.grads.zero_()
        dh3 = torch.empty_like(h3)
        _lib.check("a3d_mlp_head", lib.a3d_mlp_head(
            h3.data_ptr(), n, V["w4"].data_ptr(), V["b4"].data_ptr(), target.data_ptr(), float(under_weight),
            y.data_ptr(), dh3.data_ptr(), G["w4"].data_ptr(), G["b4"].data_ptr(), loss.data_ptr(), self.stream))
        # layer 3: dW3 = h2^T dh3, db3 = colsum(dh3), dh2 = (dh3 W3^T) * (h2 > 0)
        self._gemm(h2, dh3, 1, N_HID, N_HID, 1, N_HID, N_HID, n, Cf=G["W3"], acc=True)
        _lib.check("a3d_mlp_colsum", lib.a3d_mlp_colsum(dh3.data_ptr(), n, N_HID, G["b3"].data_ptr(), self.stream))
        dh2 = torch.empty_like(h2)
        self._gemm(dh3, W["W3"], N_HID, 1, 1, N_HID, n, N_HID, N_HID, mask=h2, Cb=dh2)
        self._gemm(h1, dh2, 1, N_HID, N_HID, 1, N_HID, N_HID, n, Cf=G["W2"], acc=True)
        _lib.check("a3d_mlp_colsum", lib.a3d_mlp_colsum(dh2.data_ptr(), n, N_HID, G["b2"].data_ptr(), self.stream))
        dh1 = torch.empty_like(h1)
        self._gemm(dh2, W["W2"], N_HID, 1, 1, N_HID, n, N_HID, N_HID, mask=h1, Cb=dh1)
        self._gemm(feat, dh1, 1, N_IN, N_HID, 1, N_IN, N_HID, n, Cf=G["W1"], acc=True)
        _lib.check("a3d_mlp_colsum", lib.a3d_mlp_colsum(dh1.data_ptr(), n, N_HID, G["b1"].data_ptr(), self.stream))
        return y, loss

    def adam_step(self, lr: float):
        self.step += 1
        _lib.check("a3d_adam", _bind().a3d_adam(self.params.data_ptr(), self.grads.data_ptr(), self.m.data_ptr(),
                                                self.v.data_ptr(), self.params.numel(), float(lr), 0.9, 0.999, 1e-8,
                                                self.step, self.stream))
        self._refresh_bf16()

    def fit(self, x: torch.Tensor, dist: torch.Tensor, epochs: int = 8, batch: int = 32768, lr: float = 2e-3,
            seed: int = 0):
        """Train on (points, plain-traversal distances); returns the loss history."""
        x = x.to(self.dev, torch.float32).contiguous()
        dist = dist.to(self.dev, torch.float32).contiguous()
        if self.log_space:
            dist = torch.log(dist + self.eps)
        n = x.shape[0]
        g = torch.Generator(device=self.dev).manual_seed(seed)
        hist = []
        total = epochs * max(1, n // batch)
        it = 0
        for _ in range(epochs):
            perm = torch.randperm(n, device=self.dev, generator=g)
            for s in range(0, n - batch + 1, batch):
                idx = perm[s:s + batch]
                cur_lr = lr * 0.5 * (1 + math.cos(math.pi * it / total))
                _, loss = self.forward_backward(x[idx].contiguous(), dist[idx].contiguous())
                self.adam_step(cur_lr)
                hist.append(loss)
                it += 1
        return torch.cat(hist).cpu() if hist else torch.zeros(0)

    def predict(self, x: torch.Tensor) -> torch.Tensor:
        """The network's output through the training kernels (log(distance +
        eps) in log space)."""
        y, _ = self.forward_backward(x.to(self.dev, torch.float32).contiguous(), None)
        return y

    def calibrate(self, x: torch.Tensor, dist: torch.Tensor, coverage: float = 0.995, slack: float = 1.02):
        """Choose scale/margin so that ``coverage`` of the samples satisfy
        dist <= max(y, 0) * scale + margin (exp(y) in log space)."""
        raw = self._raw_bound(x)
        self.scale = float(slack)
        excess = dist.to(self.dev).float() - raw * self.scale
        self.margin = max(0.0, float(torch.quantile(excess[:1 << 24], coverage)))
        return self.margin

    def _raw_bound(self, x):
        s, m = self.scale, self.margin
        self.scale, self.margin = 1.0, 0.0
        b = self(x)
        self.scale, self.margin = s, m
        return b

    # -------------------------------------------------------------- inference
    def weights(self) -> MlpWeights:
        V = self.views
        return MlpWeights(self._t["W1"].data_ptr(), self._t["W2"].data_ptr(), self._t["W3"].data_ptr(),
                          V["b1"].data_ptr(), V["b2"].data_ptr(), V["b3"].data_ptr(), V["w4"].data_ptr(),
                          float(V["b4"].item()), self.freq.data_ptr(), (ctypes.c_float * 4)(*self.norm),
                          float(self.scale), float(self.margin), int(self.log_space))

    def __call__(self, x: torch.Tensor, out: Optional[torch.Tensor] = None, weights: Optional[MlpWeights] = None):
        """Per-query bound (fused tcgen05 inference kernel)."""
        x = x.to(self.dev, torch.float32).contiguous()
        out = torch.empty(x.shape[0], dtype=torch.float32, device=self.dev) if out is None else out
        w = self.weights() if weights is None else weights
        _lib.check("a3d_mlp_bound", _bind().a3d_mlp_bound(ctypes.byref(w), x.data_ptr(), x.shape[0],
                                                          out.data_ptr(), self.stream))
        return out


    def status(self) -> int:
        """Status word of the last inference launch on this device (waits
        for it): bit 0 when a tile's tensor-core wait ran out."""
        st = ctypes.c_uint(0)
        _lib.check("a3d_mlp_bound_status", _bind().a3d_mlp_bound_status(ctypes.byref(st), self.stream))
        return int(st.value)


def _time_query(mesh, x, bound, reps: int = 3) -> float:
    bvh = mesh._bvh
    bvh.query(x, bound=bound, want_uvw=False)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        bvh.query(x, bound=bound, want_uvw=False)
    e1.record()
    torch.cuda.synchronize(mesh.device)
    return e0.elapsed_time(e1) / reps


def tune_coverage(lb: "LearnedBound", mesh, x: torch.Tensor, dist: torch.Tensor,
                  coverages=(0.97, 0.99, 0.997, 0.999), scales=(1.0, 1.1, 1.25, 1.5)) -> float:
    """Choose the bound's scale and calibration coverage whose bound makes the
    traversal of the held-out samples fastest (CUDA events on the held-out
    set only; results never depend on the choice).  A looser bound prunes
    less, a tighter one makes more queries restart; the trade-off depends on
    the mesh and the query distribution, so it is measured rather than
    fixed."""
    x = x.to(lb.dev, torch.float32).contiguous()
    d = dist.to(lb.dev).float()
    raw = lb._raw_bound(x)
    best = (float("inf"), coverages[0], 1.0, 0.0)
    for sc in scales:
        excess = (d - raw * sc)[:1 << 24]
        for c in coverages:
            margin = max(0.0, float(torch.quantile(excess, c)))
            ms = _time_query(mesh, x, raw * sc + margin)
            if ms < best[0]:
                best = (ms, c, sc, margin)
    lb.coverage, lb.scale, lb.margin = best[1], best[2], best[3]
    return lb.coverage


def train_for_mesh(mesh, samples: torch.Tensor, epochs: int = 8, coverage: float = 0.995, seed: int = 0,
                   tune: bool = False, log_space: bool = False, sigma: float = 1.5, lr: float = 2e-3):
    """Fit a LearnedBound on plain-traversal distances of ``samples``: a
    random 90% trains it, the other 10% sets its margin.  With ``tune`` the
    bound's scale and the margin's coverage are picked by timing the
    traversal on the held-out samples."""
    lo = mesh.get_bounds()[0].cpu()
    hi = mesh.get_bounds()[1].cpu()
    lb = LearnedBound(lo, hi, device=mesh.device, seed=seed, log_space=log_space, sigma=sigma)
    n = samples.shape[0]
    ntr = int(n * 0.9)
    x = samples.to(mesh.device, torch.float32)
    d = mesh.udf(x)
    # a random split: the held-out tenth follows the samples' distribution
    # whatever order they come in
    perm = torch.randperm(n, generator=torch.Generator().manual_seed(seed + 1)).to(mesh.device)
    tr, ho = perm[:ntr], perm[ntr:]
    lb.fit(x[tr], d[tr], epochs=epochs, seed=seed, lr=lr)
    lb.calibrate(x[ho], d[ho], coverage=coverage)
    lb.coverage = coverage
    if tune:
        tune_coverage(lb, mesh, x[ho], d[ho])
    return lb
