"""The device-wide exclusive scan and radix sort at sizes where every part
of the tile-sum pass is used: element counts whose tile count reaches the
last warp of the 1024-thread tile-sum block, in several bucket sizes, both
sides of the 2,048-tile switch between the two-launch scan (offsets summed
in each block) and the three-launch scan, and a sort whose digit histogram
(256 x tiles entries) does the same."""

import ctypes

import numpy as np
import pytest
import torch

from atom3d_b200 import _lib

pytestmark = pytest.mark.gpu

TILE = 2048  # scan tile: 256 threads x 8 items


def _scan(x: torch.Tensor) -> torch.Tensor:
    lib = _lib.lib()
    n = x.numel()
    out = torch.empty(n + 1, dtype=torch.int64, device="cuda")
    ws = _lib.workspace(lib.a3d_exclusive_scan_workspace_bytes(n), "cuda")
    _lib.call("a3d_exclusive_scan_u32", x.data_ptr(), n, out.data_ptr(), ws.data_ptr(), ws.numel(),
              _lib.stream_ptr(torch.device("cuda")))
    return out


@pytest.mark.parametrize("n", [0, 1, 2047, 2049, 992 * TILE + 1, 1024 * TILE, 2 * 992 * TILE + 5,
                               3 * 992 * TILE + 77, 6_195_477, 2048 * TILE, 2048 * TILE + 1,
                               17 * 1000 * TILE + 3])
def test_exclusive_scan_matches_cumsum(n):
    g = torch.Generator(device="cuda")
    g.manual_seed(n)
    x = torch.randint(0, 1000, (max(n, 1),), generator=g, device="cuda", dtype=torch.int64)[:n]
    x32 = x.to(torch.int32).contiguous()
    out = _scan(x32).cpu().numpy()
    exp = np.zeros(n + 1, np.int64)
    np.cumsum(x.cpu().numpy(), out=exp[1:])
    assert np.array_equal(out, exp)


def test_radix_sort_with_full_histogram_scan():
    # 256 digit bins x 8,180 tiles of 4,096 keys: the histogram scan's tile
    # count (1,022) reaches the last warp of its tile-sum block
    n = 8180 * 4096 - 123
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    keys = torch.randint(0, 2 ** 62, (n,), generator=g, device="cuda", dtype=torch.int64)
    vals = torch.arange(n, device="cuda", dtype=torch.int32)
    k0 = keys.clone()
    lib = _lib.lib()
    ws = _lib.workspace(lib.a3d_sort_pairs_workspace_bytes(n), "cuda")
    _lib.call("a3d_sort_pairs_u64", keys.data_ptr(), vals.data_ptr(), n, 0, 64, ws.data_ptr(), ws.numel(),
              _lib.stream_ptr(torch.device("cuda")))
    ref, order = torch.sort(k0, stable=True)
    assert torch.equal(keys, ref)
    assert torch.equal(vals.long(), order)
