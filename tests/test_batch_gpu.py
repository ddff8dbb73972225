"""Batched multi-mesh build + query: per-mesh results against the
single-mesh path and the FP64 oracle, CUDA-graph replay, autotuned launch
shapes, edge cases (single-triangle meshes, meshes without queries) and
the build's error status."""

import numpy as np
import pytest
import torch

from atom3d_b200 import MeshBVH, synthetic
from atom3d_b200.batch import BatchedMeshBVH, UdfTuning, offsets

pytestmark = pytest.mark.gpu


def _small_batch(seed=11, n=10):
    meshes = synthetic.batch_meshes(n, seed=seed, min_level=1, max_level=4, queries_per_tri=8, device="cuda")
    g = torch.Generator(device="cuda").manual_seed(seed)
    # edge cases: a lone triangle and a two-triangle mesh
    tri = torch.tensor([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]], device="cuda")
    meshes.append((tri, torch.tensor([[0, 1, 2]], dtype=torch.int32, device="cuda"),
                   torch.rand(500, 3, device="cuda", generator=g) * 2 - 0.5))
    quad = torch.tensor([[0.0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], device="cuda") + 3.0
    meshes.append((quad, torch.tensor([[0, 1, 2], [0, 2, 3]], dtype=torch.int32, device="cuda"),
                   torch.rand(700, 3, device="cuda", generator=g) * 2 + 2.5))
    return meshes


def _check_against_single(meshes, dist, fid, cp):
    """Each mesh's slice equals what MeshBVH(v, f).udf returns for it."""
    from oracle import orc

    o = 0
    for v, f, q in meshes:
        k = q.shape[0]
        if k == 0:
            continue
        single = MeshBVH(v, f)
        ref = single.udf(q, return_closest=True, return_face_ids=True)
        assert single._bvh.status()["faults"] == 0
        d, fi = dist[o:o + k], fid[o:o + k].long()
        # the minimum of the same FP32 triangle distances: bit-identical
        assert torch.equal(d, ref.distances), float((d - ref.distances).abs().max())
        same = fi == ref.face_ids.long()
        if not bool(same.all()):
            # only exact ties may pick another face: both at the same FP64
            # distance up to FP32 rounding
            qq = q[~same].cpu().numpy()
            vv, ff = v.cpu().numpy(), f.cpu().numpy()
            d_b = orc.tri_dist(vv, ff, qq, fi[~same].cpu().numpy())
            d_s = orc.tri_dist(vv, ff, qq, ref.face_ids[~same].cpu().numpy())
            diag = float((v.max(0).values - v.min(0).values).norm())
            assert np.abs(d_b - d_s).max() <= 1e-6 * diag + 1e-7
            assert float((~same).float().mean()) < 0.05
        o += k


def test_batch_matches_single_mesh_path():
    meshes = _small_batch()
    bb = BatchedMeshBVH([(v, f) for v, f, _ in meshes])
    q = torch.cat([q for _, _, q in meshes])
    dist, fid, cp = bb.udf(q, [q.shape[0] for _, _, q in meshes])
    st = bb.query_status()
    assert st["faults"] == 0 and st["overflow"] == 0
    _check_against_single(meshes, dist, fid, cp)
    assert 0 < int(bb.num_nodes.item()) <= bb.num_faces


def test_batch_against_fp64_oracle(orc):
    meshes = _small_batch(seed=12, n=6)
    bb = BatchedMeshBVH([(v, f) for v, f, _ in meshes])
    q = torch.cat([q for _, _, q in meshes])
    dist, fid, cp = bb.udf(q, [q.shape[0] for _, _, q in meshes])
    o = 0
    for v, f, qm in meshes:
        k = qm.shape[0]
        exact = orc.udf_exact(v.cpu().numpy(), f.cpu().numpy(), qm.cpu().numpy())[0]
        diag = float((v.max(0).values - v.min(0).values).norm())
        err = np.abs(dist[o:o + k].cpu().numpy().astype(np.float64) - exact).max()
        assert err <= 1e-6 * diag + 1e-7, err
        o += k


def test_queries_per_mesh_may_be_empty():
    meshes = _small_batch(seed=13, n=5)
    keep = [(v, f, q if i % 2 == 0 else q[:0]) for i, (v, f, q) in enumerate(meshes)]
    bb = BatchedMeshBVH([(v, f) for v, f, _ in keep])
    q = torch.cat([q for _, _, q in keep])
    dist, fid, cp = bb.udf(q, [q.shape[0] for _, _, q in keep])
    _check_against_single(keep, dist, fid, cp)


def test_graph_replay_and_tuned_shapes_give_identical_results():
    meshes = _small_batch(seed=14, n=12)
    bb = BatchedMeshBVH([(v, f) for v, f, _ in meshes])
    q = torch.cat([q for _, _, q in meshes]).contiguous()
    counts = [q.shape[0] for _, _, q in meshes]
    qoff = offsets(counts, "cuda")
    ref = bb.udf(q, counts)
    info = bb.autotune(q, qoff, sample=4096, leaf_sizes=(2, 4))
    assert info["best"]["pool"] in (32, 64, 128, 256) and info["best"]["blocks_per_sm"] >= 1
    dist = torch.empty_like(ref[0])
    fid = torch.empty_like(ref[1])
    cp = torch.empty_like(ref[2])
    g = bb.capture(q, qoff, dist, fid, cp)
    for _ in range(2):
        dist.zero_()
        g.replay()
    torch.cuda.synchronize()
    bb.check()
    assert bb.query_status()["faults"] == 0
    # the tuned leaf size may build another tree: distances identical, ids up to ties
    assert torch.equal(dist, ref[0])
    _check_against_single(meshes, dist, fid, cp)
    for pool, bps in ((32, 1), (256, 2)):
        d2, f2, c2 = torch.empty_like(dist), torch.empty_like(fid), torch.empty_like(cp)
        bb.udf_into(q, qoff, d2, f2, c2, tuning=UdfTuning(pool, bps, 0, 0))
        assert torch.equal(d2, dist) and torch.equal(f2, fid) and torch.equal(c2, cp)


def test_more_queries_than_one_launch(orc):
    # two launches of the traversal (the second one partial), queries of one
    # mesh split between them
    v, f = synthetic.displaced_sphere(3, 8, 0.05, 7)
    v2 = v * 0.5 + 2.0
    g = torch.Generator().manual_seed(3)
    n1, n2 = (1 << 24) - 1000, 300_000
    q1 = synthetic.mixed_queries(v, f, n1, g).cuda()
    q2 = synthetic.mixed_queries(v2, f, n2, g).cuda()
    bb = BatchedMeshBVH([(v.cuda(), f.cuda()), (v2.cuda(), f.cuda())])
    dist, fid, cp = bb.udf(torch.cat([q1, q2]), [n1, n2])
    assert bb.query_status()["faults"] == 0
    for vm, q, sl in ((v, q1, slice(0, n1)), (v2, q2, slice(n1, n1 + n2))):
        ref = MeshBVH(vm.cuda(), f.cuda()).udf(q, return_face_ids=True)
        assert torch.equal(dist[sl], ref.distances)
        # face ids equal, or tied: both faces at the same FP64 distance within
        # 1e-6 of the box diagonal (the batched tree differs from the single one)
        diff = torch.nonzero(fid[sl].long() != ref.face_ids.long()).flatten()
        if diff.numel():
            qd = q[diff].cpu().numpy()
            a = orc.tri_dist(vm.numpy(), f.numpy(), qd, fid[sl][diff].cpu().numpy())
            b = orc.tri_dist(vm.numpy(), f.numpy(), qd, ref.face_ids[diff].cpu().numpy())
            diag = float((vm.double().max(0).values - vm.double().min(0).values).norm())
            assert np.abs(a - b).max() <= 1e-6 * diag, (diff.numel(), np.abs(a - b).max())


def test_bad_face_index_is_reported():
    v = torch.rand(4, 3, device="cuda")
    f = torch.tensor([[0, 1, 2], [1, 2, 7]], dtype=torch.int32, device="cuda")
    with pytest.raises(ValueError):
        BatchedMeshBVH([(v, f), (v, f[:1])])
