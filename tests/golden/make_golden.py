"""Generate the golden fixtures under tests/golden/ by running the reference
package (Luo-Yihao/Atom3d) on the CPU of the build container.

The reference is imported from a scratch copy (its JIT build writes into its
own tree); its CUDA kernels cannot run without a GPU, so only host-side and
pure-PyTorch parts are recorded:

  morton.npz        OctreeIndexer._ijk_to_morton / _morton_to_ijk
  bvh_small.npz     build_bvh (host SAH build) nodes/triangles of the
                    level-3 and udf-small meshes (for the reference-tree
                    traversal restated in the oracle)
  normals.npz       MeshBVH pseudo-normal precompute (face normals, angles,
                    vertex/edge pseudo-normals, half-edge -> edge map)
  sign.npz          MeshBVH._compute_sign on closest points produced by the
                    oracle's restatement of bvh_udf_kernel over the
                    reference tree
  octree_cpu.npz    CPU octree_traverse (AABB-only broadphase: a superset
                    of the SAT result) on a small mesh
  dmc_small.npz     SparseDiffDMC forward (train and eval) and autograd
                    gradients w.r.t. sdf and deform on a small sphere union

Usage:  python tests/golden/make_golden.py --reference <Atom3d checkout>
"""

from __future__ import annotations

import argparse
import os
import shutil
import sys
import tempfile

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from atom3d_b200 import synthetic  # noqa: E402
from oracle import orc  # noqa: E402


def import_reference(path: str):
    tmp = tempfile.mkdtemp(prefix="atom3d_ref_")
    shutil.copytree(os.path.join(path, "atom3d"), os.path.join(tmp, "atom3d"))
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0")
    sys.path.insert(0, tmp)
    import atom3d  # noqa: F401

    return atom3d


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="path of the Atom3d checkout (read only)")
    args = ap.parse_args()
    atom3d = import_reference(args.reference)
    from atom3d.grid.octree_indexer import OctreeIndexer
    from atom3d.core.mesh_bvh import MeshBVH
    from atom3d.kernels.bvh import get_bvh_kernels
    from atom3d.mesh_extractor import SparseDiffDMC

    torch.manual_seed(0)
    g = torch.Generator().manual_seed(11)

    # ---- Morton -------------------------------------------------------------
    oc = OctreeIndexer(max_level=10, device="cpu")
    ijk = torch.randint(0, 1024, (4096, 3), generator=g, dtype=torch.int64)
    ijk[:8] = torch.tensor([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1023, 1023, 1023], [5, 9, 3],
                            [512, 0, 511], [1, 2, 4]])
    m = oc._ijk_to_morton(ijk)
    back = oc._morton_to_ijk(m, 10)
    back5 = oc._morton_to_ijk(m, 5)
    np.savez_compressed(os.path.join(HERE, "morton.npz"), ijk=ijk.numpy(), morton=m.numpy(), ijk_l10=back.numpy(),
                        ijk_l5=back5.numpy())

    # ---- reference host BVH build --------------------------------------------
    k = get_bvh_kernels()
    v3, f3 = synthetic.icosphere(3)
    vs, fs, qs = synthetic.udf_small(n_queries=4000)
    n3, t3 = k.build_bvh(v3.contiguous(), f3.contiguous(), 4)
    ns, ts = k.build_bvh(vs.contiguous(), fs.contiguous(), 4)
    np.savez_compressed(os.path.join(HERE, "bvh_small.npz"), v3=v3.numpy(), f3=f3.numpy(), nodes3=n3.numpy(),
                        tris3=t3.numpy(), vs=vs.numpy(), fs=fs.numpy(), nodes_s=ns.numpy(), tris_s=ts.numpy(),
                        qs=qs.numpy())

    # ---- pseudo-normals -----------------------------------------------------------
    mb = MeshBVH(vs, fs, device="cpu")
    np.savez_compressed(os.path.join(HERE, "normals.npz"), face_normals=mb._face_normals.numpy(),
                        face_angles=mb._face_angles.numpy(), vertex_pn=mb._vertex_pn.numpy(),
                        edge_pn=mb._edge_pn.numpy(), he_edge_idx=mb._he_edge_idx.numpy())

    # ---- sign on reference-tree closest points --------------------------------------
    d, fid, cp, uvw = orc.ref_bvh_udf(ns.numpy(), ts.numpy(), qs.numpy())
    signs = mb._compute_sign(qs, torch.from_numpy(cp), torch.from_numpy(fid), uvw=torch.from_numpy(uvw))
    np.savez_compressed(os.path.join(HERE, "sign.npz"), dist=d, fid=fid, cp=cp, uvw=uvw, signs=signs.numpy())

    # ---- CPU octree (AABB-only superset) --------------------------------------------------
    vo, fo = synthetic.displaced_sphere(3, 8, 0.05, 2)
    bounds = torch.tensor([[-1.5] * 3, [1.5] * 3])
    mo = MeshBVH(vo, fo, device="cpu")
    oc5 = OctreeIndexer(max_level=5, bounds=bounds, device="cpu")
    cand = oc5.octree_traverse(mo, min_level=2)
    np.savez_compressed(os.path.join(HERE, "octree_cpu.npz"), v=vo.numpy(), f=fo.numpy(), cand=cand.numpy())

    # ---- DMC ---------------------------------------------------------------------------------
    vox, sdf, cidx, vijk = synthetic.dmc_spheres(res=48, seed=5, n_spheres=6)
    res = 48
    gd = torch.Generator().manual_seed(21)
    deform = (torch.randn(sdf.shape[0], 3, generator=gd) * 0.002).float()
    out = {}
    for mode in ("train", "eval"):
        dmc = SparseDiffDMC(device="cpu")
        if mode == "eval":
            dmc.eval()
        s = sdf.clone().requires_grad_(True)
        de = deform.clone().requires_grad_(True)
        o = dmc(vox, s, cidx, res, deform=de)
        loss = (o.vertices ** 2).sum()
        loss.backward()
        out[f"{mode}_vertices"] = o.vertices.detach().numpy()
        out[f"{mode}_faces"] = o.faces.numpy()
        out[f"{mode}_L_dev"] = o.L_dev.detach().numpy()
        out[f"{mode}_p_alpha"] = o.p_alpha.detach().numpy()
        out[f"{mode}_n_alpha"] = o.n_alpha.detach().numpy()
        out[f"{mode}_grad_sdf"] = s.grad.numpy()
        out[f"{mode}_grad_deform"] = de.grad.numpy()
    # weighted variant: alpha / beta given
    dmc = SparseDiffDMC(device="cpu")
    ga = torch.Generator().manual_seed(22)
    alpha = torch.randn(vox.shape[0], 8, generator=ga) * 0.5
    beta = torch.randn(vox.shape[0], 12, generator=ga) * 0.5
    s = sdf.clone().requires_grad_(True)
    o = dmc(vox, s, cidx, res, alpha=alpha, beta=beta)
    (o.vertices ** 2).sum().backward()
    out["ab_vertices"] = o.vertices.detach().numpy()
    out["ab_faces"] = o.faces.numpy()
    out["ab_grad_sdf"] = s.grad.numpy()
    out["ab_L_dev"] = o.L_dev.detach().numpy()
    np.savez_compressed(os.path.join(HERE, "dmc_small.npz"), vox=vox.numpy(), sdf=sdf.numpy(), cidx=cidx.numpy(),
                        deform=deform.numpy(), alpha=alpha.numpy(), beta=beta.numpy(), res=np.int64(res), **out)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
