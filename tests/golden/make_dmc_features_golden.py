"""Record the reference SparseDiffDMC with per-corner features and weights.

Runs the reference's pure-PyTorch SparseDiffDMC (atom3d/mesh_extractor/
sparse_diffdmc.py) on the CPU on a small sphere union (40^3, 5 spheres) with
v_features [M, 4], alpha [N, 8] and beta [N, 12]:
  * training mode: vertices, faces, v_features (dual vertices then quad
    centres) and the autograd gradients of
    loss = sum |v|^2 + sum v_features^2 with respect to sdf, v_features,
    alpha and beta;
  * QEF inference mode (eval) with alpha and v_features: vertices, faces,
    p_alpha and v_features.
Only the mesh_extractor package and constants.py are loaded (scratch copy).

Usage: python tests/golden/make_dmc_features_golden.py --reference <Atom3d checkout>
"""

from __future__ import annotations

import argparse
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

from atom3d_b200 import synthetic  # noqa: E402
from make_dmc512_golden import import_reference_dmc  # noqa: E402

OUT = os.path.join(HERE, "dmc_features.npz")
RES = 40


def inputs():
    vox, sdf, cidx, _ = synthetic.dmc_spheres(res=RES, seed=8, n_spheres=5)
    g = torch.Generator().manual_seed(31)
    feat = torch.randn(sdf.shape[0], 4, generator=g)
    alpha = torch.randn(vox.shape[0], 8, generator=g) * 0.5
    beta = torch.randn(vox.shape[0], 12, generator=g) * 0.5
    return vox, sdf, cidx, feat, alpha, beta


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="path of the Atom3d checkout (read only)")
    args = ap.parse_args(argv)
    SparseDiffDMC = import_reference_dmc(args.reference)
    vox, sdf, cidx, feat, alpha, beta = inputs()
    out = {}
    s = sdf.clone().requires_grad_(True)
    f = feat.clone().requires_grad_(True)
    a = alpha.clone().requires_grad_(True)
    b = beta.clone().requires_grad_(True)
    o = SparseDiffDMC(device="cpu")(vox, s, cidx, RES, alpha=a, beta=b, v_features=f)
    ((o.vertices ** 2).sum() + (o.v_features ** 2).sum()).backward()
    out.update(train_vertices=o.vertices.detach().numpy(), train_faces=o.faces.numpy(),
               train_v_features=o.v_features.detach().numpy(), grad_sdf=s.grad.numpy(), grad_feat=f.grad.numpy(),
               grad_alpha=a.grad.numpy(), grad_beta=b.grad.numpy())
    dmc = SparseDiffDMC(device="cpu")
    dmc.eval()
    with torch.no_grad():
        o = dmc(vox, sdf, cidx, RES, alpha=alpha, v_features=feat)
    out.update(eval_vertices=o.vertices.numpy(), eval_faces=o.faces.numpy(), eval_p_alpha=o.p_alpha.numpy(),
               eval_v_features=o.v_features.numpy())
    np.savez_compressed(OUT, res=np.int64(RES), **out)
    print(f"{vox.shape[0]} cubes, {out['train_vertices'].shape[0]} train vertices -> {OUT}")


if __name__ == "__main__":
    main()
