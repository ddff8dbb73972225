"""Record the reference SparseDiffDMC at the full 512^3 sphere-union workload.

Runs the reference's pure-PyTorch SparseDiffDMC (atom3d/mesh_extractor/
sparse_diffdmc.py:76-232) on the CPU, training mode, on
``synthetic.dmc_spheres(512)`` (32 seeded spheres, 2-voxel band, N(0, 1e-3)
noise: about 2.2M active cubes), with loss = sum of squared vertex norms, and
keeps what a fixture can hold:

  faces_sha256       digest of the int64 face array (topology, bit-exact)
  n_vertices, n_faces
  vert_idx, vertices a seeded sample of 4,096 vertex rows
  ldev_idx, L_dev    a seeded sample of 4,096 L_dev entries
  grad_idx, grad_sdf d loss / d sdf at 1,000 seeded corners whose gradient is
                     non-zero (the reference's autograd)
  sdf_sum            float64 sum of the input sdf (checks that the regenerated
                     input is the same)

Only the mesh_extractor package and constants.py are loaded, from a scratch
copy arranged as the package expects.  About 30 s on 8 cores.

Usage: python tests/golden/make_dmc512_golden.py --reference <Atom3d checkout>
"""

from __future__ import annotations

import argparse
import hashlib
import os
import shutil
import sys
import tempfile
import time

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from atom3d_b200 import synthetic  # noqa: E402

OUT = os.path.join(HERE, "dmc512.npz")


def import_reference_dmc(path: str):
    tmp = tempfile.mkdtemp(prefix="atom3d_dmc_ref_")
    pkg = os.path.join(tmp, "atom3d")
    os.makedirs(os.path.join(pkg, "mesh_extractor"), exist_ok=True)
    open(os.path.join(pkg, "__init__.py"), "w").close()
    shutil.copy(os.path.join(path, "atom3d", "constants.py"), os.path.join(pkg, "constants.py"))
    for rel in ("__init__.py", "sparse_diffdmc.py", "tables.py"):
        shutil.copy(os.path.join(path, "atom3d", "mesh_extractor", rel), os.path.join(pkg, "mesh_extractor", rel))
    sys.path.insert(0, tmp)
    from atom3d.mesh_extractor import SparseDiffDMC

    return SparseDiffDMC


def faces_digest(faces: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(faces.astype(np.int64)).tobytes()).hexdigest()


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="path of the Atom3d checkout (read only)")
    args = ap.parse_args(argv)
    SparseDiffDMC = import_reference_dmc(args.reference)
    torch.set_num_threads(os.cpu_count())
    vox, sdf, cidx, _ = synthetic.dmc_spheres(512)
    s = sdf.clone().requires_grad_(True)
    t0 = time.time()
    o = SparseDiffDMC(device="cpu")(vox, s, cidx, 512)
    t1 = time.time()
    (o.vertices ** 2).sum().backward()
    t2 = time.time()
    g = s.grad.numpy()
    rng = np.random.default_rng(512)
    nz = np.nonzero(g != 0)[0]
    grad_idx = np.sort(rng.choice(nz, size=1000, replace=False))
    v = o.vertices.detach().numpy()
    ld = o.L_dev.detach().numpy()
    vert_idx = np.sort(rng.choice(v.shape[0], size=4096, replace=False))
    ldev_idx = np.sort(rng.choice(ld.shape[0], size=min(4096, ld.shape[0]), replace=False))
    np.savez_compressed(OUT, faces_sha256=np.array(faces_digest(o.faces.numpy())),
                        n_vertices=np.int64(v.shape[0]), n_faces=np.int64(o.faces.shape[0]), vert_idx=vert_idx,
                        vertices=v[vert_idx], ldev_idx=ldev_idx, L_dev=ld[ldev_idx], grad_idx=grad_idx,
                        grad_sdf=g[grad_idx], sdf_sum=np.float64(sdf.double().sum()),
                        n_cubes=np.int64(vox.shape[0]), ref_cpu_s=np.array([t1 - t0, t2 - t1]))
    print(f"{vox.shape[0]} cubes, {v.shape[0]} vertices, {o.faces.shape[0]} faces; reference CPU forward "
          f"{t1 - t0:.1f} s, backward {t2 - t1:.2f} s on {torch.get_num_threads()} threads -> {OUT}")


if __name__ == "__main__":
    main()
