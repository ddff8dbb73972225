"""Generate tests/golden/ray_small.npz by running the reference package's
MeshBVH.intersect_ray on CPU tensors in the build container.

On the CPU the reference answers nearest-hit ray queries with its brute-force
path (MeshBVH._intersect_ray_bruteforce, atom3d/core/mesh_bvh.py:1266-1325):
the same Moller-Trumbore maths as its GPU kernel with a 1e-6 instead of 1e-8
lower bound on t and inf instead of max_t for a miss.  The fixture pins the
oracle's restatement of that maths (hit flags, t, face ids, hit points).

Usage:  python tests/golden/make_ray_golden.py --reference <Atom3d checkout>
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
from make_golden import import_reference  # noqa: E402


def rays(seed: int = 21, n: int = 1500):
    """Half from random points in [-1.5, 1.5]^3 in random directions, half from
    outside the unit sphere aimed at random points inside it."""
    g = torch.Generator().manual_seed(seed)
    h = n // 2
    o1 = torch.rand(h, 3, generator=g) * 3 - 1.5
    d1 = torch.randn(h, 3, generator=g)
    o2 = torch.randn(n - h, 3, generator=g)
    o2 = o2 / o2.norm(dim=1, keepdim=True) * 2.5
    tgt = torch.rand(n - h, 3, generator=g) * 1.2 - 0.6
    d2 = tgt - o2
    o = torch.cat([o1, o2])
    d = torch.cat([d1, d2])
    d = d / d.norm(dim=1, keepdim=True)
    return o.float().contiguous(), d.float().contiguous()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="path of the Atom3d checkout (read only)")
    args = ap.parse_args()
    import_reference(args.reference)
    from atom3d.core.mesh_bvh import MeshBVH

    v, f = synthetic.displaced_sphere(3, 8, 0.05, 7)
    o, d = rays()
    mb = MeshBVH(v, f, device="cpu")
    r = mb.intersect_ray(o, d, max_t=1e10)
    np.savez_compressed(os.path.join(HERE, "ray_small.npz"), v=v.numpy(), f=f.numpy(), o=o.numpy(), d=d.numpy(),
                        hit=r.hit.numpy(), t=r.t.numpy(), face_ids=r.face_ids.numpy(),
                        hit_points=r.hit_points.numpy())
    print("rays", o.shape[0], "hits", int(r.hit.sum()))


if __name__ == "__main__":
    main()
