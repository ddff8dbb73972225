"""Per-query traversal counts of the plain closest-point method on the
reference's binary SAH tree, for the 1.31M-triangle benchmark mesh.

Builds the tree with the reference's own host builder (build_bvh, run on the
CPU of the build container from a scratch copy of the reference), then runs
the oracle's instrumented restatement of bvh_udf_kernel over a 16,384-query
sample of the benchmark distribution.  Writes udf_large_counts.json, which
bench.py uses for the roofline's algorithmic bytes per query:
    32 B compulsory + 24 B x node box evaluations + 36 B x triangle evaluations.
"""

import json
import os
import sys
import time

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from make_golden import import_reference  # noqa: E402

from atom3d_b200 import synthetic  # noqa: E402
from oracle import orc  # noqa: E402


def main():
    import argparse

    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="path of the Atom3d checkout (read only)")
    import_reference(ap.parse_args().reference)
    from atom3d.kernels.bvh import get_bvh_kernels

    v, f, q = synthetic.udf_large()
    sample = q[torch.randperm(q.shape[0], generator=torch.Generator().manual_seed(0))[:16384]].contiguous()
    t0 = time.time()
    nodes, tris = get_bvh_kernels().build_bvh(v.contiguous(), f.contiguous(), 4)
    t_build = time.time() - t0
    nn, nt = orc.ref_bvh_udf_counts(nodes.numpy(), tris.numpy(), sample.numpy())
    out = {
        "mesh": "udf_large (icosphere L8, 16 sinusoids, seed 3)",
        "triangles": int(f.shape[0]),
        "reference_nodes": int(nodes.shape[0]),
        "sample_queries": int(sample.shape[0]),
        "nodes_per_query": nn / sample.shape[0],
        "tris_per_query": nt / sample.shape[0],
        "reference_host_build_s": t_build,
    }
    with open(os.path.join(HERE, "udf_large_counts.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print(out)


if __name__ == "__main__":
    main()
