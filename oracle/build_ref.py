"""Compile the reference's own CUDA extensions for sm_100a (TEST INFRASTRUCTURE ONLY).

Builds ``bvh_cuda`` (atom3d/kernels/bvh_kernels.cu) and ``floodfill_cuda``
(atom3d/kernels/flood_fill_kernels.cu) from the reference sources where they
lie, with the reference's own compiler flags (``-O3 --use_fast_math``,
atom3d/kernels/bvh.py:43-48, atom3d/kernels/flood_fill.py:54-60) and the arch
fixed to sm_100a.  Outputs go to ``oracle/_ref/<name>/<name>.so`` only; the
directory is git-ignored and travels with the working tree, so the GPU tests
and the bench's reference legs can load the reference's kernels on a machine
that has no copy of the reference sources.

The reference's Python layers are not built or copied: ``oracle/ref_gpu.py``
drives these modules through their pybind entry points (``build_bvh``,
``bvh_udf``, ``bvh_aabb_intersect``, ``flood_fill``) and restates the few lines
of host glue around them.

Usage: ``python oracle/build_ref.py --reference <path to the Atom3d checkout>``
(the build takes about three minutes per module).
"""

from __future__ import annotations

import argparse
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")

# module name -> source path inside the reference checkout
MODULES = {
    "bvh_cuda": os.path.join("atom3d", "kernels", "bvh_kernels.cu"),
    "floodfill_cuda": os.path.join("atom3d", "kernels", "flood_fill_kernels.cu"),
}


def so_path(name: str) -> str:
    return os.path.join(OUT, name, name + ".so")


def built() -> bool:
    return all(os.path.exists(so_path(n)) for n in MODULES)


def build(reference: str, force: bool = False, verbose: bool = False) -> list[str]:
    """Build every module whose .so is missing (or all with ``force``)."""
    os.environ["TORCH_CUDA_ARCH_LIST"] = "10.0a"
    from torch.utils.cpp_extension import load

    outs = []
    for name, rel in MODULES.items():
        src = os.path.join(reference, rel)
        if not os.path.exists(src):
            raise FileNotFoundError(src)
        out = so_path(name)
        if force or not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(src):
            bdir = os.path.dirname(out)
            os.makedirs(bdir, exist_ok=True)
            load(name=name, sources=[src], build_directory=bdir, extra_cuda_cflags=["-O3", "--use_fast_math"],
                 verbose=verbose)
        outs.append(out)
    return outs


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", required=True, help="path of the Atom3d checkout (read only)")
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args(argv)
    for p in build(args.reference, force=args.force, verbose=True):
        print(p)


if __name__ == "__main__":
    sys.exit(main())
